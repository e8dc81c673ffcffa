// Pass kernels of the 2^13-point transform.
#include "ntt_impl.cuh"

namespace fides {
void ntt_transform_13(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                       cudaStream_t s) {
  nttk::run_transform<13>(c, a, L, inverse, in, out, s);
}
}  // namespace fides
