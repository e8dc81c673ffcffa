// Pass kernels of the 2^10-point transform.
#include "ntt_impl.cuh"

namespace fides {
void ntt_transform_10(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                       cudaStream_t s) {
  nttk::run_transform<10>(c, a, L, inverse, in, out, s);
}
}  // namespace fides
