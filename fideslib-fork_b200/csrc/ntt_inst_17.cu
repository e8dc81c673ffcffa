// Pass kernels of the 2^17-point transform.
#include "ntt_impl.cuh"

namespace fides {
void ntt_transform_17(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                       cudaStream_t s) {
  nttk::run_transform<17>(c, a, L, inverse, in, out, s);
}
}  // namespace fides
