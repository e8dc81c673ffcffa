// Pass kernels of the 2^15-point transform.
#include "ntt_impl.cuh"

namespace fides {
void ntt_transform_15(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                       cudaStream_t s) {
  nttk::run_transform<15>(c, a, L, inverse, in, out, s);
}
}  // namespace fides
