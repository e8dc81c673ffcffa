// Pass kernels of the 2^12-point transform.
#include "ntt_impl.cuh"

namespace fides {
void ntt_transform_12(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                       cudaStream_t s) {
  nttk::run_transform<12>(c, a, L, inverse, in, out, s);
}
}  // namespace fides
