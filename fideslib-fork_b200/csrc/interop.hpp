#pragma once
// Interop with the reference's raw host formats (interop.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "context.hpp"

namespace fides {
// limbs: [n_polys][level] host pointers; format 0 = EVALUATION, 1 = COEFFICIENT; natural = 1:
// evaluation vectors in natural (not bit-reversed) order.  out / in: [n_polys][level][N] device.
void op_ct_import(Context* c, int n_polys, const uint64_t* const* limbs, const uint64_t* moduli, int level,
                  int format, int natural, uint64_t* out, cudaStream_t s);
void op_ct_export(Context* c, int n_polys, const uint64_t* in, int level, int format, int natural,
                  uint64_t* const* limbs, cudaStream_t s);
// limbs: [2][dnum][n_q + K] host pointers (null = a zero limb) -> a device key (cudaMalloc).
uint64_t* op_key_import(Context* c, const uint64_t* const* limbs, int natural, cudaStream_t s);
}  // namespace fides
