#pragma once
// CKKS slot encode / decode on the device (encode.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "context.hpp"

namespace fides {
// n_pts plaintexts of n_slots complex slots ((re, im) doubles, device) at `scale` -> level limbs
// each in EVALUATION form, out = [n_pts][level][N].
void op_encode(Context* c, const double* slots, int n_slots, int n_pts, double scale, int level, uint64_t* out,
               cudaStream_t s);
// op_encode into the extended basis: level Q limbs followed by the first `special` special
// limbs, out = [n_pts][level + special][N].
void op_encode_ext(Context* c, const double* slots, int n_slots, int n_pts, double scale, int level, int special,
                   uint64_t* out, cudaStream_t s);
// n_pts plaintexts [n_pts][level][N] (EVALUATION form; limb 0 is read) -> n_slots complex slots
// each, divided by `scale`, slots = [n_pts][n_slots][2] doubles (device).
void op_decode(Context* c, const uint64_t* pts, int level, int n_pts, int n_slots, double scale, double* slots,
               cudaStream_t s);
}  // namespace fides
