// Negacyclic NTT / INTT over lists of limbs.
//
// Replaces the reference's NTT_/INTT_/NTTBatch_ kernels (src/NTT.cu:42-802) and their
// launchers ApplyNTT/ApplyINTT (src/CKKS/LimbPartition.cu:433-550).  Same transform
// (forward: Cooley-Tukey with bit-reversed psi powers, output in bit-reversed EVALUATION
// order; inverse: Gentleman-Sande with N^-1 folded into the last stage), a different
// schedule:
//   * N = 2^LOG1 x 2^LOG2.  Pass COL runs global stages [0, LOG1) on strided columns,
//     pass ROW runs stages [LOG1, logN) on contiguous rows.  Forward = COL then ROW,
//     inverse = ROW then COL; each pass reads and writes every limb once.
//   * each thread keeps 2^LOGE elements in registers and runs LOGE stages per chunk;
//     chunks exchange through padded shared memory (conflict-free);
//   * Harvey lazy butterflies: values stay in [0, 4q) (forward) / [0, 2q) (inverse)
//     between stages, one 64-bit Shoup product per butterfly, so primes must be < 2^62;
//   * one launch covers any list of limbs (any polynomials, any levels): blockIdx.y
//     indexes a limb descriptor (pointer + prime id) passed by value.
#pragma once
#include <cuda_runtime.h>

#include "context.hpp"

namespace fides {

struct LimbRef {
  uint64_t* ptr;
  int prime;
  int pad;
};

constexpr int MAX_NTT_LIMBS = 1024;

struct NttLimbList {
  int n;
  int pad;
  LimbRef limbs[MAX_NTT_LIMBS];
};

// Launch a full forward or inverse transform over `n` limbs (any n; split internally).
void ntt_limbs(Context* c, const LimbRef* limbs, int n, bool inverse, cudaStream_t s);
// Convenience: n_polys polynomials of `n_limbs` consecutive limbs starting at `data`,
// limb i of each poly using prime id prime_ids[i].
void ntt_polys(Context* c, uint64_t* data, int n_polys, int n_limbs, const int* prime_ids, bool inverse,
               cudaStream_t s);

}  // namespace fides
