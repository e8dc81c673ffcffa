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
//   * each thread keeps 2^LE elements in registers (16, or 8 at N >= 2^15 where the
//     autotuner picks it) and runs LE stages per chunk; chunks exchange through padded
//     shared memory;
//   * lazy butterflies with one 64-bit Shoup product each (primes < 2^62): the forward
//     transform skips every conditional subtraction for q < 2^58 (values stay below 35q)
//     and uses Harvey's [0, 4q) form otherwise; the inverse tracks a bound B (a multiple
//     of q) and subtracts only once B passes 2^62;
//   * one launch covers any list of limbs (any polynomials, any levels): blockIdx.y
//     indexes a limb descriptor (pointer + prime id) passed by value;
//   * the first pass may read from a separate source (out of place) or compute its input
//     (prologue), and the last pass may combine its result with other operands before
//     storing (epilogue) -- the reference's NTT fusion modes (src/NTT.cuh:39-69,
//     src/NTTfusions.cuh:12-336) as compile-time variants.
#pragma once
#include <cuda_runtime.h>

#include "context.hpp"

namespace fides {

// What the first pass loads.
enum NttIn {
  IN_PLAIN = 0,    // x = src[i]  (src = ptr when in place)
  IN_MUL = 1,      // inverse only: x = src[i] * pro[i] mod q   (tensor term a1 b1)
  IN_SWITCH = 2,   // forward only: x = SwitchModulus(pro[i]) from prime aux - 1 (rescale)
  IN_CONV_SW = 3,  // forward only: x = src[i] + P SwitchModulus(pro[i]) from prime aux - 1
  IN_ADD_PMUL = 4, // inverse only: x = src[i] + P pro[i]
  IN_SIGNED = 5,   // forward only: x = pro[i] read as a signed 64-bit integer, reduced mod q (encode)
};
// What the last pass stores to ptr.
enum NttOut {
  OUT_PLAIN = 0,
  OUT_MODDOWN = 1,   // forward only: out = (ep0[i] - v) P^-1 (+ ep1[i])     (ModDown finish)
  OUT_RESCALE = 2,   // forward only: out = qinv_l ep0[i] + QlQlInv_l v, l = aux (rescale finish)
  OUT_MDRS = 3,      // forward only: out = (ep0[i] - v) (P q_(l-1))^-1 (+ q_(l-1)^-1 ep1[i]), l = aux
  OUT_SUB_PINV = 4,  // inverse only: out = (v - ep0[i]) P^-1
};

struct LimbRef {
  uint64_t* ptr;          // output (and input of the first pass when src is null)
  const uint64_t* src;    // optional input of the first pass
  const uint64_t* pro;    // prologue operand
  const uint64_t* ep0;    // epilogue operands
  const uint64_t* ep1;
  int prime;
  int aux;  // IN_SWITCH / IN_CONV_SW / OUT_RESCALE / OUT_MDRS: the level l being rescaled (top prime l - 1)
  uint64_t pad;
};

inline LimbRef lref(uint64_t* p, int prime) { return LimbRef{p, nullptr, nullptr, nullptr, nullptr, prime, 0, 0}; }

#ifndef FIDES_MAX_NTT_LIMBS
#define FIDES_MAX_NTT_LIMBS 448
#endif
constexpr int MAX_NTT_LIMBS = FIDES_MAX_NTT_LIMBS;

struct NttLimbList {
  int n;
  int pad;
  LimbRef limbs[MAX_NTT_LIMBS];
};

// Launch a full forward or inverse transform over `n` limbs (any n; split internally).
// The prologue/epilogue modes apply to every limb of the call.
void ntt_limbs(Context* c, const LimbRef* limbs, int n, bool inverse, cudaStream_t s, NttIn in = IN_PLAIN,
               NttOut out = OUT_PLAIN);
// Convenience: n_polys polynomials of `n_limbs` consecutive limbs starting at `data`,
// limb i of each poly using prime id prime_ids[i].
void ntt_polys(Context* c, uint64_t* data, int n_polys, int n_limbs, const int* prime_ids, bool inverse,
               cudaStream_t s);

}  // namespace fides
