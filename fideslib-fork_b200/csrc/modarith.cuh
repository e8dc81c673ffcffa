// Exact 64-bit modular arithmetic for residues modulo primes q < 2^62.
//
// Replaces the reference's modmult family (src/ModMult.cuh:42-297) and modadd/modsub
// (src/AddSub.cuh:37-50).  Two primitives carry everything:
//   * Shoup multiplication by a precomputed constant w (w' = floor(w 2^64 / q)): exact for
//     any 64-bit x, result in [0, 2q) ("lazy") or [0, q);
//   * 128-bit reduction of an accumulated sum of products, by splitting x = hi 2^64 + lo and
//     Shoup-multiplying hi by R = 2^64 mod q and lo by 1.  This replaces the reference's
//     128-bit `%` (modreduce<ALGO_NATIVE>, ModMult.cuh:287-297), a software division.
#pragma once
#include <cstdint>

namespace fides {

struct __align__(16) DevPrime {
  uint64_t q;     // the prime
  uint64_t q2;    // 2q
  uint64_t one_s; // floor(2^64 / q): Shoup companion of 1
  uint64_t r64;   // 2^64 mod q
  uint64_t r64_s; // Shoup companion of r64
  uint64_t ninv;  // N^-1 mod q
  uint64_t ninv_s;
  uint64_t pad;
};

__host__ __device__ __forceinline__ uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// x * w mod q in [0, 2q), any x < 2^64, w < q, ws = floor(w 2^64 / q).
__host__ __device__ __forceinline__ uint64_t shoup_lazy(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
  return x * w - mulhi64(x, ws) * q;
}
__host__ __device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t m) { return x >= m ? x - m : x; }
__host__ __device__ __forceinline__ uint64_t shoup(uint64_t x, uint64_t w, uint64_t ws, uint64_t q) {
  return csub(shoup_lazy(x, w, ws, q), q);
}
__host__ __device__ __forceinline__ uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }
__host__ __device__ __forceinline__ uint64_t submod(uint64_t a, uint64_t b, uint64_t q) {
  return a >= b ? a - b : a + q - b;
}

// 128-bit accumulator (lo, hi).
struct U128 {
  uint64_t lo, hi;
};

__device__ __forceinline__ void mac128(U128& acc, uint64_t a, uint64_t b) {
  uint64_t lo = a * b;
  uint64_t hi = __umul64hi(a, b);
  asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;" : "+l"(acc.lo), "+l"(acc.hi) : "l"(lo), "l"(hi));
}

// Full reduction of a 128-bit value modulo q (q < 2^62).
__device__ __forceinline__ uint64_t reduce128(U128 x, const DevPrime& p) {
  uint64_t r = shoup_lazy(x.hi, p.r64, p.r64_s, p.q) + shoup_lazy(x.lo, 1, p.one_s, p.q);  // < 4q
  return csub(csub(r, p.q2), p.q);
}

// a * b mod q for a, b < q (data x data product).
__device__ __forceinline__ uint64_t mulmod(uint64_t a, uint64_t b, const DevPrime& p) {
  U128 t{a * b, __umul64hi(a, b)};
  return reduce128(t, p);
}

// A signed integer (two's complement, |v| < 2^63) as its residue modulo q.
__device__ __forceinline__ uint64_t signed_mod(uint64_t v, const DevPrime& p) {
  const bool neg = (int64_t)v < 0;
  const uint64_t a = neg ? 0 - v : v;
  const uint64_t r = shoup(a, 1, p.one_s, p.q);
  return neg && r ? p.q - r : r;
}

// OpenFHE SwitchModulus as restated in the reference (src/CKKS/Rescale.cuh:44-64): a
// residue of the old prime `om` re-expressed modulo `nm` with the centred lift.
__device__ __forceinline__ uint64_t switch_modulus(uint64_t a, const DevPrime& om, const DevPrime& nm) {
  const uint64_t half = om.q >> 1;
  if (nm.q > om.q) {
    if (a > half) a += nm.q - om.q;
    return a;
  }
  const uint64_t diff = nm.q - shoup(om.q, 1, nm.one_s, nm.q);  // nm - (om mod nm)
  if (a > half) a += diff;
  if (a >= nm.q) a = shoup(a, 1, nm.one_s, nm.q);
  return a;
}

}  // namespace fides
