// Templates of the NTT pass kernels (see ntt.cuh).  Each ntt_inst_<logN>.cu instantiates
// the passes of one ring dimension so that the variants compile in parallel.
#pragma once
#include <algorithm>

#include "ntt.cuh"

namespace fides {
namespace nttk {

constexpr int COL = 0, ROW = 1;

// Residues per thread, 2^LE (LE = 4: 16, four butterfly stages per register chunk; LE = 3: 8,
// three stages per chunk, one more shared-memory exchange per pass, twice the threads), and
// sub-transforms per CTA (G: 4, 8 or 16) are template parameters of every pass, chosen per
// launch by the context's tables (fides_ctx_autotune).  The butterflies, their pairs and
// twiddles and their order are the same for every LE and G, so the results are identical.

// Asynchronous 16-byte global -> shared copies (cp.async), used to fetch an epilogue operand
// while the butterflies run.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Whether pass PASS of a transform stages its epilogue operand ep0 in shared memory: the
// forward row pass (the last one) with a ModDown / rescale epilogue.  A CTA's rows are one
// contiguous block of ep0, copied with cp.async at the start of the pass.
template <int PASS, bool FWD, int OUT>
struct EpStage {
  static constexpr bool on = PASS == ROW && FWD && (OUT == OUT_MODDOWN || OUT == OUT_MDRS || OUT == OUT_RESCALE);
};

// Twiddle loads carry an L2 evict-last policy: a launch streams hundreds of limbs through L2
// while every limb of one prime re-reads that prime's twiddle table, so the tables should
// outlive the streaming data in L2.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ ShoupConst ld_tw(const ShoupConst* p, uint64_t pol) {
  uint64_t w, ws;
  asm("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(w), "=l"(ws) : "l"(p), "l"(pol));
  return ShoupConst{w, ws};
}
__device__ __forceinline__ double ld_tww(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double2 ld_twf(const double2* p, uint64_t pol) {
  double2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol));
  return v;
}

// Cooley-Tukey butterfly, Harvey lazy form: x, y in [0, 4q) -> [0, 4q).
__device__ __forceinline__ void ct_bf(uint64_t& x, uint64_t& y, ShoupConst w, uint64_t q, uint64_t q2) {
  uint64_t a = csub(x, q2);
  uint64_t t = shoup_lazy(y, w.w, w.ws, q);
  x = a + t;
  y = a - t + q2;
}

// Cooley-Tukey butterfly without any conditional subtraction, for q < 2^58: inputs below
// B give outputs below B + 2q; over at most 17 stages from [0, q) values stay below 35q.
__device__ __forceinline__ void ct_bf_small(uint64_t& x, uint64_t& y, ShoupConst w, uint64_t q, uint64_t q2) {
  uint64_t t = shoup_lazy(y, w.w, w.ws, q);
  uint64_t a = x;
  x = a + t;
  y = a - t + q2;
}

// Gentleman-Sande butterfly with a tracked bound B (a multiple of q, values < B <= 2^63):
// the sum doubles the bound unless `red` (B > 2^62), in which case it is brought back
// below B by one conditional subtraction; the difference path leaves a Shoup product in
// [0, 2q).  With q < 2^62 this degenerates to Harvey's form once B reaches 2q.
__device__ __forceinline__ void gs_bf(uint64_t& x, uint64_t& y, ShoupConst w, uint64_t q, uint64_t B, bool red) {
  uint64_t s = x + y;
  if (red) s = csub(s, B);
  uint64_t d = x - y + B;
  y = shoup_lazy(d, w.w, w.ws, q);
  x = s;
}

// ---- FP64 butterflies for primes q < 2^50.  The residues are integers held in doubles
// (signed, |x| < 2^51), and every operation below is exact:
//   * y w = p + e exactly (p = fl(y w), e = fma(y, w, -p));
//   * k = rint(y (w/q)) from one fma with the rounding constant 1.5 2^52 (|y w/q| < 2^51);
//     |k - y w / q| <= 1/2 + |y| 2^-53 because w/q is correctly rounded;
//   * p - k q is an integer below 2^52 in magnitude, so fma(-k, q, p) is exact, and so is
//     adding e: r = y w - k q with |r| <= q (1/2 + |y| 2^-53).
// A forward butterfly reduces x the same way (x - rint(x / q) q) before x +- r on every other
// stage of a pass (stages 0, 2, 4, ...): after a reducing stage values are within
// (1 + A/8) q, after the next within (13/8 + 9A/64) q, so with A the bound entering a reducing
// stage, A <= 1.9 and every operand of a product stays below 2q <= 2^51 for q < 2^50.  The
// inverse reduces the sum and multiplies the difference on every stage (values within q).
// Between the two passes of a transform the doubles are stored as they are (their bits);
// only the last pass writes canonical residues.  On B200 the FP64 pipe runs this
// product at ~1.7x the rate of the 64-bit integer Shoup product, which is the NTT's bound.
constexpr double F64_RND = 6755399441055744.0;  // 1.5 * 2^52
constexpr double F64_TWO52 = 4503599627370496.0;
__device__ __forceinline__ double f_mulmod(double y, double w, double wq, double q) {
  const double p = __dmul_rn(y, w);
  const double e = __fma_rn(y, w, -p);
  const double k = __dadd_rn(__fma_rn(y, wq, F64_RND), -F64_RND);
  return __dadd_rn(__fma_rn(-k, q, p), e);
}
__device__ __forceinline__ double f_reduce(double x, double q, double qinv) {
  const double k = __dadd_rn(__fma_rn(x, qinv, F64_RND), -F64_RND);
  return __fma_rn(-k, q, x);
}
// u64 < 2^52 -> double (exact), and a value |v| < 2q -> its canonical residue in [0, q):
// v + 2q + 2^52 lies in [2^52, 2^53), where the double's low 52 bits are the integer v + 2q.
__device__ __forceinline__ double f_from_u64(uint64_t v) {
  return __dadd_rn(__longlong_as_double((long long)(0x4330000000000000ull | v)), -F64_TWO52);
}
__device__ __forceinline__ uint64_t f_to_canon(double v, double q2_two52, uint64_t qi) {
  uint64_t u = (uint64_t)__double_as_longlong(__dadd_rn(v, q2_two52)) & ((1ull << 52) - 1);  // v + 2q
  u = u >= 2 * qi ? u - 2 * qi : u;
  return u >= qi ? u - qi : u;
}

struct PassArgs {
  const DevPrime* primes;
  const ShoupConst* tw;        // forward or inverse twiddles, [prime][N]
  const double2* twf;          // the same twiddles as (w, w / q) doubles (q < 2^50)
  const double* tww;           // w / q alone: the row passes (one twiddle per row and stage each)
                               // read half the bytes and derive w
  const F64Prime* f64;         // [prime]
  const ShoupConst* inv_last;  // [prime]: psi_rev^-1[1] * N^-1
  const ShoupConst* pinv;      // [Q prime]: P^-1 mod q (OUT_MODDOWN)
  const RescaleConst* rescale; // [level][Q prime] (OUT_RESCALE, OUT_MDRS)
  const ShoupConst* pmod;      // [Q prime]: P mod q (IN_CONV_SW, IN_ADD_PMUL)
  const ShoupConst* pqinv;     // [level][Q prime]: (P q_(level-1))^-1 mod q (OUT_MDRS)
  int logN;
  int log1;  // size of the column sub-transform
  int n_q;
};

// Element index u of register r for thread t, when the register index spans bits
// [lo, lo + LE) of u.
template <int LO, int LE>
__device__ __forceinline__ int u_of(int t, int r) {
  // disjoint bit fields: '+' lets the compiler fold the register-index part into offsets
  return ((t >> LO) << (LO + LE)) + (r << LO) + (t & ((1 << LO) - 1));
}

template <int LE>
__device__ __forceinline__ int padu(int u) {
  return u + (u >> LE);
}

// Butterflies of pair bits [BLO, BHI] (in u) for a thread whose registers span bits
// [LO, LO + LE).  FWD walks bits high -> low, inverse low -> high.
template <int LE, int LOGP, int LO, int BHI, int BLO, bool FWD, int PASS, bool SMALL>
__device__ __forceinline__ void run_chunk(uint64_t (&x)[1 << LE], int t, int sub, int sbase, const ShoupConst* tw,
                                          const DevPrime& pr, ShoupConst last, uint64_t& B, uint64_t pol) {
  constexpr int E = 1 << LE;
  const int th = t >> LO;
#pragma unroll
  for (int k = 0; k <= BHI - BLO; ++k) {
    const int b = FWD ? (BHI - k) : (BLO + k);
    const int rb = b - LO;
    const int sig = LOGP - 1 - b;  // stage within this pass
    const int s = sbase + sig;     // global stage
    const uint32_t base = (1u << s) + ((uint32_t)sub << sig) + ((uint32_t)th << (LO + LE - b - 1));
    const bool red = !FWD && B > (1ull << 62);
#pragma unroll
    for (int hi = 0; hi < (E >> (rb + 1)); ++hi) {
      if (!FWD && PASS == COL && b == LOGP - 1) {
        // last inverse stage (global stage 0): fold N^-1 into both outputs
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          uint64_t a = x[r0], c = x[r1];
          x[r0] = shoup(a + c, pr.ninv, pr.ninv_s, pr.q);
          x[r1] = shoup(a - c + B, last.w, last.ws, pr.q);
        }
      } else {
        const ShoupConst w = ld_tw(tw + base + hi, pol);
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          if (FWD && SMALL)
            ct_bf_small(x[r0], x[r1], w, pr.q, pr.q2);
          else if (FWD)
            ct_bf(x[r0], x[r1], w, pr.q, pr.q2);
          else
            gs_bf(x[r0], x[r1], w, pr.q, B, red);
        }
      }
    }
    if (!FWD && !red) B <<= 1;
  }
}

// run_chunk on FP64 residues (q < 2^50): the same stages, pairs and twiddles.
template <int LE, int LOGP, int LO, int BHI, int BLO, bool FWD, int PASS>
__device__ __forceinline__ void run_chunk_f64(double (&x)[1 << LE], int t, int sub, int sbase, const double2* tw,
                                              const double* tww, const F64Prime& fp, uint64_t pol) {
  constexpr int E = 1 << LE;
  const int th = t >> LO;
#pragma unroll
  for (int k = 0; k <= BHI - BLO; ++k) {
    const int b = FWD ? (BHI - k) : (BLO + k);
    const int rb = b - LO;
    const int sig = LOGP - 1 - b;
    const int s = sbase + sig;
    const uint32_t base = (1u << s) + ((uint32_t)sub << sig) + ((uint32_t)th << (LO + LE - b - 1));
#pragma unroll
    for (int hi = 0; hi < (E >> (rb + 1)); ++hi) {
      if (!FWD && PASS == COL && b == LOGP - 1) {
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          const double a = x[r0], c = x[r1];
          x[r0] = f_mulmod(__dadd_rn(a, c), fp.ninv, fp.ninv_q, fp.q);
          x[r1] = f_mulmod(__dsub_rn(a, c), fp.last, fp.last_q, fp.q);
        }
      } else {
        double2 w;
        if constexpr (PASS == ROW) {
          // w from the stored, correctly rounded w / q: (w / q) q lies within q 2^-54 < 1/2
          // of the integer w, so one fma with the rounding constant recovers w exactly
          w.y = ld_tww(tww + base + hi, pol);
          w.x = __dadd_rn(__fma_rn(w.y, fp.q, F64_RND), -F64_RND);
        } else {
          w = ld_twf(tw + base + hi, pol);
        }
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          if (FWD) {
            const double a = (sig & 1) ? x[r0] : f_reduce(x[r0], fp.q, fp.qinv);
            const double r = f_mulmod(x[r1], w.x, w.y, fp.q);
            x[r0] = __dadd_rn(a, r);
            x[r1] = __dsub_rn(a, r);
          } else {
            const double a = x[r0], c = x[r1];
            x[r0] = f_reduce(__dadd_rn(a, c), fp.q, fp.qinv);
            x[r1] = f_mulmod(__dsub_rn(a, c), w.x, w.y, fp.q);
          }
        }
      }
    }
  }
}

// Bound of the inverse transform's values after `stages` stages from reduced input.
__device__ __forceinline__ uint64_t inv_bound(uint64_t q, int stages) {
  uint64_t B = q;
  for (int i = 0; i < stages; ++i)
    if (B <= (1ull << 62)) B <<= 1;
  return B;
}



// Register span of chunk c.
template <int LE, int LOGP, bool FWD, int C>
struct Chunk {
  // forward: bits from the top; inverse: bits from the bottom
  static constexpr int BHI = FWD ? (LOGP - 1 - C * LE) : (C * LE + LE - 1 < LOGP - 1 ? C * LE + LE - 1 : LOGP - 1);
  static constexpr int BLO = FWD ? (LOGP - (C + 1) * LE > 0 ? LOGP - (C + 1) * LE : 0) : C * LE;
  static constexpr int LO = FWD ? BLO : (BLO + LE <= LOGP ? BLO : LOGP - LE);
};

// The register chunks of one pass, separated by shared-memory exchanges.
template <int LE, int LOGP, int PASS, bool FWD, bool SMALL, typename SIDX>
__device__ __forceinline__ void chunks(uint64_t (&x)[1 << LE], uint64_t* sm, SIDX sidx, int g, int t, int subtw,
                                       int sbase, const ShoupConst* tw, const DevPrime& pr, ShoupConst last,
                                       uint64_t& B, bool direct_load, uint64_t pol) {
  constexpr int E = 1 << LE;
  constexpr int NCH = (LOGP + LE - 1) / LE;
  using C0 = Chunk<LE, LOGP, FWD, 0>;
  run_chunk<LE, LOGP, C0::LO, C0::BHI, C0::BLO, FWD, PASS, SMALL>(x, t, subtw, sbase, tw, pr, last, B, pol);
  if constexpr (NCH > 1) {
    using C1 = Chunk<LE, LOGP, FWD, 1>;
    if (!direct_load) __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<C0::LO, LE>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<C1::LO, LE>(t, r))];
    run_chunk<LE, LOGP, C1::LO, C1::BHI, C1::BLO, FWD, PASS, SMALL>(x, t, subtw, sbase, tw, pr, last, B, pol);
  }
  if constexpr (NCH > 2) {
    using C1 = Chunk<LE, LOGP, FWD, 1>;
    using C2 = Chunk<LE, LOGP, FWD, 2>;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<C1::LO, LE>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<C2::LO, LE>(t, r))];
    run_chunk<LE, LOGP, C2::LO, C2::BHI, C2::BLO, FWD, PASS, SMALL>(x, t, subtw, sbase, tw, pr, last, B, pol);
  }
  static_assert(NCH <= 3, "sub-transform too large");
}

// chunks() on FP64 residues; the shared-memory exchanges move the doubles' bits.
template <int LE, int LOGP, int PASS, bool FWD, typename SIDX>
__device__ __forceinline__ void chunks_f64(double (&x)[1 << LE], uint64_t* smu, SIDX sidx, int g, int t, int subtw,
                                           int sbase, const double2* tw, const double* tww, const F64Prime& fp,
                                           bool direct_load, uint64_t pol) {
  constexpr int E = 1 << LE;
  constexpr int NCH = (LOGP + LE - 1) / LE;
  double* sm = reinterpret_cast<double*>(smu);
  using C0 = Chunk<LE, LOGP, FWD, 0>;
  run_chunk_f64<LE, LOGP, C0::LO, C0::BHI, C0::BLO, FWD, PASS>(x, t, subtw, sbase, tw, tww, fp, pol);
  if constexpr (NCH > 1) {
    using C1 = Chunk<LE, LOGP, FWD, 1>;
    if (!direct_load) __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<C0::LO, LE>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<C1::LO, LE>(t, r))];
    run_chunk_f64<LE, LOGP, C1::LO, C1::BHI, C1::BLO, FWD, PASS>(x, t, subtw, sbase, tw, tww, fp, pol);
  }
  if constexpr (NCH > 2) {
    using C1 = Chunk<LE, LOGP, FWD, 1>;
    using C2 = Chunk<LE, LOGP, FWD, 2>;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<C1::LO, LE>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<C2::LO, LE>(t, r))];
    run_chunk_f64<LE, LOGP, C2::LO, C2::BHI, C2::BLO, FWD, PASS>(x, t, subtw, sbase, tw, tww, fp, pol);
  }
}

template <int LOGN, int PASS>
struct PassShape {
  static constexpr int LOG1 = (LOGN + 1) / 2, LOG2 = LOGN / 2;
  static constexpr int LOGP = PASS == COL ? LOG1 : LOG2;
};

// One pass of a transform of 2^LOGN points.  Every index is a compile-time function of
// LOGN, so global and shared addresses are a per-thread base plus immediate offsets.
// Threads of a pass CTA, and CTAs per SM the register budget is sized for: with 16 residues
// per thread 768 threads = 24 warps per SM, i.e. 80 registers (FIDES_NTT_THREADS_PER_SM
// overrides it); with 8, 1024 threads = 32 warps, 64 registers (no spills in the plain passes).
#ifndef FIDES_NTT_THREADS_PER_SM
#define FIDES_NTT_THREADS_PER_SM 768
#endif
template <int LOGN, int PASS, int G, int LE>
struct PassThreads {
  static constexpr int TPS = LE == 3 ? 1024 : FIDES_NTT_THREADS_PER_SM;
  static constexpr int NT = (1 << (PassShape<LOGN, PASS>::LOGP - LE)) * G;
  static constexpr int MINB = NT >= TPS ? 1 : (TPS / NT > 32 ? 32 : TPS / NT);
};

// Ring dimensions whose passes are also built with 8 residues per thread (measured faster for
// small launches at N >= 2^15; smaller rings keep 16 only).
template <int LOGN>
struct HasLe3 {
  static constexpr bool value = LOGN >= 15;
};

template <int LOGN, int PASS, bool FWD, int IN, int OUT, int G, int LE>
__global__ void __launch_bounds__(PassThreads<LOGN, PASS, G, LE>::NT, PassThreads<LOGN, PASS, G, LE>::MINB)
    ntt_pass(const PassArgs a, const __grid_constant__ NttLimbList L) {
  constexpr int LOGP = PassShape<LOGN, PASS>::LOGP;
  constexpr int P = 1 << LOGP, E = 1 << LE, T = P / E, NT = T * G;
  constexpr int NCH = (LOGP + LE - 1) / LE;
  constexpr int PADP = P + P / E;
  extern __shared__ uint64_t sm[];

  const LimbRef lr = L.limbs[blockIdx.y];
  const DevPrime pr = a.primes[lr.prime];
  constexpr int N = 1 << LOGN;
  const ShoupConst* tw = a.tw + (size_t)lr.prime * N;
  const ShoupConst last = FWD ? ShoupConst{0, 0} : a.inv_last[lr.prime];
  uint64_t* data = lr.ptr;
  const int tid = threadIdx.x;
  int g, t;
  if (PASS == COL) {
    g = tid % G;
    t = tid / G;
  } else {
    t = tid % T;
    g = tid / T;
  }
  constexpr int S = N >> LOGP;  // stride of a column (COL) / number of rows (ROW)
  const int sub0 = blockIdx.x * G;
  const int sub = sub0 + g;
  constexpr int sbase = PASS == COL ? 0 : PassShape<LOGN, COL>::LOGP;
  const int subtw = PASS == COL ? 0 : sub;

  auto gidx = [&](int s_, int u) -> int { return PASS == COL ? s_ + u * S : s_ * P + u; };
  auto sidx = [&](int gg, int u) -> int { return PASS == COL ? u * G + gg : gg * PADP + padu<LE>(u); };

  uint64_t x[E];

  // ---- input of this pass: the first pass applies the prologue
  constexpr bool first_pass = FWD ? (PASS == COL) : (PASS == ROW);
  const uint64_t* in = (first_pass && lr.src) ? lr.src : data;
  DevPrime opr;
  if (IN == IN_SWITCH || IN == IN_CONV_SW) opr = a.primes[lr.aux - 1];
  ShoupConst pm{0, 0};
  if (IN == IN_CONV_SW || IN == IN_ADD_PMUL) pm = a.pmod[lr.prime];
  auto load = [&](size_t i) -> uint64_t {
    if (first_pass && IN == IN_SWITCH) return switch_modulus(lr.pro[i], opr, pr);
    if (first_pass && IN == IN_SIGNED) return signed_mod(lr.pro[i], pr);
    if (first_pass && IN == IN_MUL) return mulmod(in[i], lr.pro[i], pr);
    if (first_pass && IN == IN_CONV_SW) return in[i];  // + P SwitchModulus(top) below
    if (first_pass && IN == IN_ADD_PMUL) return addmod(in[i], shoup(lr.pro[i], pm.w, pm.ws, pr.q), pr.q);
    return in[i];
  };

  // ---- load chunk 0 (direct when lanes map to consecutive addresses, else staged)
  constexpr int LO0 = Chunk<LE, LOGP, FWD, 0>::LO;
  constexpr bool direct_load = (PASS == COL) || (LO0 == LOGP - LE);
  // conv + P SwitchModulus(top) (a column pass): the tile of the top limb is copied into the
  // exchange buffer by cp.async while the conv loads are in flight, so the prologue waits for
  // memory once (loading both operands per element serialised the loads: long-scoreboard
  // stalls 10x a plain pass's)
  constexpr bool STAGE_PRO = first_pass && IN == IN_CONV_SW;
  static_assert(!STAGE_PRO || PASS == COL, "the conv-switch prologue is a column-pass prologue");
  if constexpr (STAGE_PRO) {
#pragma unroll
    for (int k = 0; k < G * P / 2 / NT; ++k) {
      const int c = k * NT + tid, u = c / (G / 2), h = c % (G / 2);
      cp_async16(sm + u * G + 2 * h, lr.pro + (size_t)u * S + sub0 + 2 * h);
    }
    cp_async_commit();
  }
  if (direct_load) {
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = load(gidx(sub, u_of<LO0, LE>(t, r)));
    if constexpr (STAGE_PRO) {
      cp_async_wait_all();
      __syncthreads();
#pragma unroll
      for (int r = 0; r < E; ++r)
        x[r] = addmod(x[r], shoup(switch_modulus(sm[u_of<LO0, LE>(t, r) * G + g], opr, pr), pm.w, pm.ws, pr.q), pr.q);
    }
  } else {
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = k * NT + tid;
      int gg = e / P, u = e % P;
      sm[sidx(gg, u)] = load(gidx(sub0 + gg, u));
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<LO0, LE>(t, r))];
  }

  // ---- epilogue operand: start fetching it into shared memory (after the data region)
  constexpr bool EPS = EpStage<PASS, FWD, OUT>::on;
  uint64_t* sep = sm + G * PADP;
  if constexpr (EPS) {
    const uint64_t* e0 = lr.ep0 + (size_t)sub0 * P;
#pragma unroll
    for (int k = 0; k < G * P / 2 / NT; ++k) cp_async16(sep + 2 * (k * NT + tid), e0 + 2 * (k * NT + tid));
    cp_async_commit();
  }

  // ---- chunks
  const uint64_t pol = l2_evict_last_policy();
  const bool f64 = pr.q < (1ull << 50);  // uniform per CTA: one limb per CTA
  if (f64) {
    // FP64 butterflies; every pass of such a limb stores canonical residues
    const F64Prime fp = a.f64[lr.prime];
    double xf[E];
    if (first_pass) {
      // canonical inputs in [0, q): the first stage reduces (forward: the x operand, as on every
      // even stage; inverse: every sum) and takes operands below q into its products
#pragma unroll
      for (int r = 0; r < E; ++r) xf[r] = f_from_u64(x[r]);
    } else {
#pragma unroll
      for (int r = 0; r < E; ++r) xf[r] = __longlong_as_double((long long)x[r]);  // the first pass's doubles
    }
    chunks_f64<LE, LOGP, PASS, FWD>(xf, sm, sidx, g, t, subtw, sbase, a.twf + (size_t)lr.prime * N,
                                a.tww + (size_t)lr.prime * N, fp, direct_load && !STAGE_PRO, pol);
    if (first_pass) {
#pragma unroll
      for (int r = 0; r < E; ++r) x[r] = (uint64_t)__double_as_longlong(xf[r]);
    } else {
      const double q2t = __dadd_rn(2.0 * fp.q, F64_TWO52);
#pragma unroll
      for (int r = 0; r < E; ++r) x[r] = f_to_canon(xf[r], q2t, pr.q);
    }
  } else {
  uint64_t B = pr.q;  // inverse: bound of the values (a multiple of q)
  if (!FWD && PASS == COL) B = inv_bound(pr.q, PassShape<LOGN, ROW>::LOGP);
  if (FWD && pr.q < (1ull << 58))
    chunks<LE, LOGP, PASS, FWD, true>(x, sm, sidx, g, t, subtw, sbase, tw, pr, last, B, direct_load && !STAGE_PRO, pol);
  else
    chunks<LE, LOGP, PASS, FWD, false>(x, sm, sidx, g, t, subtw, sbase, tw, pr, last, B, direct_load && !STAGE_PRO, pol);

  // ---- final reduction of the completed transform
  if (FWD && PASS == ROW) {
    if (pr.q < (1ull << 58)) {
#pragma unroll
      for (int r = 0; r < E; ++r) x[r] = shoup(x[r], 1, pr.one_s, pr.q);  // x < 35q
    } else {
#pragma unroll
      for (int r = 0; r < E; ++r) x[r] = csub(csub(x[r], pr.q2), pr.q);   // x < 4q
    }
  }
  }

  // ---- store (the last pass applies the epilogue)
  ShoupConst pinv{0, 0};
  RescaleConst rsc{0, 0, 0, 0};
  if (OUT == OUT_MODDOWN || OUT == OUT_SUB_PINV) pinv = a.pinv[lr.prime];
  if (OUT == OUT_MDRS) pinv = a.pqinv[(size_t)lr.aux * a.n_q + lr.prime];
  if (OUT == OUT_RESCALE || OUT == OUT_MDRS) rsc = a.rescale[(size_t)lr.aux * a.n_q + lr.prime];
  auto ep0 = [&](size_t i) -> uint64_t {
    if constexpr (EPS) return sep[i - (size_t)sub0 * P];
    return lr.ep0[i];
  };
  auto store = [&](size_t i, uint64_t v) {
    if (OUT == OUT_MODDOWN || OUT == OUT_MDRS) {
      v = shoup(submod(ep0(i), v, pr.q), pinv.w, pinv.ws, pr.q);
      if (lr.ep1) {
        const uint64_t e = lr.ep1[i];
        v = addmod(v, OUT == OUT_MDRS ? shoup(e, rsc.qinv, rsc.qinv_s, pr.q) : e, pr.q);
      }
    } else if (OUT == OUT_RESCALE) {
      v = addmod(shoup(ep0(i), rsc.qinv, rsc.qinv_s, pr.q), shoup(v, rsc.m, rsc.m_s, pr.q), pr.q);
    } else if (OUT == OUT_SUB_PINV) {
      v = shoup(submod(v, lr.ep0[i], pr.q), pinv.w, pinv.ws, pr.q);
    }
    data[i] = v;
  };
  constexpr int LOL = Chunk<LE, LOGP, FWD, NCH - 1>::LO;
  constexpr bool direct_store = (PASS == COL) || (LOL == LOGP - LE);
  if constexpr (EPS) {
    cp_async_wait_all();
    if (direct_store) __syncthreads();  // the staged store below synchronises anyway
  }
  if (direct_store) {
#pragma unroll
    for (int r = 0; r < E; ++r) store(gidx(sub, u_of<LOL, LE>(t, r)), x[r]);
  } else {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<LOL, LE>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = k * NT + tid;
      int gg = e / P, u = e % P;
      store(gidx(sub0 + gg, u), sm[sidx(gg, u)]);
    }
  }
}


template <int LOGN, int PASS, bool FWD, int IN, int OUT, int G, int LE>
void launch_pass_g(Context* c, const PassArgs& a, const NttLimbList& L, cudaStream_t s) {
  constexpr int LOGP = PassShape<LOGN, PASS>::LOGP;
  constexpr int P = 1 << LOGP, T = P / (1 << LE);
  constexpr int smem = (PASS == COL ? P * G : G * (P + P / (1 << LE))) * (int)sizeof(uint64_t) +
                       (EpStage<PASS, FWD, OUT>::on ? G * P * (int)sizeof(uint64_t) : 0);
  static bool attr_set = false;  // per instantiation; set before first launch
  if (!attr_set) {
    FIDES_CUDA(cudaFuncSetAttribute(ntt_pass<LOGN, PASS, FWD, IN, OUT, G, LE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set = true;
  }
  dim3 grid(((1 << LOGN) >> LOGP) / G, L.n);
  // algorithmic bytes: half of a transform's read + write of each limb (two passes)
  LaunchScope ls(c, s, KK_NTT, 8.0 * (1 << LOGN) * L.n);
  ntt_pass<LOGN, PASS, FWD, IN, OUT, G, LE><<<grid, T * G, smem, s>>>(a, L);
  FIDES_CUDA(cudaGetLastError());
}

// The pass with the sub-transforms-per-CTA and residues per thread the context's tables pick
// for this launch.
template <int LOGN, int PASS, bool FWD, int IN, int OUT, int LE>
void launch_pass_le(Context* c, const PassArgs& a, const NttLimbList& L, cudaStream_t s) {
  switch (c->ntt_shape(!FWD, PASS, L.n)) {
    case 4: launch_pass_g<LOGN, PASS, FWD, IN, OUT, 4, LE>(c, a, L, s); break;
    case 8: launch_pass_g<LOGN, PASS, FWD, IN, OUT, 8, LE>(c, a, L, s); break;
    default: launch_pass_g<LOGN, PASS, FWD, IN, OUT, 16, LE>(c, a, L, s);
  }
}
template <int LOGN, int PASS, bool FWD, int IN, int OUT>
void launch_pass(Context* c, const PassArgs& a, const NttLimbList& L, cudaStream_t s) {
  if constexpr (HasLe3<LOGN>::value) {
    if (c->ntt_residues(!FWD, PASS, L.n) == 8) {
      launch_pass_le<LOGN, PASS, FWD, IN, OUT, 3>(c, a, L, s);
      return;
    }
  }
  launch_pass_le<LOGN, PASS, FWD, IN, OUT, 4>(c, a, L, s);
}

// The pass sequence of one transform for a given ring dimension.
template <int LOGN>
void run_transform(Context* c, const PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, NttOut out,
                   cudaStream_t s) {
  if (!inverse) {
    if (in == IN_SWITCH)
      launch_pass<LOGN, COL, true, IN_SWITCH, OUT_PLAIN>(c, a, L, s);
    else if (in == IN_SIGNED)
      launch_pass<LOGN, COL, true, IN_SIGNED, OUT_PLAIN>(c, a, L, s);
    else if (in == IN_CONV_SW)
      launch_pass<LOGN, COL, true, IN_CONV_SW, OUT_PLAIN>(c, a, L, s);
    else
      launch_pass<LOGN, COL, true, IN_PLAIN, OUT_PLAIN>(c, a, L, s);
    if (out == OUT_MODDOWN)
      launch_pass<LOGN, ROW, true, IN_PLAIN, OUT_MODDOWN>(c, a, L, s);
    else if (out == OUT_RESCALE)
      launch_pass<LOGN, ROW, true, IN_PLAIN, OUT_RESCALE>(c, a, L, s);
    else if (out == OUT_MDRS)
      launch_pass<LOGN, ROW, true, IN_PLAIN, OUT_MDRS>(c, a, L, s);
    else
      launch_pass<LOGN, ROW, true, IN_PLAIN, OUT_PLAIN>(c, a, L, s);
  } else {
    if (in == IN_MUL)
      launch_pass<LOGN, ROW, false, IN_MUL, OUT_PLAIN>(c, a, L, s);
    else if (in == IN_ADD_PMUL)
      launch_pass<LOGN, ROW, false, IN_ADD_PMUL, OUT_PLAIN>(c, a, L, s);
    else
      launch_pass<LOGN, ROW, false, IN_PLAIN, OUT_PLAIN>(c, a, L, s);
    if (out == OUT_SUB_PINV)
      launch_pass<LOGN, COL, false, IN_PLAIN, OUT_SUB_PINV>(c, a, L, s);
    else
      launch_pass<LOGN, COL, false, IN_PLAIN, OUT_PLAIN>(c, a, L, s);
  }
}

}  // namespace nttk

// Defined in ntt_inst_<logN>.cu.
#define FIDES_NTT_DECL(LN)                                                                                  \
  void ntt_transform_##LN(Context* c, const nttk::PassArgs& a, const NttLimbList& L, bool inverse, NttIn in, \
                          NttOut out, cudaStream_t s);
FIDES_NTT_DECL(10)
FIDES_NTT_DECL(11)
FIDES_NTT_DECL(12)
FIDES_NTT_DECL(13)
FIDES_NTT_DECL(14)
FIDES_NTT_DECL(15)
FIDES_NTT_DECL(16)
FIDES_NTT_DECL(17)
#undef FIDES_NTT_DECL

}  // namespace fides
