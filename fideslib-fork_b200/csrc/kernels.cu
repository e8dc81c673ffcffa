// Elementwise RNS kernels, basis conversion and KSK inner product.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "kernels.cuh"
#include "conv_tc.hpp"

namespace fides {

namespace {

// automorph_slot (reference src/Rotation.cuh:14-26): j -> brev(((2 brev(j) + 1) k mod 2N) >> 1)
__device__ __forceinline__ uint32_t auto_slot(int logN, uint32_t k, uint32_t j) {
  uint32_t jr = __brev(j) >> (32 - logN);
  uint32_t r = ((((jr << 1) + 1) * k) & ((2u << logN) - 1)) >> 1;
  return __brev(r) >> (32 - logN);
}

constexpr int MAX_SRC = 64;   // limbs on the source side of one conversion
constexpr int MAX_DST = 128;  // limbs on the destination side

// Basis conversion.  NS (source limbs) is a template parameter so that the pre-scaled
// sources stay in registers; NS = 0 is the generic width.  Each thread converts two
// adjacent coefficients (16-byte accesses); destination primes, output positions and the
// conversion matrix are staged in shared memory (broadcast reads).
template <int NS>
__global__ void __launch_bounds__(EW_THREADS) conv_kernel(const __grid_constant__ ConvJobList L, const DevPrime* primes,
                                                          int logN) {
  const ConvJob& J = L.j[blockIdx.y];
  const ConvTable& T = J.t;
  extern __shared__ uint64_t sm[];
  const int ns = NS ? NS : T.n_src, nd = T.n_dst, lift = T.lift;
  ShoupConst* pre = reinterpret_cast<ShoupConst*>(sm);       // [ns]
  DevPrime* dp = reinterpret_cast<DevPrime*>(sm + 2 * ns);   // [nd]
  uint64_t* mat = sm + 2 * ns + 8 * nd;                      // [ns + lift][nd]
  int* dpos = reinterpret_cast<int*>(mat + (ns + lift) * nd); // [nd]
  for (int i = threadIdx.x; i < (ns + lift) * nd; i += blockDim.x) mat[i] = T.mat[i];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) pre[i] = T.pre[i];
  for (int j = threadIdx.x; j < nd; j += blockDim.x) {
    dp[j] = primes[T.dst_prime[j]];
    dpos[j] = T.dst_pos[j];
  }
  __syncthreads();
  const int N = 1 << logN;
  const int n = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  constexpr int R = NS ? NS : MAX_SRC;
  uint64_t y0[R], y1[R];
  uint64_t lift0 = 0, lift1 = 0;  // reduced-noise lift: sources above q_i / 2
#pragma unroll
  for (int i = 0; i < R; ++i) {
    if (NS == 0 && i >= ns) break;
    const uint64_t q = primes[T.src_prime[i]].q;
    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(J.src + (size_t)T.src_pos[i] * N + n);
    y0[i] = shoup(v.x, pre[i].w, pre[i].ws, q);
    y1[i] = shoup(v.y, pre[i].w, pre[i].ws, q);
    lift0 += y0[i] > (q >> 1);
    lift1 += y1[i] > (q >> 1);
  }
  uint64_t* dst = J.dst + n;
  for (int j = 0; j < nd; ++j) {
    const DevPrime p = dp[j];
    U128 a0{0, 0}, a1{0, 0};
#pragma unroll
    for (int i = 0; i < R; ++i) {
      if (NS == 0 && i >= ns) break;
      if (i && (i & 7) == 0) {  // keep the sums below 2^128
        a0 = U128{reduce128(a0, p), 0};
        a1 = U128{reduce128(a1, p), 0};
      }
      const uint64_t m = mat[i * nd + j];
      mac128(a0, y0[i], m);
      mac128(a1, y1[i], m);
    }
    if (lift) {  // count (<= 64) times [-Q_src]_{p_j}: below 2^69, no reduction needed first
      const uint64_t m = mat[ns * nd + j];
      mac128(a0, lift0, m);
      mac128(a1, lift1, m);
    }
    *reinterpret_cast<ulonglong2*>(dst + (size_t)dpos[j] * N) = make_ulonglong2(reduce128(a0, p), reduce128(a1, p));
  }
}

// CPT adjacent coefficients per thread (the launches use CPT = 2: 16-byte loads of every
// stream; one coefficient per thread was measured 13 % slower).  MAXB is the largest digit
// count of the launch's jobs (0 = any): with it known at compile time every load of a job --
// all digits, the own-digit and tensor operands -- is issued before its first product.  JG:
// jobs per group (one CTA runs a group; its jobs share the key tile, read once); the grouped
// form keeps three CTAs per SM at the cost of a few spilled registers, which measured faster
// (KSK -9 % with groups of 4) than the unbounded register count (two CTAs per SM).
template <int CPT>
struct KVec {
  uint64_t c[CPT];
};
template <int CPT>
__device__ __forceinline__ KVec<CPT> kld(const uint64_t* q) {
  KVec<CPT> v;
  if constexpr (CPT == 2) {
    const ulonglong2 t = *reinterpret_cast<const ulonglong2*>(q);
    v.c[0] = t.x;
    v.c[1] = t.y;
  } else {
    v.c[0] = *q;
  }
  return v;
}

// FP64 products for limbs of primes q < 2^50 (the NTT's FP64 residues, here on canonical
// inputs a, b < q): p = fl(ab), e = fma(a, b, -p) = ab - p exactly; k = rint(p (1/q)) from one
// fma with the rounding constant 1.5 2^52, within 1 of ab / q (p (1/q) is within
// (ab / q) 2^-52 <= 1/2 of ab / q); p - k q is below 2^53 in magnitude, so fma(-k, q, p) is
// exact, and so is adding e: r = ab - k q with |r| <= q.  The a side of the inner product (up to
// four digits and two tensor terms: |sum| <= 6q < 2^53, summed exactly and reduced once) and
// the own digit's a1 b1 run on the FP64 pipe; the b side keeps the 128-bit integer products on
// the FMA-heavy pipe.  (Moving the tensor terms' P products and the b side's P a0 b0 to FP64
// as well was 12 % slower.)
__device__ __forceinline__ double ksk_f64(uint64_t v) {
  return __dadd_rn(__longlong_as_double((long long)(0x4330000000000000ull | v)), -4503599627370496.0);
}
__device__ __forceinline__ double ksk_mul_f64(uint64_t a, uint64_t b, double q, double qinv) {
  const double x = ksk_f64(a), y = ksk_f64(b);
  const double p = __dmul_rn(x, y);
  const double e = __fma_rn(x, y, -p);
  const double k = __dadd_rn(__fma_rn(p, qinv, 6755399441055744.0), -6755399441055744.0);
  return __dadd_rn(__fma_rn(-k, q, p), e);
}
// canonical residue of an exact sum |s| < 2^53
__device__ __forceinline__ uint64_t ksk_canon_f64(double s, double q, double qinv) {
  const double k = __dadd_rn(__fma_rn(s, qinv, 6755399441055744.0), -6755399441055744.0);
  double r = __fma_rn(-k, q, s);  // |r| <= q / 2 + 1
  if (r < 0) r = __dadd_rn(r, q);
  return (uint64_t)__double_as_longlong(__dadd_rn(r, 4503599627370496.0)) & ((1ull << 52) - 1);
}

// Three CTAs (24 warps) per SM: 80 registers.  The grouped forms spill a few registers there
// (measured faster than two CTAs per SM); the single-job forms with up to three digits fit
// without spills (they took 96-120 registers, two CTAs per SM, when unbounded).
template <int MAXB, int JG>
struct KskMinBlocks {
  static constexpr int value = (JG > 1 || (MAXB >= 1 && MAXB <= 3)) ? 3 : 1;
};

template <int MAXB, int JG, int CPT, bool SHARE_DIGITS = false>
__global__ void __launch_bounds__(EW_THREADS, KskMinBlocks<MAXB, JG>::value) ksk_kernel(const __grid_constant__ KskJobList L, const DevPrime* primes,
                                                            const ShoupConst* pmod, const F64Prime* f64, int logN,
                                                            int n_q, int K, int dnum, int alpha) {
  using V = KVec<CPT>;
  const int g0 = L.gstart[blockIdx.z], gn = L.gcount[blockIdx.z];
  const KskJob& J0 = L.j[g0];  // the group's jobs share key, level and extras
  const int l = J0.l, ext = l + K;
  const int i = blockIdx.y;
  if (i >= ext) return;
  const int N = 1 << logN;
  const int n = CPT * (blockIdx.x * blockDim.x + threadIdx.x);
  const int pid = i < l ? i : n_q + (i - l);
  const DevPrime p = primes[pid];
  const int beta = (l + alpha - 1) / alpha;
  const int own = i < l ? i / alpha : -1;
  const size_t kstride = (size_t)(n_q + K) * N;
  const size_t off = (size_t)i * N + n, koff = (size_t)pid * N + n;
  const bool tensor = J0.a0 && i < l;
  // FP64 a side: limbs of primes below 2^50, at most 4 digits (so at most 6 summed terms)
  const bool fa_on = MAXB > 0 && p.q < (1ull << 50);
  double fq = 0, fqinv = 0;
  if (fa_on) {
    fq = f64[pid].q;
    fqinv = f64[pid].qinv;
  }
  // one job: sum_d D_d key_d (+ extras), reduced and stored; ka / kb: the group's key tile, or
  // vd: the group's digit tile (MAXB > 0; the other one is loaded here).  FA: the a side's
  // products and the own digit's a1 b1 in FP64.
  auto run = [&](const KskJob& J, const V* ka_g, const V* kb_g, const V* vd, auto fa_) {
    constexpr bool FA = decltype(fa_)::value;
    U128 sa[CPT], sb[CPT];
    double fs[CPT];  // FA: the a side
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      sa[c] = sb[c] = U128{0, 0};
      fs[c] = 0;
    }
    V x1{}, y1{};  // a1, b1 of this limb (own digit)
    auto digit = [&](int d, V v, const V& a_, const V& b_) {
      if (d == own && J.x2) {  // the own digit is x * x2 (tensor term a1 b1)
        x1 = v;
#pragma unroll
        for (int c = 0; c < CPT; ++c)
          v.c[c] = FA ? ksk_canon_f64(ksk_mul_f64(v.c[c], y1.c[c], fq, fqinv), fq, fqinv) : mulmod(v.c[c], y1.c[c], p);
      }
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        if constexpr (FA)
          fs[c] = __dadd_rn(fs[c], ksk_mul_f64(v.c[c], a_.c[c], fq, fqinv));
        else
          mac128(sa[c], v.c[c], a_.c[c]);
        mac128(sb[c], v.c[c], b_.c[c]);
      }
    };
    auto tensor_terms = [&](const V& x0, const V& y0) {
      const ShoupConst pm = pmod[i];
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const uint64_t py0 = shoup(y0.c[c], pm.w, pm.ws, p.q), py1 = shoup(y1.c[c], pm.w, pm.ws, p.q);
        mac128(sb[c], x0.c[c], py0);  // + P a0 b0
        if constexpr (FA) {           // + P (a0 b1 + a1 b0)
          fs[c] = __dadd_rn(fs[c], __dadd_rn(ksk_mul_f64(x0.c[c], py1, fq, fqinv), ksk_mul_f64(x1.c[c], py0, fq, fqinv)));
        } else {
          mac128(sa[c], x0.c[c], py1);
          mac128(sa[c], x1.c[c], py0);
        }
      }
    };
    if constexpr (MAXB > 0) {
      V v[MAXB], ka[MAXB], kb[MAXB];
#pragma unroll
      for (int d = 0; d < MAXB; ++d)
        if (d < beta) {
          if (SHARE_DIGITS) {
            v[d] = vd[d];
            ka[d] = kld<CPT>(J.key + (size_t)d * kstride + koff);
            kb[d] = kld<CPT>(J.key + (size_t)(dnum + d) * kstride + koff);
          } else {
            v[d] = kld<CPT>((d == own && J.x) ? J.x + off : J.digits + ((size_t)d * ext + i) * N + n);
            ka[d] = ka_g[d];
            kb[d] = kb_g[d];
          }
        }
      if (own >= 0 && J.x2) y1 = kld<CPT>(J.x2 + off);
      V x0{}, y0{};
      if (tensor) {
        x0 = kld<CPT>(J.a0 + off);
        y0 = kld<CPT>(J.b0 + off);
      }
#pragma unroll
      for (int d = 0; d < MAXB; ++d)
        if (d < beta) digit(d, v[d], ka[d], kb[d]);
      if (tensor) tensor_terms(x0, y0);
    } else {
      if (own >= 0 && J.x2) y1 = kld<CPT>(J.x2 + off);
      for (int d = 0; d < beta; ++d) {
        const uint64_t* src = (d == own && J.x) ? J.x + off : J.digits + ((size_t)d * ext + i) * N + n;
        digit(d, kld<CPT>(src), kld<CPT>(J.key + (size_t)d * kstride + koff),
              kld<CPT>(J.key + (size_t)(dnum + d) * kstride + koff));
      }
      if (tensor) {
        // every Q limb has one own digit, so x1 / y1 hold a1 / b1 here
        if (beta > 12) {  // keep the sums below 2^128: at most 15 products of two values < 2^62
#pragma unroll
          for (int c = 0; c < CPT; ++c) {
            sa[c] = U128{reduce128(sa[c], p), 0};
            sb[c] = U128{reduce128(sb[c], p), 0};
          }
        }
        tensor_terms(kld<CPT>(J.a0 + off), kld<CPT>(J.b0 + off));
      }
    }
    uint64_t ra[CPT], rb[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
      if constexpr (FA)
        ra[c] = ksk_canon_f64(fs[c], fq, fqinv);
      else
        ra[c] = reduce128(sa[c], p);
      rb[c] = reduce128(sb[c], p);
    }
    if (J.c0 && i < l) {
      const ShoupConst pm = pmod[i];
      const V cv = kld<CPT>(J.c0 + off);
#pragma unroll
      for (int c = 0; c < CPT; ++c) rb[c] = addmod(rb[c], shoup(cv.c[c], pm.w, pm.ws, p.q), p.q);
    }
    if (J.c0x) {
      const V cv = kld<CPT>(J.c0x + off);
#pragma unroll
      for (int c = 0; c < CPT; ++c) rb[c] = addmod(rb[c], cv.c[c], p.q);
    }
    uint64_t* oa = J.out_a + (size_t)i * N;
    uint64_t* ob = J.out_b + (size_t)i * N;
    if (J.auto_k) {
#pragma unroll
      for (int c = 0; c < CPT; ++c) {
        const uint32_t o = auto_slot(logN, J.auto_k, (uint32_t)(n + c));
        oa[o] = ra[c];
        ob[o] = rb[c];
      }
    } else if constexpr (CPT == 2) {
      *reinterpret_cast<ulonglong2*>(oa + n) = make_ulonglong2(ra[0], ra[1]);
      *reinterpret_cast<ulonglong2*>(ob + n) = make_ulonglong2(rb[0], rb[1]);
    } else {
      oa[n] = ra[0];
      ob[n] = rb[0];
    }
  };
  if constexpr (MAXB > 0 && SHARE_DIGITS) {
    V vd[MAXB];  // the group's digit tile (hoisted rotations of one ciphertext), read once
#pragma unroll
    for (int d = 0; d < MAXB; ++d)
      if (d < beta) vd[d] = kld<CPT>((d == own && J0.x) ? J0.x + off : J0.digits + ((size_t)d * ext + i) * N + n);
    if (fa_on) {
#pragma unroll
      for (int jj = 0; jj < JG; ++jj)
        if (jj < gn) run(L.j[g0 + jj], nullptr, nullptr, vd, std::true_type{});
    } else {
#pragma unroll
      for (int jj = 0; jj < JG; ++jj)
        if (jj < gn) run(L.j[g0 + jj], nullptr, nullptr, vd, std::false_type{});
    }
  } else if constexpr (MAXB > 0) {
    V ka[MAXB], kb[MAXB];  // the group's key tile, read once
#pragma unroll
    for (int d = 0; d < MAXB; ++d)
      if (d < beta) {
        ka[d] = kld<CPT>(J0.key + (size_t)d * kstride + koff);
        kb[d] = kld<CPT>(J0.key + (size_t)(dnum + d) * kstride + koff);
      }
    if (fa_on) {
#pragma unroll
      for (int jj = 0; jj < JG; ++jj)
        if (jj < gn) run(L.j[g0 + jj], ka, kb, nullptr, std::true_type{});
    } else {
#pragma unroll
      for (int jj = 0; jj < JG; ++jj)
        if (jj < gn) run(L.j[g0 + jj], ka, kb, nullptr, std::false_type{});
    }
  } else {
    for (int jj = 0; jj < gn; ++jj) run(L.j[g0 + jj], nullptr, nullptr, nullptr, std::false_type{});
  }
}

__global__ void __launch_bounds__(EW_THREADS) moddown_finish_kernel(const __grid_constant__ FinJobList L,
                                                                    const DevPrime* primes, const ShoupConst* pinv,
                                                                    int logN) {
  const FinJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l) return;
  const size_t off = ((size_t)j << logN) + blockIdx.x * blockDim.x + threadIdx.x;
  const DevPrime p = primes[j];
  const ShoupConst pi = pinv[j];
  uint64_t v = shoup(submod(J.x[off], J.conv[off], p.q), pi.w, pi.ws, p.q);
  if (J.add) v = addmod(v, J.add[off], p.q);
  J.out[off] = v;
}

__global__ void __launch_bounds__(EW_THREADS) tensor_kernel(const __grid_constant__ TensorJobList L,
                                                            const DevPrime* primes, int logN) {
  const TensorJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l) return;
  const size_t off = ((size_t)j << logN) + blockIdx.x * blockDim.x + threadIdx.x;
  const DevPrime p = primes[j];
  const uint64_t x0 = J.a0[off], x1 = J.a1[off], y0 = J.b0[off], y1 = J.b1[off];
  J.d0[off] = mulmod(x0, y0, p);
  U128 acc{0, 0};
  mac128(acc, x0, y1);
  mac128(acc, x1, y0);
  J.d1[off] = reduce128(acc, p);
  if (J.d2) J.d2[off] = mulmod(x1, y1, p);
}

__global__ void __launch_bounds__(EW_THREADS) switch_kernel(const __grid_constant__ SwitchJobList L,
                                                            const DevPrime* primes, int logN) {
  const SwitchJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l - 1) return;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const DevPrime om = primes[J.l - 1], nm = primes[j];
  J.out[((size_t)j << logN) + n] = switch_modulus(J.top[n], om, nm);
}

__global__ void __launch_bounds__(EW_THREADS) rescale_finish_kernel(const __grid_constant__ RescaleJobList L,
                                                                    const DevPrime* primes, const RescaleConst* rs,
                                                                    int logN, int n_q) {
  const RescaleJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l - 1) return;
  const size_t off = ((size_t)j << logN) + blockIdx.x * blockDim.x + threadIdx.x;
  const DevPrime p = primes[j];
  const RescaleConst r = rs[(size_t)J.l * n_q + j];
  uint64_t a = shoup(J.x[off], r.qinv, r.qinv_s, p.q);
  uint64_t b = shoup(J.t[off], r.m, r.m_s, p.q);
  J.out[off] = addmod(a, b, p.q);
}

__global__ void __launch_bounds__(EW_THREADS) addsub_kernel(const __grid_constant__ AddSubJobList L,
                                                            const DevPrime* primes, int logN) {
  const AddSubJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l) return;
  const size_t off = ((size_t)j << logN) + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const DevPrime p = primes[ext_prime(j, J.lq, J.nq)];
  const uint64_t q = p.q;
  const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(J.a + off);
  ulonglong2 y;
  if (J.sub >= EW_MUL_SCALAR) {
    y.x = y.y = J.b[j];
  } else {
    y = *reinterpret_cast<const ulonglong2*>(J.b + off);
  }
  ulonglong2 r;
  switch (J.sub) {
    case EW_SUB:
      r.x = submod(x.x, y.x, q);
      r.y = submod(x.y, y.y, q);
      break;
    case EW_MUL:
    case EW_MUL_SCALAR:
      r.x = mulmod(x.x, y.x, p);
      r.y = mulmod(x.y, y.y, p);
      break;
    default:  // EW_ADD, EW_ADD_SCALAR
      r.x = addmod(x.x, y.x, q);
      r.y = addmod(x.y, y.y, q);
  }
  *reinterpret_cast<ulonglong2*>(J.out + off) = r;
}

__global__ void __launch_bounds__(EW_THREADS) scalar_kernel(const __grid_constant__ ScalarJobList L,
                                                            const DevPrime* primes, int logN) {
  const ScalarJob& J = L.j[blockIdx.z];
  const int j = blockIdx.y;
  if (j >= J.l) return;
  const size_t off = ((size_t)j << logN) + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const DevPrime p = primes[j];
  const uint64_t sc = J.s[j];
  const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(J.a + off);
  ulonglong2 r;
  if (J.op == EW_MUL_SCALAR) {
    r.x = mulmod(x.x, sc, p);
    r.y = mulmod(x.y, sc, p);
  } else {
    r.x = addmod(x.x, sc, p.q);
    r.y = addmod(x.y, sc, p.q);
  }
  *reinterpret_cast<ulonglong2*>(J.out + off) = r;
}

// Two adjacent coefficients per thread; sums of up to 15 products (< 2^124 each) stay below
// 2^128 before a reduction.
constexpr int LC_BLOCK = 4;  // terms per block of loads (lincomb_kernel, dot_plain_kernel)

__global__ void __launch_bounds__(EW_THREADS) dot_plain_kernel(const __grid_constant__ DotJob J,
                                                               const DevPrime* primes, int logN) {
  const int lane = blockIdx.x, j = blockIdx.z;
  const DevPrime p = primes[ext_prime(j, J.lq, J.nq)];
  const size_t off = ((size_t)j << logN) + 2 * (blockIdx.y * blockDim.x + threadIdx.x);
  auto ld2 = [](const uint64_t* q) { return *reinterpret_cast<const ulonglong2*>(q); };
  U128 a0{0, 0}, a1{0, 0}, b0{0, 0}, b1{0, 0};
  for (int t0 = 0; t0 < J.n; t0 += LC_BLOCK) {  // as lincomb_kernel
    if (t0 && t0 % 12 == 0) {
      a0 = U128{reduce128(a0, p), 0};
      a1 = U128{reduce128(a1, p), 0};
      b0 = U128{reduce128(b0, p), 0};
      b1 = U128{reduce128(b1, p), 0};
    }
    ulonglong2 w[LC_BLOCK], x[LC_BLOCK], y[LC_BLOCK];
#pragma unroll
    for (int u = 0; u < LC_BLOCK; ++u)
      if (t0 + u < J.n) {
        w[u] = ld2(J.pt[t0 + u] + off);
        x[u] = ld2(J.c0[lane][t0 + u] + off);
        y[u] = ld2(J.c1[lane][t0 + u] + off);
      }
#pragma unroll
    for (int u = 0; u < LC_BLOCK; ++u)
      if (t0 + u < J.n) {
        mac128(a0, w[u].x, x[u].x);
        mac128(a1, w[u].y, x[u].y);
        mac128(b0, w[u].x, y[u].x);
        mac128(b1, w[u].y, y[u].y);
      }
  }
  *reinterpret_cast<ulonglong2*>(J.out0[lane] + off) = make_ulonglong2(reduce128(a0, p), reduce128(a1, p));
  *reinterpret_cast<ulonglong2*>(J.out1[lane] + off) = make_ulonglong2(reduce128(b0, p), reduce128(b1, p));
}

// One CTA per (giant step, lane, coefficient tile, limb): a thread loads its coefficient of the
// lane's baby steps and of the giant step's diagonals in one round of independent loads and
// forms one output pair.  The CTAs of one (tile, limb) are adjacent (giant step fastest, then
// lane), so the other giant steps' reads of a baby-step tile and the other lanes' reads of a
// diagonal tile come from L2: DRAM reads each tile once.  (Looping over the giant steps inside a
// thread exposed one memory latency per giant step: 15 long-scoreboard stalls per issue.)
// NB: register capacity for the baby steps.
template <int NB>
__global__ void __launch_bounds__(EW_THREADS) bsgs_dot_kernel(const __grid_constant__ BsgsJob J,
                                                              const DevPrime* primes, int logN) {
  const int i = blockIdx.x % J.ng, lane = blockIdx.x / J.ng, j = blockIdx.z;
  const DevPrime p = primes[ext_prime(j, J.lq, J.nq)];
  const size_t off = ((size_t)j << logN) + blockIdx.y * blockDim.x + threadIdx.x;
  uint64_t a[NB], b[NB], w[NB];
#pragma unroll
  for (int k = 0; k < NB; ++k)
    if (k < J.nb && J.pt[i][k]) {
      w[k] = J.pt[i][k][off];
      a[k] = J.x0[lane][k][off];
      b[k] = J.x1[lane][k][off];
    }
  U128 s0{0, 0}, s1{0, 0};
#pragma unroll
  for (int k = 0; k < NB; ++k) {
    if (k == 15) {  // keep the sums below 2^128: at most 15 products of values below 2^62
      s0 = U128{reduce128(s0, p), 0};
      s1 = U128{reduce128(s1, p), 0};
    }
    if (k < J.nb && J.pt[i][k]) {
      mac128(s0, w[k], a[k]);
      mac128(s1, w[k], b[k]);
    }
  }
  J.out0[lane][i][off] = reduce128(s0, p);
  J.out1[lane][i][off] = reduce128(s1, p);
}

// bsgs_dot_kernel with two consecutive coefficients per thread (16-byte loads and stores), for
// at most 8 baby steps (the products stay below 2^128 without an intermediate reduction) and
// operands whose addresses are 16-byte aligned (checked by the launcher).
__global__ void __launch_bounds__(EW_THREADS) bsgs_dot2_kernel(const __grid_constant__ BsgsJob J,
                                                               const DevPrime* primes, int logN) {
  constexpr int NB = 8;
  const int i = blockIdx.x % J.ng, lane = blockIdx.x / J.ng, j = blockIdx.z;
  const DevPrime p = primes[ext_prime(j, J.lq, J.nq)];
  const size_t off = ((size_t)j << logN) + 2 * ((size_t)blockIdx.y * blockDim.x + threadIdx.x);
  auto ld2 = [](const uint64_t* q) { return *reinterpret_cast<const ulonglong2*>(q); };
  ulonglong2 a[NB], b[NB], w[NB];
#pragma unroll
  for (int k = 0; k < NB; ++k)
    if (k < J.nb && J.pt[i][k]) {
      w[k] = ld2(J.pt[i][k] + off);
      a[k] = ld2(J.x0[lane][k] + off);
      b[k] = ld2(J.x1[lane][k] + off);
    }
  U128 s0x{0, 0}, s0y{0, 0}, s1x{0, 0}, s1y{0, 0};
#pragma unroll
  for (int k = 0; k < NB; ++k)
    if (k < J.nb && J.pt[i][k]) {
      mac128(s0x, w[k].x, a[k].x);
      mac128(s0y, w[k].y, a[k].y);
      mac128(s1x, w[k].x, b[k].x);
      mac128(s1y, w[k].y, b[k].y);
    }
  *reinterpret_cast<ulonglong2*>(J.out0[lane][i] + off) = ulonglong2{reduce128(s0x, p), reduce128(s0y, p)};
  *reinterpret_cast<ulonglong2*>(J.out1[lane][i] + off) = ulonglong2{reduce128(s1x, p), reduce128(s1y, p)};
}

__global__ void __launch_bounds__(EW_THREADS) lincomb_kernel(const __grid_constant__ LinCombJob J,
                                                             const DevPrime* primes, int logN) {
  const int j = blockIdx.y, lane = blockIdx.z;
  const DevPrime p = primes[ext_prime(j, J.lq, J.nq)];
  const size_t off = ((size_t)j << logN) + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  auto ld2 = [](const uint64_t* q) { return *reinterpret_cast<const ulonglong2*>(q); };
  U128 a0{0, 0}, a1{0, 0}, b0{0, 0}, b1{0, 0};
  // terms in blocks of LC_BLOCK whose loads are all issued before their products, so that a
  // thread waits for memory once per block rather than once per term; the sums are reduced
  // every 12 terms (below 2^128: a residue plus 12 products of values below 2^62)
  for (int t0 = 0; t0 < J.n; t0 += LC_BLOCK) {
    if (t0 && t0 % 12 == 0) {
      a0 = U128{reduce128(a0, p), 0};
      a1 = U128{reduce128(a1, p), 0};
      b0 = U128{reduce128(b0, p), 0};
      b1 = U128{reduce128(b1, p), 0};
    }
    ulonglong2 x[LC_BLOCK], y[LC_BLOCK];
#pragma unroll
    for (int u = 0; u < LC_BLOCK; ++u)
      if (t0 + u < J.n) {
        x[u] = ld2(J.x0[lane][t0 + u] + off);
        y[u] = ld2(J.x1[lane][t0 + u] + off);
      }
#pragma unroll
    for (int u = 0; u < LC_BLOCK; ++u)
      if (t0 + u < J.n) {
        const uint64_t w = J.s[t0 + u][j];
        mac128(a0, w, x[u].x);
        mac128(a1, w, x[u].y);
        mac128(b0, w, y[u].x);
        mac128(b1, w, y[u].y);
      }
  }
  const uint64_t ad = J.add0[j];
  *reinterpret_cast<ulonglong2*>(J.out0[lane] + off) =
      make_ulonglong2(addmod(reduce128(a0, p), ad, p.q), addmod(reduce128(a1, p), ad, p.q));
  *reinterpret_cast<ulonglong2*>(J.out1[lane] + off) = make_ulonglong2(reduce128(b0, p), reduce128(b1, p));
}

template <typename List, typename Job>
int fill(List& L, const Job* jobs, int n) {
  L.n = n;
  std::copy(jobs, jobs + n, L.j);
  return n;
}

}  // namespace

int kernel_binary_version(int device) {
  FIDES_CUDA(cudaSetDevice(device));
  cudaFuncAttributes a{};
  FIDES_CUDA(cudaFuncGetAttributes(&a, addsub_kernel));
  return a.binaryVersion;
}

void launch_conv(Context* c, const ConvJob* jobs, int n, cudaStream_t s) {
  static thread_local ConvJobList L;
  // Tables with a tensor-core form go to the tcgen05 kernel unless the SIMT engine is forced;
  // the rest are grouped by source width so each launch uses one specialised kernel.
  std::vector<ConvJob> tc;
  std::vector<ConvJob> byw[MAX_SRC + 1];
  const bool use_tc = c->conv_engine == CONV_TENSOR || (c->conv_engine == CONV_AUTO && kConvAutoTensor);
  for (int i = 0; i < n; ++i) {
    const ConvTable& t = jobs[i].t;
    if (t.n_src > MAX_SRC || t.n_dst > MAX_DST || t.n_src < 1) throw Error(-1, "basis conversion width out of range");
    if (use_tc && t.tc_b)
      tc.push_back(jobs[i]);
    else
      byw[t.n_src].push_back(jobs[i]);
  }
  if (!tc.empty()) launch_conv_tc(c, tc.data(), (int)tc.size(), s);
  for (int w = 1; w <= MAX_SRC; ++w) {
    const auto& v = byw[w];
    for (size_t off = 0; off < v.size(); off += MAX_CONV_JOBS) {
      int m = (int)std::min<size_t>(MAX_CONV_JOBS, v.size() - off);
      fill(L, v.data() + off, m);
      size_t smem = 0;
      double bytes = 0;
      for (int i = 0; i < m; ++i) {
        const ConvTable& t = L.j[i].t;
        smem = std::max(smem, (size_t)(t.n_src + t.lift) * t.n_dst * 8 + (size_t)t.n_src * 16 + (size_t)t.n_dst * 68);
        bytes += 8.0 * c->N * (t.n_src + t.n_dst);
      }
      dim3 grid(c->N / (2 * EW_THREADS), m);
      LaunchScope ls(c, s, KK_CONV, bytes);
      switch (w) {
#define FIDES_CONV_CASE(K)                                                                                    \
  case K: {                                                                                                   \
    static bool attr = false;                                                                                 \
    if (!attr) {                                                                                              \
      FIDES_CUDA(cudaFuncSetAttribute(conv_kernel<K>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)); \
      attr = true;                                                                                            \
    }                                                                                                         \
    conv_kernel<K><<<grid, EW_THREADS, smem, s>>>(L, c->d_prime, c->logN);                                    \
    break;                                                                                                    \
  }
        FIDES_CONV_CASE(1) FIDES_CONV_CASE(2) FIDES_CONV_CASE(3) FIDES_CONV_CASE(4) FIDES_CONV_CASE(5)
        FIDES_CONV_CASE(6) FIDES_CONV_CASE(7) FIDES_CONV_CASE(8) FIDES_CONV_CASE(9) FIDES_CONV_CASE(10)
        FIDES_CONV_CASE(11) FIDES_CONV_CASE(12) FIDES_CONV_CASE(13) FIDES_CONV_CASE(14) FIDES_CONV_CASE(15)
        FIDES_CONV_CASE(16)
#undef FIDES_CONV_CASE
        default: {
          static bool attr = false;
          if (!attr) {
            FIDES_CUDA(cudaFuncSetAttribute(conv_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr = true;
          }
          conv_kernel<0><<<grid, EW_THREADS, smem, s>>>(L, c->d_prime, c->logN);
        }
      }
      FIDES_CUDA(cudaGetLastError());
    }
  }
}

void launch_dot_plain(Context* c, const DotJob& job, cudaStream_t s) {
  if (job.n < 1 || job.n > MAX_DOT_TERMS) throw Error(-1, "dot product needs 1..32 terms");
  if (job.lanes < 1 || job.lanes > MAX_DOT_LANES) throw Error(-1, "dot product needs 1..8 lanes");
  dim3 grid(job.lanes, c->N / (2 * EW_THREADS), job.l);
  LaunchScope ls(c, s, KK_ELEM, 8.0 * c->N * job.l * (job.n + job.lanes * (2.0 * job.n + 2)));
  dot_plain_kernel<<<grid, EW_THREADS, 0, s>>>(job, c->d_prime, c->logN);
  FIDES_CUDA(cudaGetLastError());
}

void launch_bsgs_dot(Context* c, const BsgsJob& job, cudaStream_t s) {
  if (job.nb < 1 || job.nb > MAX_BSGS_BABY || job.ng < 1 || job.ng > MAX_BSGS_GIANT || job.lanes < 1 ||
      job.lanes > MAX_BSGS_LANES || job.l < 1)
    throw Error(-1, "BSGS inner products need 1..16 baby steps, 1..16 giant steps, 1..8 lanes");
  int terms = 0;
  for (int i = 0; i < job.ng; ++i)
    for (int k = 0; k < job.nb; ++k) terms += job.pt[i][k] != nullptr;
  bool aligned = c->N >= 2 * EW_THREADS;  // the paired form: 16-byte aligned operands, a whole tile of pairs
  auto al = [&](const void* q) { aligned = aligned && (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  for (int i = 0; i < job.ng; ++i)
    for (int k = 0; k < job.nb; ++k)
      if (job.pt[i][k]) al(job.pt[i][k]);
  for (int ln = 0; ln < job.lanes; ++ln) {
    for (int k = 0; k < job.nb; ++k) al(job.x0[ln][k]), al(job.x1[ln][k]);
    for (int i = 0; i < job.ng; ++i) al(job.out0[ln][i]), al(job.out1[ln][i]);
  }
  LaunchScope ls(c, s, KK_ELEM, 8.0 * c->N * job.l * (terms + job.lanes * 2.0 * (job.nb + job.ng)));
  if (job.nb <= 8 && aligned) {
    dim3 grid2(job.lanes * job.ng, c->N / (2 * EW_THREADS), job.l);
    bsgs_dot2_kernel<<<grid2, EW_THREADS, 0, s>>>(job, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
    return;
  }
  dim3 grid(job.lanes * job.ng, c->N / EW_THREADS, job.l);
  if (job.nb <= 8)
    bsgs_dot_kernel<8><<<grid, EW_THREADS, 0, s>>>(job, c->d_prime, c->logN);
  else
    bsgs_dot_kernel<MAX_BSGS_BABY><<<grid, EW_THREADS, 0, s>>>(job, c->d_prime, c->logN);
  FIDES_CUDA(cudaGetLastError());
}

void launch_lincomb(Context* c, const LinCombJob& job, cudaStream_t s) {
  if (job.n < 1 || job.n > MAX_LC_TERMS || job.l < 1 || job.l > MAX_LC_LIMBS || job.lanes < 1 ||
      job.lanes > MAX_LC_LANES)
    throw Error(-1, "linear combination needs 1..16 terms of 1..64 limbs in 1..8 lanes");
  dim3 grid(c->N / (2 * EW_THREADS), job.l, job.lanes);
  LaunchScope ls(c, s, KK_ELEM, 8.0 * c->N * job.l * job.lanes * (2.0 * job.n + 2));
  lincomb_kernel<<<grid, EW_THREADS, 0, s>>>(job, c->d_prime, c->logN);
  FIDES_CUDA(cudaGetLastError());
}

void launch_ksk(Context* c, const KskJob* jobs, int n, cudaStream_t s) {
  static thread_local KskJobList L;
  for (int off = 0; off < n; off += MAX_KSK_JOBS) {
    int m = std::min(MAX_KSK_JOBS, n - off);
    fill(L, jobs + off, m);
    // groups of consecutive jobs with one key, level and set of extras (a batch under one
    // switching key), or else with one digit set (hoisted rotations of one ciphertext)
    auto same_key = [](const KskJob& a, const KskJob& b) {
      return a.key == b.key && a.l == b.l && a.auto_k == b.auto_k && !a.x2 == !b.x2 && !a.a0 == !b.a0 &&
             !a.c0 == !b.c0 && !a.x == !b.x && !a.c0x == !b.c0x;
    };
    auto same_digits = [](const KskJob& a, const KskJob& b) {
      return a.digits == b.digits && a.x == b.x && a.x2 == b.x2 && a.l == b.l && !a.a0 == !b.a0 && !a.c0 == !b.c0 &&
             !a.c0x == !b.c0x;
    };
    // groups of up to MAX_KSK_GROUP jobs sharing a key, or else sharing a digit tile
    auto group = [&](auto same, int cap) {
      L.ngroups = 0;
      int gm = 1;
      for (int i = 0; i < m;) {
        int k = 1;
        while (i + k < m && k < cap && same(L.j[i], L.j[i + k])) ++k;
        L.gstart[L.ngroups] = (uint8_t)i;
        L.gcount[L.ngroups] = (uint8_t)k;
        ++L.ngroups;
        gm = std::max(gm, k);
        i += k;
      }
      return gm;
    };
    int gmax = group(same_key, MAX_KSK_GROUP);
    bool share_digits = false;
    if (gmax == 1) {
      gmax = group(same_digits, 4);
      share_digits = gmax > 1;
      if (!share_digits) group(same_key, MAX_KSK_GROUP);
    }
    int mx = 0;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l + c->K);
    const int jg = gmax == 1 ? 1 : gmax == 2 ? 2 : 4;
    int maxb = 0;
    for (int i = 0; i < m; ++i) maxb = std::max(maxb, c->beta(L.j[i].l));
    dim3 grid(c->N / (2 * EW_THREADS), mx, L.ngroups);
    // algorithmic bytes: each job's digits, outputs and extra operands, and each group's key once
    double bytes = 0;
    for (int i = 0; i < m; ++i) {
      const int l = L.j[i].l, ext = l + c->K, b = c->beta(l);
      bytes += 8.0 * c->N * ((double)ext * (b + 2) + (L.j[i].c0 ? l : 0) + (L.j[i].a0 ? 2 * l : 0) +
                             (L.j[i].c0x ? ext : 0));
    }
    for (int g = 0; g < L.ngroups; ++g) {
      const int l = L.j[L.gstart[g]].l, b = c->beta(l), ext = l + c->K;
      // the shared tile once per group, the other per job
      bytes += 8.0 * c->N * (share_digits ? (double)b * ext + 2.0 * b * ext * L.gcount[g] - (double)b * ext * L.gcount[g]
                                          : 2.0 * b * ext);
    }
    LaunchScope ls(c, s, KK_KSK, bytes);
    auto go = [&](auto kern) { kern<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->d_pmod, c->d_f64, c->logN, c->n_q,
                                                              c->K, c->dnum, c->alpha); };
    switch (maxb * 16 + jg + (share_digits ? 128 : 0)) {
#define FIDES_KSK_CASE(B, G)                    \
  case B * 16 + G:                              \
    go(ksk_kernel<B, G, 2>);                    \
    break;                                      \
  case 128 + B * 16 + G:                        \
    go(ksk_kernel<B, G, 2, true>);              \
    break;
      FIDES_KSK_CASE(1, 1) FIDES_KSK_CASE(1, 2) FIDES_KSK_CASE(1, 4)
      FIDES_KSK_CASE(2, 1) FIDES_KSK_CASE(2, 2) FIDES_KSK_CASE(2, 4)
      FIDES_KSK_CASE(3, 1) FIDES_KSK_CASE(3, 2) FIDES_KSK_CASE(3, 4)
      FIDES_KSK_CASE(4, 1) FIDES_KSK_CASE(4, 2) FIDES_KSK_CASE(4, 4)
#undef FIDES_KSK_CASE
      default:
        go(ksk_kernel<0, 1, 2>);
    }
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_moddown_finish(Context* c, const FinJob* jobs, int n, cudaStream_t s) {
  static thread_local FinJobList L;
  for (int off = 0; off < n; off += MAX_FIN_JOBS) {
    int m = std::min(MAX_FIN_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 0;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l);
    dim3 grid(c->N / EW_THREADS, mx, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * ((L.j[i].add ? 4.0 : 3.0) * L.j[i].l);
    LaunchScope ls(c, s, KK_ELEM, bytes);
    moddown_finish_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->d_pinv, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_tensor(Context* c, const TensorJob* jobs, int n, cudaStream_t s) {
  static thread_local TensorJobList L;
  for (int off = 0; off < n; off += MAX_TENSOR_JOBS) {
    int m = std::min(MAX_TENSOR_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 0;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l);
    dim3 grid(c->N / EW_THREADS, mx, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * ((L.j[i].d2 ? 7.0 : 6.0) * L.j[i].l);
    LaunchScope ls(c, s, KK_ELEM, bytes);
    tensor_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_switch_modulus(Context* c, const SwitchJob* jobs, int n, cudaStream_t s) {
  static thread_local SwitchJobList L;
  for (int off = 0; off < n; off += MAX_RS_JOBS) {
    int m = std::min(MAX_RS_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 1;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l - 1);
    dim3 grid(c->N / EW_THREADS, mx, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * (1.0 + (L.j[i].l - 1));
    LaunchScope ls(c, s, KK_ELEM, bytes);
    switch_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_rescale_finish(Context* c, const RescaleJob* jobs, int n, cudaStream_t s) {
  static thread_local RescaleJobList L;
  for (int off = 0; off < n; off += MAX_RS_JOBS) {
    int m = std::min(MAX_RS_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 1;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l - 1);
    dim3 grid(c->N / EW_THREADS, mx, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * (3.0 * (L.j[i].l - 1));
    LaunchScope ls(c, s, KK_ELEM, bytes);
    rescale_finish_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->d_rescale, c->logN, c->n_q);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_addsub(Context* c, const AddSubJob* jobs, int n, cudaStream_t s) {
  static thread_local AddSubJobList L;
  for (int off = 0; off < n; off += MAX_ADDSUB_JOBS) {
    int m = std::min(MAX_ADDSUB_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 1;
    double bytes = 0;
    for (int i = 0; i < m; ++i) {
      mx = std::max(mx, L.j[i].l);
      bytes += 8.0 * c->N * 3.0 * L.j[i].l;
    }
    dim3 grid(c->N / (2 * EW_THREADS), mx, m);
    LaunchScope ls(c, s, KK_ELEM, bytes);
    addsub_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_scalar(Context* c, const ScalarJob* jobs, int n, cudaStream_t s) {
  static thread_local ScalarJobList L;
  for (int off = 0; off < n; off += MAX_SCALAR_JOBS) {
    int m = std::min(MAX_SCALAR_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 1;
    double bytes = 0;
    for (int i = 0; i < m; ++i) {
      if (L.j[i].l > MAX_SCALAR_LIMBS) throw Error(-1, "scalar op on more than 64 limbs");
      mx = std::max(mx, L.j[i].l);
      bytes += 8.0 * c->N * 2.0 * L.j[i].l;
    }
    dim3 grid(c->N / (2 * EW_THREADS), mx, m);
    LaunchScope ls(c, s, KK_ELEM, bytes);
    scalar_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

}  // namespace fides
