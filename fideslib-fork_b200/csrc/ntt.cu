// Negacyclic NTT / INTT kernels (see ntt.cuh for the design).
#include <algorithm>
#include <vector>

#include "ntt.cuh"

namespace fides {

namespace {

constexpr int COL = 0, ROW = 1;
constexpr int LOGE = 4;  // 16 elements per thread
constexpr int G = 16;    // sub-transforms per CTA

__device__ __forceinline__ ShoupConst ld_tw(const ShoupConst* p) {
  ulonglong2 v = __ldg(reinterpret_cast<const ulonglong2*>(p));
  return ShoupConst{v.x, v.y};
}

// Cooley-Tukey butterfly, Harvey lazy form: x, y in [0, 4q) -> [0, 4q).
__device__ __forceinline__ void ct_bf(uint64_t& x, uint64_t& y, ShoupConst w, uint64_t q, uint64_t q2) {
  uint64_t a = csub(x, q2);
  uint64_t t = shoup_lazy(y, w.w, w.ws, q);
  x = a + t;
  y = a - t + q2;
}

// Gentleman-Sande butterfly, Harvey lazy form: x, y in [0, 2q) -> [0, 2q).
__device__ __forceinline__ void gs_bf(uint64_t& x, uint64_t& y, ShoupConst w, uint64_t q, uint64_t q2) {
  uint64_t s = csub(x + y, q2);
  uint64_t d = x - y + q2;
  y = shoup_lazy(d, w.w, w.ws, q);
  x = s;
}

struct PassArgs {
  const DevPrime* primes;
  const ShoupConst* tw;        // forward or inverse twiddles, [prime][N]
  const ShoupConst* inv_last;  // [prime]: psi_rev^-1[1] * N^-1
  int logN;
  int log1;  // size of the column sub-transform
};

// Element index u of register r for thread t, when the register index spans bits
// [lo, lo + LOGE) of u.
template <int LO>
__device__ __forceinline__ int u_of(int t, int r) {
  return ((t >> LO) << (LO + LOGE)) | (r << LO) | (t & ((1 << LO) - 1));
}

template <int LOGP>
__device__ __forceinline__ int padu(int u) {
  return u + (u >> LOGE);
}

// Butterflies of pair bits [BLO, BHI] (in u) for a thread whose registers span bits
// [LO, LO + LOGE).  FWD walks bits high -> low, inverse low -> high.
template <int LOGP, int LO, int BHI, int BLO, bool FWD, int PASS>
__device__ __forceinline__ void run_chunk(uint64_t (&x)[1 << LOGE], int t, int sub, int sbase, const ShoupConst* tw,
                                          const DevPrime& pr, ShoupConst last) {
  constexpr int E = 1 << LOGE;
  const int th = t >> LO;
#pragma unroll
  for (int k = 0; k <= BHI - BLO; ++k) {
    const int b = FWD ? (BHI - k) : (BLO + k);
    const int rb = b - LO;
    const int sig = LOGP - 1 - b;  // stage within this pass
    const int s = sbase + sig;     // global stage
    const uint32_t base = (1u << s) + ((uint32_t)sub << sig) + ((uint32_t)th << (LO + LOGE - b - 1));
#pragma unroll
    for (int hi = 0; hi < (E >> (rb + 1)); ++hi) {
      if (!FWD && PASS == COL && b == LOGP - 1) {
        // last inverse stage (global stage 0): fold N^-1 into both outputs
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          uint64_t a = x[r0], c = x[r1];
          x[r0] = shoup(a + c, pr.ninv, pr.ninv_s, pr.q);
          x[r1] = shoup(a - c + pr.q2, last.w, last.ws, pr.q);
        }
      } else {
        const ShoupConst w = ld_tw(tw + base + hi);
#pragma unroll
        for (int lr = 0; lr < (1 << rb); ++lr) {
          const int r0 = (hi << (rb + 1)) | lr, r1 = r0 | (1 << rb);
          if (FWD)
            ct_bf(x[r0], x[r1], w, pr.q, pr.q2);
          else
            gs_bf(x[r0], x[r1], w, pr.q, pr.q2);
        }
      }
    }
  }
}

// Register span of chunk c.
template <int LOGP, bool FWD, int C>
struct Chunk {
  // forward: bits from the top; inverse: bits from the bottom
  static constexpr int BHI = FWD ? (LOGP - 1 - C * LOGE) : (C * LOGE + LOGE - 1 < LOGP - 1 ? C * LOGE + LOGE - 1 : LOGP - 1);
  static constexpr int BLO = FWD ? (LOGP - (C + 1) * LOGE > 0 ? LOGP - (C + 1) * LOGE : 0) : C * LOGE;
  static constexpr int LO = FWD ? BLO : (BLO + LOGE <= LOGP ? BLO : LOGP - LOGE);
};

template <int LOGP, int PASS, bool FWD>
__global__ void __launch_bounds__((1 << (LOGP - LOGE)) * G) ntt_pass(const PassArgs a, const __grid_constant__ NttLimbList L) {
  constexpr int P = 1 << LOGP, E = 1 << LOGE, T = P / E, NT = T * G;
  constexpr int NCH = (LOGP + LOGE - 1) / LOGE;
  constexpr int PADP = P + P / E;
  extern __shared__ uint64_t sm[];

  const LimbRef lr = L.limbs[blockIdx.y];
  const DevPrime pr = a.primes[lr.prime];
  const int N = 1 << a.logN;
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
  const int S = N >> LOGP;  // stride of a column (COL) / number of rows (ROW)
  const int sub0 = blockIdx.x * G;
  const int sub = sub0 + g;
  const int sbase = PASS == COL ? 0 : a.log1;
  const int subtw = PASS == COL ? 0 : sub;

  auto gidx = [&](int s_, int u) -> size_t {
    return PASS == COL ? (size_t)s_ + (size_t)u * S : (size_t)s_ * P + u;
  };
  auto sidx = [&](int gg, int u) -> int { return PASS == COL ? u * G + gg : gg * PADP + padu<LOGP>(u); };

  uint64_t x[E];

  // ---- load chunk 0 (direct when lanes map to consecutive addresses, else staged)
  constexpr int LO0 = Chunk<LOGP, FWD, 0>::LO;
  constexpr bool direct_load = (PASS == COL) || (LO0 == LOGP - LOGE);
  if (direct_load) {
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = data[gidx(sub, u_of<LO0>(t, r))];
  } else {
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = k * NT + tid;
      int gg = e / P, u = e % P;
      sm[sidx(gg, u)] = data[gidx(sub0 + gg, u)];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<LO0>(t, r))];
  }

  // ---- chunks
  run_chunk<LOGP, Chunk<LOGP, FWD, 0>::LO, Chunk<LOGP, FWD, 0>::BHI, Chunk<LOGP, FWD, 0>::BLO, FWD, PASS>(
      x, t, subtw, sbase, tw, pr, last);
  if constexpr (NCH > 1) {
    constexpr int LO1 = Chunk<LOGP, FWD, 1>::LO;
    if (!direct_load) __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<LO0>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<LO1>(t, r))];
    run_chunk<LOGP, LO1, Chunk<LOGP, FWD, 1>::BHI, Chunk<LOGP, FWD, 1>::BLO, FWD, PASS>(x, t, subtw, sbase, tw, pr,
                                                                                          last);
  }
  if constexpr (NCH > 2) {
    constexpr int LO1 = Chunk<LOGP, FWD, 1>::LO;
    constexpr int LO2 = Chunk<LOGP, FWD, 2>::LO;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<LO1>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = sm[sidx(g, u_of<LO2>(t, r))];
    run_chunk<LOGP, LO2, Chunk<LOGP, FWD, 2>::BHI, Chunk<LOGP, FWD, 2>::BLO, FWD, PASS>(x, t, subtw, sbase, tw, pr,
                                                                                          last);
  }
  static_assert(NCH <= 3, "sub-transform too large");

  // ---- final reduction of the completed transform
  const bool final_pass = FWD ? (PASS == ROW) : (PASS == COL);
  if (final_pass && FWD) {
#pragma unroll
    for (int r = 0; r < E; ++r) x[r] = csub(csub(x[r], pr.q2), pr.q);
  }

  // ---- store
  constexpr int LOL = Chunk<LOGP, FWD, NCH - 1>::LO;
  constexpr bool direct_store = (PASS == COL) || (LOL == LOGP - LOGE);
  if (direct_store) {
#pragma unroll
    for (int r = 0; r < E; ++r) data[gidx(sub, u_of<LOL>(t, r))] = x[r];
  } else {
    __syncthreads();
#pragma unroll
    for (int r = 0; r < E; ++r) sm[sidx(g, u_of<LOL>(t, r))] = x[r];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = k * NT + tid;
      int gg = e / P, u = e % P;
      data[gidx(sub0 + gg, u)] = sm[sidx(gg, u)];
    }
  }
}

template <int LOGP, int PASS, bool FWD>
void launch_pass(Context* c, const PassArgs& a, const NttLimbList& L, cudaStream_t s) {
  constexpr int P = 1 << LOGP, T = P / (1 << LOGE);
  const int smem = (PASS == COL ? P * G : G * (P + P / (1 << LOGE))) * (int)sizeof(uint64_t);
  static bool attr_set = false;  // per instantiation; set before first launch
  if (!attr_set) {
    FIDES_CUDA(cudaFuncSetAttribute(ntt_pass<LOGP, PASS, FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set = true;
  }
  dim3 grid((c->N >> LOGP) / G, L.n);
  // algorithmic bytes: half of a transform's read + write of each limb (two passes)
  LaunchScope ls(c, s, KK_NTT, 8.0 * c->N * L.n);
  ntt_pass<LOGP, PASS, FWD><<<grid, T * G, smem, s>>>(a, L);
  FIDES_CUDA(cudaGetLastError());
}

template <int PASS, bool FWD>
void dispatch(Context* c, int logp, const PassArgs& a, const NttLimbList& L, cudaStream_t s) {
  switch (logp) {
    case 5: launch_pass<5, PASS, FWD>(c, a, L, s); break;
    case 6: launch_pass<6, PASS, FWD>(c, a, L, s); break;
    case 7: launch_pass<7, PASS, FWD>(c, a, L, s); break;
    case 8: launch_pass<8, PASS, FWD>(c, a, L, s); break;
    case 9: launch_pass<9, PASS, FWD>(c, a, L, s); break;
    default: throw Error(-1, "unsupported NTT pass size 2^" + std::to_string(logp));
  }
}

}  // namespace

void ntt_limbs(Context* c, const LimbRef* limbs, int n, bool inverse, cudaStream_t s) {
  if (n <= 0) return;
  if (c->logN < 10) throw Error(-1, "GPU NTT needs logN >= 10");
  const int log1 = (c->logN + 1) / 2, log2 = c->logN / 2;
  PassArgs a;
  a.primes = c->d_prime;
  a.tw = inverse ? c->d_tw_inv : c->d_tw_fwd;
  a.inv_last = c->d_inv_last;
  a.logN = c->logN;
  a.log1 = log1;
  static thread_local NttLimbList L;  // 16 KB: keep off the stack
  for (int off = 0; off < n; off += MAX_NTT_LIMBS) {
    L.n = std::min(MAX_NTT_LIMBS, n - off);
    std::copy(limbs + off, limbs + off + L.n, L.limbs);
    if (!inverse) {
      dispatch<COL, true>(c, log1, a, L, s);
      dispatch<ROW, true>(c, log2, a, L, s);
    } else {
      dispatch<ROW, false>(c, log2, a, L, s);
      dispatch<COL, false>(c, log1, a, L, s);
    }
  }
}

void ntt_polys(Context* c, uint64_t* data, int n_polys, int n_limbs, const int* prime_ids, bool inverse,
               cudaStream_t s) {
  std::vector<LimbRef> v((size_t)n_polys * n_limbs);
  for (int p = 0; p < n_polys; ++p)
    for (int i = 0; i < n_limbs; ++i)
      v[(size_t)p * n_limbs + i] = LimbRef{data + ((size_t)p * n_limbs + i) * c->N, prime_ids[i], 0};
  ntt_limbs(c, v.data(), (int)v.size(), inverse, s);
}

}  // namespace fides
