// Tensor-core basis conversion (tcgen05, kind::i8).  The arithmetic identity is stated in
// conv_tc.hpp; this file holds the table builder and the kernel.
//
// One CTA converts 128 coefficients (the MMA's M, one TMEM lane each) of one job:
//   1. warp 0 allocates 64 TMEM columns; the CTA starts cp.async copies of the table's B image
//      (the shared-memory form of the byte matrix) and, while they are in flight, writes A: the
//      eight bytes of every pre-scaled residue y_i of its 128 coefficients, K-major;
//   2. per chunk of 8 destination limbs (64 columns: 8 byte planes each), thread 0 issues
//      K/32 MMAs (M 128, N 8 x limbs, K 32) and commits them to an mbarrier;
//   3. after a bounded wait, each warp reads its 32 TMEM lanes (tcgen05.ld 32x32b), folds the
//      eight s32 planes of each output into 64 bits and reduces modulo the destination prime.
// Operands use the no-swizzle K-major canonical layout: core matrices of 8 rows x 16 bytes,
// rows 16 bytes apart, 8-row groups 128 bytes apart (SBO) and the two 16-byte K halves of an
// MMA LBO apart.  A is stored as [K/16][128 rows][16 B], B as [K/16][8 nd_pad rows][16 B].
#include <algorithm>
#include <cstring>

#include "conv_tc.hpp"
#include "kernels.cuh"

#ifndef FIDES_TC_SMEM_GUARD
#define FIDES_TC_SMEM_GUARD 0
#endif

namespace fides {

void build_tc_image(const uint64_t* mat, int ns, int nd, const std::vector<int>& dst_prime,
                    const uint64_t* primes, std::vector<uint8_t>& b, std::vector<TcDest>& dst,
                    int& kpad, int& nd_pad) {
  kpad = tc_kpad(ns);
  nd_pad = tc_nd_pad(nd);
  const int nb = 8 * nd_pad;  // B rows
  b.assign((size_t)kpad * nb, 0);
  dst.assign(nd_pad, TcDest{0, 0});
  for (int j = 0; j < nd; ++j) {
    const uint64_t p = primes[dst_prime[j]];
    const double qinv = 1.0 / (double)p;
    dst[j].q = p;
    std::memcpy(&dst[j].qinv, &qinv, sizeof(double));
    for (int i = 0; i < ns; ++i)
      for (int a = 0; a < 8; ++a) {
        const uint64_t v = h_mulmod(mat[(size_t)i * nd + j] % p, h_powmod(2, 8 * a, p), p);
        const int k = 8 * i + a;
        for (int cb = 0; cb < 8; ++cb) {
          const int n = 8 * j + cb;
          b[((size_t)(k / 16) * nb + n) * 16 + (k % 16)] = (uint8_t)(v >> (8 * cb));
        }
      }
  }
}

namespace {

constexpr int TC_M = 128;          // coefficients per CTA = TMEM lanes = MMA M
constexpr int TC_DCHUNK = 8;       // destination limbs per MMA chunk
constexpr uint32_t TC_COLS = 64;   // TMEM columns held by one CTA (8 limbs x 8 byte planes)
// Shared memory of at least this size per CTA keeps at most 7 CTAs (448 TMEM columns of the
// SM's 512) resident, so tcgen05.alloc never waits for another CTA.
constexpr int TC_SMEM_FLOOR = 29 * 1024;

struct TcLayout {
  int o_dst, o_pos, o_a, o_b, total;
};
__host__ __device__ inline TcLayout tc_layout(int kpad, int ndp) {
  TcLayout L;
  L.o_dst = 16;  // [0, 8): mbarrier, [8, 12): TMEM address
  L.o_pos = L.o_dst + ndp * (int)sizeof(TcDest);
  L.o_a = (L.o_pos + ndp * 4 + 127) & ~127;
  L.o_b = L.o_a + TC_M * kpad;
  L.total = L.o_b + kpad * 8 * ndp;
  return L;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle, sm_100 descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor, kind::i8: s32 accumulator (bits 4-5 = 2), A and B unsigned
// (formats 0), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
__device__ __forceinline__ uint32_t idesc_u8(int n) {
  return (2u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint32_t bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(phase)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the barrier phase for at most about one second; false if it gave up.
__device__ bool bar_wait_bounded(uint32_t bar, uint32_t phase) {
  const uint64_t t0 = globaltimer();
  for (uint32_t it = 1;; ++it) {
    if (bar_try_wait(bar, phase)) return true;
    if ((it & 63) == 0 && globaltimer() - t0 > 1000000000ull) return false;
  }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&d)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
// Orders later uses of d after tcgen05.wait::ld.
__device__ __forceinline__ void pin8(uint32_t (&d)[8]) {
  asm volatile("" : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3]), "+r"(d[4]), "+r"(d[5]), "+r"(d[6]), "+r"(d[7]));
}

// sum_c 2^(8c) d[c] mod q for planes d[c] < 2^23 and a prime 2^48 < q < 2^62.
// V = x + 2^32 y with x, y < 2^49 (V < 2^79.01 for K <= 128) is reduced by floating-point
// Barrett reduction (the double-precision quotient estimate of NTL's MulMod): the integers
// x, y convert to doubles exactly (2^52 exponent trick), and vd = fl(V), qinv = fl(1/q) give
// vd qinv within 2^-20 of V/q (V/q < 2^31.01); the fma adds 2^-17 with one more rounding of
// at most 2^-21, so t lies in (V/q + 2^-17.6, V/q + 2^-16.6) and qh = floor(t) is
// floor(V/q) or one more (qh < 2^32).  V - qh q lies in [-q, q), is computed exactly in
// wrapping 64-bit arithmetic and needs one correction.  (Checked against 128-bit arithmetic
// on 40 M random, extreme and next-to-a-multiple-of-q plane sets over 4000 primes.)
__device__ __forceinline__ uint64_t tc_fold(const uint32_t (&d)[8], uint64_t q, double qinv) {
  const uint32_t a0 = d[0] + (d[1] << 8), a1 = d[2] + (d[3] << 8);  // < 2^32
  const uint32_t a2 = d[4] + (d[5] << 8), a3 = d[6] + (d[7] << 8);
  const uint64_t x = (uint64_t)a0 + ((uint64_t)a1 << 16);  // planes 0-3, < 2^49
  const uint64_t y = (uint64_t)a2 + ((uint64_t)a3 << 16);  // planes 4-7 (weight 2^32), < 2^49
  const double two52 = 4503599627370496.0;
  const double xd = __longlong_as_double((long long)(0x4330000000000000ull | x)) - two52;
  const double yd = __longlong_as_double((long long)(0x4330000000000000ull | y)) - two52;
  const double vd = fma(yd, 4294967296.0, xd);
  const uint32_t qh = (uint32_t)__double2loint(__dadd_rd(fma(vd, qinv, 0x1p-17), two52));  // floor, < 2^32
  uint64_t r = x + (y << 32) - (uint64_t)qh * q;
  return r + ((uint64_t)((int64_t)r >> 63) & q);
}

// Stores the folded outputs of one chunk of NDC destination limbs (8 byte-plane columns each,
// starting at TMEM address trow).  The TMEM loads of the next pair are in flight while the
// current pair is folded; tcgen05.wait::ld waits for all of them, so each wait follows the
// fold of the pair loaded before it.  dofs[j] = output limb position of destination j times N.
template <int NDC, bool CHECK>
__device__ __forceinline__ void tc_epilogue(uint32_t trow, int j0, int nd, const TcDest* dconst, const int* dofs,
                                            uint64_t* out) {
  uint32_t d[2][2][8];
  tmem_ld8(trow, d[0][0]);
  tmem_ld8(trow + 8, d[0][1]);
  tmem_wait_ld();
#pragma unroll
  for (int h = 0; h < NDC / 2; ++h) {
    const int cur = h & 1, nxt = cur ^ 1;
    if (h + 1 < NDC / 2) {
      tmem_ld8(trow + 8 * (2 * h + 2), d[nxt][0]);
      tmem_ld8(trow + 8 * (2 * h + 3), d[nxt][1]);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      pin8(d[cur][u]);
      const int j = j0 + 2 * h + u;
      if (!CHECK || j < nd) {
        const TcDest P = dconst[j];
        out[dofs[j]] = tc_fold(d[cur][u], P.q, __longlong_as_double((long long)P.qinv));
      }
    }
    if (h + 1 < NDC / 2) tmem_wait_ld();
  }
}

__global__ void __launch_bounds__(TC_M, 7)
    conv_tc_kernel(const __grid_constant__ ConvJobList L, const DevPrime* primes, int logN, uint32_t* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const ConvJob& J = L.j[blockIdx.y];
  const ConvTable& T = J.t;
  const int ns = T.n_src, nd = T.n_dst, kpad = T.tc_kpad, ndp = T.tc_nd_pad;
  const TcLayout Ly = tc_layout(kpad, ndp);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int N = 1 << logN;
  const int coef = blockIdx.x * TC_M + tid;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + 8);
  TcDest* dconst = reinterpret_cast<TcDest*>(sm + Ly.o_dst);
  int* dofs = reinterpret_cast<int*>(sm + Ly.o_pos);
  uint8_t* sA = sm + Ly.o_a;
  uint8_t* sB = sm + Ly.o_b;
  const uint32_t bar_a = smem_addr(bar);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(TC_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {  // B image: 16-byte cp.async copies (kpad 8 ndp bytes, a multiple of 256), waited for below
    const int n16 = kpad * ndp / 2;
    for (int k = tid; k < n16; k += TC_M) tc_cp_async16(sB + 16 * k, T.tc_b + 16 * k);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int j = tid; j < ndp; j += TC_M) {  // destination constants
    dconst[j] = T.tc_dst[j];
    dofs[j] = j < nd ? T.dst_pos[j] << logN : 0;
  }
  {  // A: the bytes of the pre-scaled residues of this thread's coefficient
    uint64_t x[TC_MAX_SRC];
#pragma unroll
    for (int i = 0; i < TC_MAX_SRC; ++i)
      if (i < ns) x[i] = J.src[(size_t)T.src_pos[i] * N + coef];
    uint64_t lifted = 0;  // reduced-noise lift: the count is source row ns of the product
#pragma unroll
    for (int i = 0; i < TC_MAX_SRC; ++i)
      if (i < ns) {
        const ShoupConst pc = T.pre[i];
        const uint64_t q = primes[T.src_prime[i]].q;
        x[i] = shoup(x[i], pc.w, pc.ws, q);
        lifted += x[i] > (q >> 1);
      }
    if (!T.lift) lifted = 0;
#pragma unroll
    for (int p = 0; p < TC_MAX_SRC / 2; ++p) {
      if (p >= kpad / 16) break;
      const uint64_t lo = 2 * p < ns ? x[2 * p] : (2 * p == ns ? lifted : 0),
                     hi = 2 * p + 1 < ns ? x[2 * p + 1] : (2 * p + 1 == ns ? lifted : 0);
      *reinterpret_cast<ulonglong2*>(sA + p * (TC_M * 16) + tid * 16) = make_ulonglong2(lo, hi);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's part of the B image
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // A and B, visible to the MMAs
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  bool ok = true;
  int failed_chunk = -1;
  const uint32_t tbase = *slot;
  const uint32_t a0 = smem_addr(sA), b0 = smem_addr(sB);
  const uint32_t trow = tbase + ((uint32_t)(warp * 32) << 16);
  const int nchunks = (ndp + TC_DCHUNK - 1) / TC_DCHUNK;
  uint64_t* out = J.dst + coef;
  for (int c = 0; ok && c < nchunks; ++c) {
    const int ndc = min(TC_DCHUNK, ndp - c * TC_DCHUNK);  // even: N = 8 ndc is a multiple of 16
    if (tid == 0) {
      const uint32_t idesc = idesc_u8(8 * ndc);
      for (int kc = 0; kc < kpad / 32; ++kc) {
        const uint64_t da = smem_desc(a0 + kc * 2 * (TC_M * 16), TC_M * 16, 128);
        const uint64_t db = smem_desc(b0 + (kc * 2 * (8 * ndp) + c * TC_DCHUNK * 8) * 16, 8 * ndp * 16, 128);
        mma_u8(tbase, da, db, idesc, kc > 0);
      }
      mma_commit(bar_a);
    }
    ok = __syncthreads_and(bar_wait_bounded(bar_a, c & 1));
    if (!ok) {
      failed_chunk = c;
      break;
    }
    tc_fence_after();
    const int j0 = c * TC_DCHUNK;
    if (ndc == TC_DCHUNK && j0 + TC_DCHUNK <= nd)
      tc_epilogue<TC_DCHUNK, false>(trow, j0, nd, dconst, dofs, out);
    else if (ndc == 2)
      tc_epilogue<2, true>(trow, j0, nd, dconst, dofs, out);
    else if (ndc == 4)
      tc_epilogue<4, true>(trow, j0, nd, dconst, dofs, out);
    else if (ndc == 6)
      tc_epilogue<6, true>(trow, j0, nd, dconst, dofs, out);
    else
      tc_epilogue<8, true>(trow, j0, nd, dconst, dofs, out);
    tc_fence_before();
    __syncthreads();  // TMEM columns are free for the next chunk
    tc_fence_after();
  }
  if (!ok) {
    // The commit of chunk failed_chunk has not arrived: its MMAs may still own the TMEM
    // columns.  tcgen05.commit arrives on the mbarrier only after every MMA this thread issued
    // before it has completed, so a second bounded wait on the same phase either sees them
    // finish (the dealloc below is then safe) or gives up after about another second, when
    // the tensor pipe is not progressing at all; the columns are freed in either case so the
    // CTA can exit, and the status word marks every output of the launch as incomplete (the
    // host's next synchronising call returns FIDES_ERR_TIMEOUT until it is cleared).
    if (tid == 0) {
      atomicOr(status, 1u);
      bar_wait_bounded(bar_a, failed_chunk & 1);
    }
    __syncthreads();
  }
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(TC_COLS) : "memory");
  }
}

}  // namespace

void launch_conv_tc(Context* c, const ConvJob* jobs, int n, cudaStream_t s) {
  static thread_local ConvJobList L;
  static bool attr = false;
  if (!attr) {
    FIDES_CUDA(cudaFuncSetAttribute(conv_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    attr = true;
  }
  for (int off = 0; off < n; off += MAX_CONV_JOBS) {
    const int m = std::min(MAX_CONV_JOBS, n - off);
    L.n = m;
    std::copy(jobs + off, jobs + off + m, L.j);
    int smem = TC_SMEM_FLOOR;
    double bytes = 0;
    for (int i = 0; i < m; ++i) {
      const ConvTable& t = L.j[i].t;
      if (!t.tc_b) throw Error(-1, "basis conversion has no tensor-core form");
      smem = std::max(smem, tc_layout(t.tc_kpad, t.tc_nd_pad).total + FIDES_TC_SMEM_GUARD);
      bytes += 8.0 * c->N * (t.n_src + t.n_dst);
    }
    dim3 grid(c->N / TC_M, m);
    LaunchScope ls(c, s, KK_CONV, bytes);
    conv_tc_kernel<<<grid, TC_M, smem, s>>>(L, c->d_prime, c->logN, c->d_status);
    FIDES_CUDA(cudaGetLastError());
  }
}

}  // namespace fides
