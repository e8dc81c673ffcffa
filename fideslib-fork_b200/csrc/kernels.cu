// Elementwise RNS kernels, basis conversion and KSK inner product.
#include <algorithm>

#include "kernels.cuh"

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

__global__ void __launch_bounds__(EW_THREADS) conv_kernel(const __grid_constant__ ConvJobList L, const DevPrime* primes,
                                                          int logN) {
  const ConvJob& J = L.j[blockIdx.y];
  const ConvTable& T = J.t;
  extern __shared__ uint64_t sm[];
  const int ns = T.n_src, nd = T.n_dst;
  ShoupConst* pre = reinterpret_cast<ShoupConst*>(sm);  // [n_src], 16-byte aligned
  uint64_t* mat = sm + 2 * ns;                          // [n_src][n_dst]
  for (int i = threadIdx.x; i < ns * nd; i += blockDim.x) mat[i] = T.mat[i];
  for (int i = threadIdx.x; i < ns; i += blockDim.x) pre[i] = T.pre[i];
  __syncthreads();
  const int N = 1 << logN;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  uint64_t y[MAX_SRC];
#pragma unroll 4
  for (int i = 0; i < ns; ++i) {
    const DevPrime& p = primes[T.src_prime[i]];
    uint64_t v = J.src[(size_t)T.src_pos[i] * N + n];
    y[i] = shoup(v, pre[i].w, pre[i].ws, p.q);
  }
  for (int j = 0; j < nd; ++j) {
    const DevPrime p = primes[T.dst_prime[j]];
    U128 acc{0, 0};
    int i = 0;
    while (i < ns) {
      const int e = min(ns, i + 8);
      for (; i < e; ++i) mac128(acc, y[i], mat[i * nd + j]);
      if (i < ns) acc = U128{reduce128(acc, p), 0};  // keep the sum below 2^128
    }
    J.dst[(size_t)T.dst_pos[j] * N + n] = reduce128(acc, p);
  }
}

__global__ void __launch_bounds__(EW_THREADS) ksk_kernel(const __grid_constant__ KskJobList L, const DevPrime* primes,
                                                         const ShoupConst* pmod, int logN, int n_q, int K, int dnum,
                                                         int alpha) {
  const KskJob& J = L.j[blockIdx.z];
  const int l = J.l, ext = l + K;
  const int i = blockIdx.y;
  if (i >= ext) return;
  const int N = 1 << logN;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const int pid = i < l ? i : n_q + (i - l);
  const DevPrime p = primes[pid];
  const int beta = (l + alpha - 1) / alpha;
  const int own = i < l ? i / alpha : -1;
  const size_t kstride = (size_t)(n_q + K) * N;
  U128 sa{0, 0}, sb{0, 0};
  for (int d = 0; d < beta; ++d) {
    uint64_t v = (d == own && J.x) ? J.x[(size_t)i * N + n] : J.digits[((size_t)d * ext + i) * N + n];
    uint64_t ka = J.key[(size_t)d * kstride + (size_t)pid * N + n];
    uint64_t kb = J.key[(size_t)(dnum + d) * kstride + (size_t)pid * N + n];
    mac128(sa, v, ka);
    mac128(sb, v, kb);
  }
  uint64_t ra = reduce128(sa, p), rb = reduce128(sb, p);
  if (J.c0 && i < l) {
    const ShoupConst pm = pmod[i];
    rb = addmod(rb, shoup(J.c0[(size_t)i * N + n], pm.w, pm.ws, p.q), p.q);
  }
  const uint32_t o = J.auto_k ? auto_slot(logN, J.auto_k, (uint32_t)n) : (uint32_t)n;
  J.out_a[(size_t)i * N + o] = ra;
  J.out_b[(size_t)i * N + o] = rb;
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
  J.d2[off] = mulmod(x1, y1, p);
}

// OpenFHE SwitchModulus as restated in the reference (src/CKKS/Rescale.cuh:44-64).
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

template <typename List, typename Job>
int fill(List& L, const Job* jobs, int n) {
  L.n = n;
  std::copy(jobs, jobs + n, L.j);
  return n;
}

}  // namespace

void launch_conv(Context* c, const ConvJob* jobs, int n, cudaStream_t s) {
  static thread_local ConvJobList L;
  for (int off = 0; off < n; off += MAX_CONV_JOBS) {
    int m = std::min(MAX_CONV_JOBS, n - off);
    fill(L, jobs + off, m);
    size_t smem = 0;
    for (int i = 0; i < m; ++i) {
      const ConvTable& t = L.j[i].t;
      if (t.n_src > MAX_SRC || t.n_dst > MAX_DST) throw Error(-1, "basis conversion too wide");
      smem = std::max(smem, (size_t)t.n_src * t.n_dst * 8 + (size_t)t.n_src * 16);
    }
    static bool attr = false;
    if (!attr) {
      FIDES_CUDA(cudaFuncSetAttribute(conv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
      attr = true;
    }
    dim3 grid(c->N / EW_THREADS, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * (L.j[i].t.n_src + L.j[i].t.n_dst);
    LaunchScope ls(c, s, KK_CONV, bytes);
    conv_kernel<<<grid, EW_THREADS, smem, s>>>(L, c->d_prime, c->logN);
    FIDES_CUDA(cudaGetLastError());
  }
}

void launch_ksk(Context* c, const KskJob* jobs, int n, cudaStream_t s) {
  static thread_local KskJobList L;
  for (int off = 0; off < n; off += MAX_KSK_JOBS) {
    int m = std::min(MAX_KSK_JOBS, n - off);
    fill(L, jobs + off, m);
    int mx = 0;
    for (int i = 0; i < m; ++i) mx = std::max(mx, L.j[i].l + c->K);
    dim3 grid(c->N / EW_THREADS, mx, m);
    double bytes = 0;
    for (int i = 0; i < m; ++i) {
      const int l = L.j[i].l, ext = l + c->K, b = c->beta(l);
      bytes += 8.0 * c->N * ((double)ext * (3 * b + 2) + (L.j[i].c0 ? l : 0));
    }
    LaunchScope ls(c, s, KK_KSK, bytes);
    ksk_kernel<<<grid, EW_THREADS, 0, s>>>(L, c->d_prime, c->d_pmod, c->logN, c->n_q, c->K, c->dnum, c->alpha);
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
    for (int i = 0; i < m; ++i) bytes += 8.0 * c->N * (7.0 * L.j[i].l);
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

}  // namespace fides
