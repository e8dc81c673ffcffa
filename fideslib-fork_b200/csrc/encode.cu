// CKKS slot encode / decode on the device (the reference's device encode,
// src/CKKS/DeviceEncodeBatch.cu: ifft_stage_ / ifft_stages_smem_ / ifft_finish_ at :444-527,
// fit_to_native_batch_ at :143, the batched encode NTT at :191).
//
// Encode: n complex slots (n a power of two, n <= N/2) -> the inverse special FFT
//   w = (1/n) V^H z,  V[j][k] = zeta^(5^j k),  zeta = exp(i pi / N),
// the coefficients m_(gap k) = round(Re w_k * scale), m_(gap (k + n)) = round(Im w_k * scale)
// (gap = N / 2n, zero elsewhere), then every requested limb in EVALUATION form.  The FFT is
// the radix-2 Gentleman-Sande network whose stage `len` multiplies the difference at position
// j < len/2 by exp(-2 pi i 5^j / 4len), followed by a bit reversal (the published special FFT
// of the HEAAN / OpenFHE encoders).  Here it runs as two FP64 passes over shared memory:
//   * a strided pass: the stages len = n .. 2S on sub-problems of P = n / S elements at
//     stride S (a CTA holds several sub-problems with consecutive offsets, so every global
//     access is a run of consecutive elements);
//   * a contiguous pass: the stages len = S .. 2 on blocks of S consecutive elements, then the
//     bit reversal, scaling and rounding, writing the coefficients as signed 64-bit integers.
//     A CTA takes the blocks whose bit-reversed indices are consecutive, so the scattered output
//     of the bit reversal becomes runs of consecutive coefficients.
// The signed coefficients feed the library's forward NTT with the signed-integer prologue (each
// limb reduces them modulo its own prime), so all limbs of a batch of plaintexts are one NTT
// launch pair and a coefficient may exceed any single prime (plaintext diagonals at scales
// close to q_0, e.g. with 59-bit scaling primes and a 60-bit q_0).  |m| must stay below 2^62;
// a larger coefficient sets bit 1 of the context's device status word and is written as 0.
//
// Decode is the transpose: INTT of limb 0, centred lift and 1/scale while loading in
// bit-reversed order, the Cooley-Tukey stages len = 2 .. S, then len = 2S .. n, giving the
// slots in natural order.  It reads limb 0 only, so it needs |m| < q_0 / 2 (true for a
// decrypted message at a scale well below q_0).
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "context.hpp"
#include "encode.hpp"
#include "modarith.cuh"
#include "ntt.cuh"

namespace fides {
namespace {

constexpr int SF_THREADS = 256;
constexpr int SF_TILE = 2048;  // double2 elements per CTA (32 KB of shared memory)
constexpr int SF_LOGS = 7;     // contiguous blocks of S = 2^7 elements (fewer when n is smaller)

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ int brev(int x, int bits) { return bits ? (int)(__brev((unsigned)x) >> (32 - bits)) : 0; }

// One butterfly stage on shared memory: the pair (lo, hi) = (lo, lo + h) of a stage of length
// 2h, twiddle tw[h + j] (j = the lower element's position within its length-2h block).
template <bool DIT>
__device__ __forceinline__ void butterfly(double2* sh, int lo, int hi, double2 w) {
  const double2 a = sh[lo], b = sh[hi];
  if (!DIT) {
    sh[lo] = cadd(a, b);
    sh[hi] = cmul(csub(a, b), w);
  } else {
    const double2 t = cmulc(b, w);
    sh[lo] = cadd(a, t);
    sh[hi] = csub(a, t);
  }
}

// Strided pass over `lp` stages: sub-problem r holds elements r + s S, s < P = 2^lp.
// DIF (encode): stages len = n, n/2, ..., 2S.  DIT (decode): len = 2S, ..., n.
// grid = (S / G, polys), G = min(SF_TILE / P, S) sub-problems per CTA; sh[s G + g].
template <bool DIT>
__global__ void __launch_bounds__(SF_THREADS) sfft_strided(const double2* __restrict__ in, double2* __restrict__ out,
                                                           const double2* __restrict__ tw, int logn, int lp) {
  __shared__ double2 sh[SF_TILE];
  const int n = 1 << logn, P = 1 << lp, S = n >> lp;
  const int G = min(SF_TILE / P, S);
  const int r0 = blockIdx.x * G;
  const double2* src = in + (size_t)blockIdx.y * n;
  double2* dst = out + (size_t)blockIdx.y * n;
  for (int e = threadIdx.x; e < G * P; e += blockDim.x) {
    const int g = e % G, s = e / G;
    sh[e] = src[r0 + g + s * S];
  }
  __syncthreads();
  for (int t = 0; t < lp; ++t) {
    const int len = DIT ? (2 * S) << t : n >> t;
    const int h = len >> 1, hs = h / S;
    for (int b = threadIdx.x; b < G * P / 2; b += blockDim.x) {
      const int g = b % G, u = b / G;
      const int blk = u / hs, off = u - blk * hs;
      const int slo = 2 * blk * hs + off;
      const int x = r0 + g + slo * S;  // global index of the lower element; x mod len < h
      butterfly<DIT>(sh, slo * G + g, (slo + hs) * G + g, tw[h + (x & (len - 1))]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < G * P; e += blockDim.x) {
    const int g = e % G, s = e / G;
    dst[r0 + g + s * S] = sh[e];
  }
}

// Contiguous encode pass: blocks b = brev_la(c0 + u), u < G (la = logn - ls), each of S = 2^ls
// elements; DIF stages len = S .. 2, then coefficient k = brev_logn(b S + r) = brev_ls(r) 2^la
// + c0 + u takes Re / Im of the element times scale / n, rounded to nearest, as a signed 64-bit
// integer (each limb's NTT prologue reduces it modulo its own prime).
__global__ void __launch_bounds__(SF_THREADS) sfft_encode_finish(const double2* __restrict__ in, uint64_t* __restrict__ coef,
                                                                 const double2* __restrict__ tw, int logn, int ls,
                                                                 int logN, double mult, uint64_t q0,
                                                                 uint32_t* __restrict__ status) {
  __shared__ double2 sh[SF_TILE];
  const int n = 1 << logn, S = 1 << ls, la = logn - ls;
  const int G = min(SF_TILE / S, n / S);
  const int c0 = blockIdx.x * G;
  const double2* src = in + (size_t)blockIdx.y * n;
  for (int e = threadIdx.x; e < G * S; e += blockDim.x) {
    const int u = e / S, r = e % S;
    sh[e] = src[(size_t)brev(c0 + u, la) * S + r];
  }
  __syncthreads();
  for (int len = S; len >= 2; len >>= 1) {
    const int h = len >> 1;
    for (int b = threadIdx.x; b < G * S / 2; b += blockDim.x) {
      const int u = b / (S / 2), v = b % (S / 2);
      const int blk = v / h, j = v - blk * h;
      const int lo = u * S + blk * len + j;
      butterfly<false>(sh, lo, lo + h, tw[h + j]);
    }
    __syncthreads();
  }
  const int gap = 1 << (logN - 1 - logn);
  uint64_t* out = coef + ((size_t)blockIdx.y << logN);
  (void)q0;
  const double lim = 4611686018427387904.0;  // 2^62
  bool bad = false;
  for (int e = threadIdx.x; e < G * S; e += blockDim.x) {
    const int u = e % G, rr = e / G;
    const int k = (rr << la) + c0 + u;
    const double2 w = sh[u * S + brev(rr, ls)];
    const double re = w.x * mult, im = w.y * mult;
    uint64_t mr = 0, mi = 0;
    if (fabs(re) < lim && fabs(im) < lim) {
      mr = (uint64_t)__double2ll_rn(re);
      mi = (uint64_t)__double2ll_rn(im);
    } else {
      bad = true;
    }
    out[(size_t)gap * k] = mr;
    out[(size_t)gap * (k + n)] = mi;
  }
  if (bad) atomicOr(status, 2u);
}

// Contiguous decode pass: loads element x = b S + r of the bit-reversed array, i.e. w_k with
// k = brev_ls(r) 2^la + c0 + u, from the centred coefficients (m_(gap k) + i m_(gap (k+n))) / scale,
// runs the DIT stages len = 2 .. S and stores the blocks contiguously.
__global__ void __launch_bounds__(SF_THREADS) sfft_decode_start(const uint64_t* __restrict__ coef, double2* __restrict__ out,
                                                                const double2* __restrict__ tw, int logn, int ls,
                                                                int logN, double inv_scale, uint64_t q0) {
  __shared__ double2 sh[SF_TILE];
  const int n = 1 << logn, S = 1 << ls, la = logn - ls;
  const int G = min(SF_TILE / S, n / S);
  const int c0 = blockIdx.x * G;
  const int gap = 1 << (logN - 1 - logn);
  const uint64_t* in = coef + ((size_t)blockIdx.y << logN);
  const uint64_t half = q0 >> 1;
  auto centred = [&](uint64_t v) -> double { return v > half ? -(double)(q0 - v) : (double)v; };
  for (int e = threadIdx.x; e < G * S; e += blockDim.x) {
    const int u = e % G, rr = e / G;
    const int k = (rr << la) + c0 + u;
    sh[u * S + brev(rr, ls)] = make_double2(centred(in[(size_t)gap * k]) * inv_scale,
                                            centred(in[(size_t)gap * (k + n)]) * inv_scale);
  }
  __syncthreads();
  for (int len = 2; len <= S; len <<= 1) {
    const int h = len >> 1;
    for (int b = threadIdx.x; b < G * S / 2; b += blockDim.x) {
      const int u = b / (S / 2), v = b % (S / 2);
      const int blk = v / h, j = v - blk * h;
      const int lo = u * S + blk * len + j;
      butterfly<true>(sh, lo, lo + h, tw[h + j]);
    }
    __syncthreads();
  }
  double2* dst = out + (size_t)blockIdx.y * n;
  for (int e = threadIdx.x; e < G * S; e += blockDim.x) {
    const int u = e / S, r = e % S;
    dst[(size_t)brev(c0 + u, la) * S + r] = sh[e];
  }
}

int log2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

void check_slots(Context* c, int n_slots) {
  if (n_slots < 1 || n_slots > c->N / 2 || (n_slots & (n_slots - 1)))
    throw Error(-1, "slots must be a power of two <= N/2");
}

}  // namespace

void op_encode(Context* c, const double* slots, int n_slots, int n_pts, double scale, int level, uint64_t* out,
               cudaStream_t s) {
  op_encode_ext(c, slots, n_slots, n_pts, scale, level, 0, out, s);
}

void op_encode_ext(Context* c, const double* slots, int n_slots, int n_pts, double scale, int level, int special,
                   uint64_t* out, cudaStream_t s) {
  if (special < 0 || special > c->K) throw Error(-1, "special limbs out of range");
  check_slots(c, n_slots);
  if (n_pts < 1) throw Error(-1, "n_pts < 1");
  if (level < 1 || level > c->n_q) throw Error(-4, "level out of range");
  if (!(scale > 0)) throw Error(-1, "scale must be positive");
  const int logn = log2i(n_slots), ls = logn < SF_LOGS ? logn : SF_LOGS, lp = logn - ls;
  const size_t N = c->N, n = n_slots;
  Scratch sc(c, n_pts * (N * sizeof(uint64_t) + (lp ? n * sizeof(double2) : 0)), s);
  uint64_t* coef = sc.u64();
  double2* work = reinterpret_cast<double2*>(coef + n_pts * N);
  const double2* tw = static_cast<const double2*>(c->d_sfft);
  const double2* z = reinterpret_cast<const double2*>(slots);
  if (2 * n < N) FIDES_CUDA(cudaMemsetAsync(coef, 0, n_pts * N * sizeof(uint64_t), s));
  const double2* fin = z;
  if (lp) {
    const int P = 1 << lp, S = 1 << ls, G = (SF_TILE / P) < S ? SF_TILE / P : S;
    LaunchScope l1(c, s, KK_ELEM, 2.0 * n_pts * n * sizeof(double2));
    sfft_strided<false><<<dim3(S / G, n_pts), SF_THREADS, 0, s>>>(z, work, tw, logn, lp);
    FIDES_CUDA(cudaGetLastError());
    fin = work;
  }
  {
    const int S = 1 << ls, nb = (int)(n >> ls), G = (SF_TILE / S) < nb ? SF_TILE / S : nb;
    LaunchScope l2(c, s, KK_ELEM, n_pts * (n * sizeof(double2) + 2.0 * n * sizeof(uint64_t)));
    sfft_encode_finish<<<dim3(nb / G, n_pts), SF_THREADS, 0, s>>>(fin, coef, tw, logn, ls, c->logN,
                                                                  scale / (double)n, c->primes[0], c->d_status);
    FIDES_CUDA(cudaGetLastError());
  }
  std::vector<LimbRef> refs;
  const int limbs = level + special;
  refs.reserve((size_t)n_pts * limbs);
  for (int p = 0; p < n_pts; ++p)
    for (int j = 0; j < limbs; ++j) {
      LimbRef r = lref(out + ((size_t)p * limbs + j) * N, j < level ? j : c->n_q + (j - level));
      r.pro = coef + p * N;  // signed coefficients, reduced by each limb's prologue
      refs.push_back(r);
    }
  ntt_limbs(c, refs.data(), (int)refs.size(), false, s, IN_SIGNED, OUT_PLAIN);
}

void op_decode(Context* c, const uint64_t* pts, int level, int n_pts, int n_slots, double scale, double* slots,
               cudaStream_t s) {
  check_slots(c, n_slots);
  if (n_pts < 1) throw Error(-1, "n_pts < 1");
  if (level < 1 || level > c->n_q) throw Error(-4, "level out of range");
  if (!(scale > 0)) throw Error(-1, "scale must be positive");
  const int logn = log2i(n_slots), ls = logn < SF_LOGS ? logn : SF_LOGS, lp = logn - ls;
  const size_t N = c->N, n = n_slots;
  Scratch sc(c, n_pts * (N * sizeof(uint64_t) + (lp ? n * sizeof(double2) : 0)), s);
  uint64_t* coef = sc.u64();
  double2* work = reinterpret_cast<double2*>(coef + n_pts * N);
  const double2* tw = static_cast<const double2*>(c->d_sfft);
  double2* z = reinterpret_cast<double2*>(slots);
  std::vector<LimbRef> refs;
  for (int p = 0; p < n_pts; ++p) {
    LimbRef r = lref(coef + p * N, 0);
    r.src = pts + (size_t)p * level * N;
    refs.push_back(r);
  }
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  {
    const int S = 1 << ls, nb = (int)(n >> ls), G = (SF_TILE / S) < nb ? SF_TILE / S : nb;
    LaunchScope l1(c, s, KK_ELEM, n_pts * (2.0 * n * sizeof(uint64_t) + n * sizeof(double2)));
    sfft_decode_start<<<dim3(nb / G, n_pts), SF_THREADS, 0, s>>>(coef, lp ? work : z, tw, logn, ls, c->logN,
                                                                 1.0 / scale, c->primes[0]);
    FIDES_CUDA(cudaGetLastError());
  }
  if (lp) {
    const int P = 1 << lp, S = 1 << ls, G = (SF_TILE / P) < S ? SF_TILE / P : S;
    LaunchScope l2(c, s, KK_ELEM, 2.0 * n_pts * n * sizeof(double2));
    sfft_strided<true><<<dim3(S / G, n_pts), SF_THREADS, 0, s>>>(work, z, tw, logn, lp);
    FIDES_CUDA(cudaGetLastError());
  }
}

}  // namespace fides
