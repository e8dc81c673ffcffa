// Measurement harness for the reference's own GPU NTT kernels (measurement only; nothing in
// the product uses it).  It compiles the reference's src/NTT.cu where it lies (the build
// recipe adds the reference's src/ to the include path and this file includes NTT.cu), fills
// the two structures those kernels read -- the __constant__ FIDESlib::Constants block and
// the device-resident Global::Globals tables -- for a given prime chain and root of unity,
// and launches the kernels with the reference's own geometry:
//   * forward: NTTBatch_<false / true, ALGO_SHOUP> (src/NTT.cu:775-800), one launch per pass
//     over polys x limbs, as RNSPoly::NTT batches them;
//   * inverse: INTT_<false / true, ALGO_SHOUP, INTT_NONE> over pointer tables, per
//     polynomial, with LimbPartition::ApplyINTT's block sizes (src/CKKS/LimbPartition.cu:526-550).
// The table contents follow the reference's SetupConstants (src/ConstantsGPU.cu:132-330),
// restated here because that file needs OpenFHE headers: natural-order powers of the root
// (2N of them), their bit-reversed first N, the middle-scale tables, the inverse tables scaled
// by N^-1, Shoup companions floor(w 2^64 / q), Barrett mu = floor(2^(2 bits + 1) / q).
// It also drives the reference's basis conversions with their geometry (block 64 x 2, one
// coefficient column per thread, LimbPartitionMGPU.cu:1296-1303 and :1642-1651):
//   * DecompAndModUpConv<ALGO_SHOUP> (src/CKKS/Conv.cu:274-423) for one digit at one level;
//   * ModDown2<ALGO_SHOUP> (src/CKKS/Conv.cu:27-133), special limbs -> Q limbs;
// with the digit metadata of the __constant__ block (contiguous digits of alpha = ceil(L /
// dnum) primes) and the Q-hat tables in the reference's index layouts (MODUPIDX_SCALE,
// MODUPIDX_MATRIX, MODDOWN_MATRIX), computed here from the primes.
// Outputs are bit-identical to this project's transforms and conversions for the same primes
// and root (tests/test_ref_kernels.py), which is how the harness is validated before timing.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "NTT.cu"
#include "CKKS/Conv.cu"

// The reference declares the block `extern __constant__` (src/ConstantsGPU.cuh:200) and
// defines it in ConstantsGPU.cu, which cannot be built here; with relocatable device code
// (-rdc=true) this is the definition.
namespace FIDESlib {
__constant__ Constants constants;
}

namespace {

using FIDESlib::Constants;
using FIDESlib::Global;
using FIDESlib::MAXP;

uint64_t mulmod_h(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((unsigned __int128)a * b % q); }
uint64_t powmod_h(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  for (; e; e >>= 1, a = mulmod_h(a, a, q))
    if (e & 1) r = mulmod_h(r, a, q);
  return r;
}
uint64_t inv_h(uint64_t a, uint64_t q) { return powmod_h(a, q - 2, q); }
uint64_t shoup_h(uint64_t w, uint64_t q) { return (uint64_t)(((unsigned __int128)w << 64) / q); }
uint32_t brev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}
int bitw(uint64_t x) { return 64 - __builtin_clzll(x); }
// the reference's table index layouts (src/ConstantsGPU.cuh: MODUPIDX_SCALE, MODUPIDX_MATRIX)
#define FIDESlib_MODUPIDX_SCALE(i, j, k) ((size_t)MAXP * MAXP * (i) + (size_t)MAXP * (j) + (k))
#define FIDESlib_MODUPIDX_MATRIX(n, i, j) ((size_t)MAXP * MAXP * (n) + (size_t)MAXP * (i) + (j))

struct State {
  int logN = 0, N = 0, np = 0, nq = 0, K = 0, dnum = 1, alpha = 1;
  std::vector<std::vector<int>> to;  // per digit: destination prime ids (primeid_digit_to order)
  Global::Globals* d_globals = nullptr;
  std::vector<void*> d_tables;
  void** d_ptrs = nullptr;  // pointer tables (data, aux)
  size_t ptr_cap = 0;
} S;

void release() {
  for (void* p : S.d_tables) cudaFree(p);
  S.d_tables.clear();
  if (S.d_globals) cudaFree(S.d_globals);
  if (S.d_ptrs) cudaFree(S.d_ptrs);
  S = State{};
}

template <typename F>
int run(F&& f) {
  cudaError_t e = f();
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? 0 : -(int)e;
}

}  // namespace

extern "C" {

// Builds the constants and tables for n_q Q primes followed by K special primes
// (primes[0..n_q+K), 2N-th roots psi[...]) at ring degree 2^logN, digits of dnum.
int ref_kernels_init(int logN, int n_q, int K, int dnum, const uint64_t* primes, const uint64_t* psi) {
  release();
  const int np = n_q + K;
  if (n_q < 1 || K < 0 || np > MAXP || dnum < 1 || dnum > FIDESlib::MAXD || dnum > n_q || logN < 10 || logN > 17)
    return -1;
  const int N = 1 << logN;
  S.logN = logN;
  S.N = N;
  S.np = np;
  S.nq = n_q;
  S.K = K;
  S.dnum = dnum;
  S.alpha = (n_q + dnum - 1) / dnum;
  Constants hc;
  std::memset(&hc, 0, sizeof(hc));
  hc.N = N;
  hc.logN = logN;
  hc.L = n_q;
  hc.K = K;
  hc.type = np >= 64 ? ~0ull : ((1ull << np) - 1);  // every limb holds 64-bit words
  hc.dnum = dnum;
  hc.reduced_noise = false;
  // the Globals block holds MAXP^3-word tables: keep it off the stack
  std::unique_ptr<Global::Globals> hgp(new Global::Globals);
  Global::Globals& hg = *hgp;
  std::memset(&hg, 0, sizeof(hg));
  const int alpha = S.alpha;
  auto mulm = [&](uint64_t a, uint64_t b, uint64_t q) { return mulmod_h(a % q, b % q, q); };
  // digit metadata: digit d = primes [d alpha, min((d + 1) alpha, n_q))
  S.to.assign(dnum, {});
  for (int d = 0; d < dnum; ++d) {
    const int lo = d * alpha, hi = std::min(n_q, (d + 1) * alpha);
    for (int i = lo; i < hi; ++i) {
      hc.primeid_digit_from[d][i - lo] = i;
      hc.primeid_digit[i] = d;
      hc.pos_in_digit[d][i] = i - lo;
    }
    for (int i = 0; i < n_q; ++i)
      if (i < lo || i >= hi) S.to[d].push_back(i);
    for (int k = 0; k < K; ++k) S.to[d].push_back(n_q + k);
    for (int j = 0; j < (int)S.to[d].size(); ++j) hc.primeid_digit_to[d][j] = S.to[d][j];
    for (int n = 1; n <= n_q; ++n) {
      hc.num_primeid_digit_from[d][n - 1] = std::max(0, std::min(hi, n) - lo);
      hc.num_primeid_digit_to[d][n - 1] = (int)S.to[d].size();
    }
    // pre-scale for every partial size c of the digit: (prod of the other c - 1 primes)^-1
    for (int c = 1; c <= hi - lo; ++c)
      for (int i = lo; i < lo + c; ++i) {
        uint64_t v = 1;
        for (int k = lo; k < lo + c; ++k)
          if (k != i) v = mulm(v, primes[k], primes[i]);
        const size_t at = FIDESlib_MODUPIDX_SCALE(d, c - 1, i);
        hg.DecompAndModUp_pre_scale[at] = inv_h(v, primes[i]);
        hg.DecompAndModUp_pre_scale_shoup[at] = shoup_h(hg.DecompAndModUp_pre_scale[at], primes[i]);
      }
  }
  // ModUp matrix at every level n: (prod of the other active primes of i's digit) mod p_j
  for (int n = 1; n <= n_q; ++n)
    for (int i = 0; i < n; ++i) {
      const int d = i / alpha, lo = d * alpha, hi = std::min(n, (d + 1) * alpha);
      for (int j = 0; j < np; ++j) {
        if (j >= lo && j < hi) continue;
        uint64_t v = 1 % primes[j];
        for (int k = lo; k < hi; ++k)
          if (k != i) v = mulm(v, primes[k], primes[j]);
        const size_t at = FIDESlib_MODUPIDX_MATRIX(n - 1, i, j);
        hg.DecompAndModUp_matrix[at] = v;
        hg.DecompAndModUp_matrix_shoup[at] = shoup_h(v, primes[j]);
      }
    }
  // ModDown: P-hat_k^-1 mod p_k and P-hat_k mod q_j
  for (int k = 0; k < K; ++k) {
    const uint64_t pk = primes[n_q + k];
    uint64_t v = 1;
    for (int t = 0; t < K; ++t)
      if (t != k) v = mulm(v, primes[n_q + t], pk);
    hg.ModDown_pre_scale[n_q + k] = inv_h(v, pk);
    hg.ModDown_pre_scale_shoup[n_q + k] = shoup_h(hg.ModDown_pre_scale[n_q + k], pk);
    for (int j = 0; j < n_q; ++j) {
      uint64_t w = 1 % primes[j];
      for (int t = 0; t < K; ++t)
        if (t != k) w = mulm(w, primes[n_q + t], primes[j]);
      hg.ModDown_matrix[(size_t)MAXP * k + j] = w;
      hg.ModDown_matrix_shoup[(size_t)MAXP * k + j] = shoup_h(w, primes[j]);
    }
  }
  for (int j = 0; j < n_q; ++j) {
    uint64_t P = 1 % primes[j];
    for (int t = 0; t < K; ++t) P = mulm(P, primes[n_q + t], primes[j]);
    hc.P[j] = P;
  }
  const int aw = (logN + 1) / 2;
  for (int i = 0; i < np; ++i) {
    const uint64_t q = primes[i], root = psi[i] % q, iroot = inv_h(root, q), ninv = inv_h((uint64_t)N % q, q);
    hc.primes[i] = q;
    hc.prime_bits[i] = (uint32_t)bitw(q);
    hc.prime_better_barret_mu[i] = (uint64_t)(((unsigned __int128)1 << (2 * bitw(q) + 1)) / q);
    hc.N_inv[i] = ninv;
    hc.N_inv_shoup[i] = shoup_h(ninv, q);
    hc.N_shoup[i] = shoup_h((uint64_t)N % q, q);
    hc.one_shoup[i] = shoup_h(1, q);
    hc.root[i] = root;
    hc.root_shoup[i] = shoup_h(root, q);
    hc.inv_root[i] = iroot;
    hc.inv_root_shoup[i] = shoup_h(iroot, q);
    if (i < n_q) hc.primeid_partition[0][i] = i;  // PARTITION(0, j): limb j uses prime j
    if (i >= n_q) hc.primeid_special_partition[i - n_q] = i;
    std::vector<uint64_t> pno(2 * N), ipno(2 * N), ps(N), ips(N), pms(N), ipms(N), psh(N), ipsh(N);
    pno[0] = ipno[0] = 1;
    for (int j = 1; j < 2 * N; ++j) {
      pno[j] = mulmod_h(root, pno[j - 1], q);
      ipno[j] = mulmod_h(iroot, ipno[j - 1], q);
    }
    for (int j = 0; j < N; ++j) {
      ps[j] = pno[brev(j, logN)];
      ips[j] = ipno[brev(j, logN)];
    }
    for (int j = 0; j < N / (1 << aw); ++j)
      for (int k = 0; k < (1 << aw); ++k) {
        pms[j * (1 << aw) + k] = pno[(size_t)j * brev(k, aw)];
        ipms[j * (1 << aw) + k] = mulmod_h(ipno[(size_t)j * brev(k, aw)], ninv, q);
      }
    for (int j = 0; j < 2 * N; ++j) ipno[j] = mulmod_h(ipno[j], ninv, q);
    for (int j = 0; j < N; ++j) {
      psh[j] = shoup_h(ps[j], q);
      ipsh[j] = shoup_h(ips[j], q);
    }
    auto up = [&](const std::vector<uint64_t>& v) -> void* {
      void* d = nullptr;
      if (cudaMalloc(&d, v.size() * 8) != cudaSuccess) return nullptr;
      cudaMemcpy(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
      S.d_tables.push_back(d);
      return d;
    };
    hg.psi[i] = up(ps);
    hg.inv_psi[i] = up(ips);
    hg.psi_no[i] = up(pno);
    hg.inv_psi_no[i] = up(ipno);
    hg.psi_middle_scale[i] = up(pms);
    hg.inv_psi_middle_scale[i] = up(ipms);
    hg.psi_shoup[i] = up(psh);
    hg.inv_psi_shoup[i] = up(ipsh);
    if (!hg.psi[i] || !hg.inv_psi[i] || !hg.psi_no[i] || !hg.inv_psi_no[i] || !hg.psi_middle_scale[i] ||
        !hg.inv_psi_middle_scale[i] || !hg.psi_shoup[i] || !hg.inv_psi_shoup[i])
      return -2;
  }
  return run([&] {
    cudaError_t e = cudaMemcpyToSymbol(FIDESlib::constants, &hc, sizeof(hc));
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&S.d_globals, sizeof(hg));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(S.d_globals, &hg, sizeof(hg), cudaMemcpyHostToDevice);
  });
}

// In-place transform of n_polys polynomials of n_limbs limbs ([n_polys][n_limbs][N], limb j
// under prime j), using aux (same size) as the reference's between-pass buffer.
int ref_ntt(uint64_t* data, uint64_t* aux, int n_polys, int n_limbs, int inverse, void* stream) {
  if (!S.d_globals || n_limbs < 1 || n_limbs > S.nq || n_polys < 1) return -1;
  const int N = S.N, logN = S.logN;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t cnt = (size_t)n_polys * n_limbs;
  if (cnt * 2 > S.ptr_cap) {
    if (S.d_ptrs) cudaFree(S.d_ptrs);
    if (cudaMalloc(&S.d_ptrs, cnt * 2 * sizeof(void*)) != cudaSuccess) return -2;
    S.ptr_cap = cnt * 2;
  }
  std::vector<void*> h(cnt * 2);
  for (size_t k = 0; k < cnt; ++k) {
    h[k] = data + k * N;
    h[cnt + k] = aux + k * N;
  }
  cudaMemcpyAsync(S.d_ptrs, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, s);
  void** dp = S.d_ptrs;
  void** ap = S.d_ptrs + cnt;
  constexpr int M = 4;
  using namespace FIDESlib;
  return run([&] {
    if (!inverse) {
      const dim3 b1{(uint32_t)(1 << ((logN + 1) / 2 - 1))}, b2{(uint32_t)(1 << (logN / 2 - 1))};
      const int s1 = 8 * b1.x * (2 * M + 2), s2 = 8 * b2.x * (2 * M + 2);
      NTTBatch_<false, ALGO_SHOUP><<<dim3(N / (b1.x * M * 2), n_limbs, n_polys), b1, s1, s>>>(S.d_globals, dp, 0, ap,
                                                                                              n_limbs);
      NTTBatch_<true, ALGO_SHOUP><<<dim3(N / (b2.x * M * 2), n_limbs, n_polys), b2, s2, s>>>(S.d_globals, ap, 0, dp,
                                                                                             n_limbs);
    } else {
      const dim3 b1{(uint32_t)(1 << (logN / 2 - 1))}, b2{(uint32_t)(1 << ((logN + 1) / 2 - 1))};
      const int s1 = 8 * b1.x * (2 * M + 2), s2 = 8 * b2.x * (2 * M + 2);
      for (int p = 0; p < n_polys; ++p) {
        INTT_<false, ALGO_SHOUP, INTT_NONE><<<dim3(N / (b1.x * M * 2), n_limbs), b1, s1, s>>>(
            S.d_globals, dp + (size_t)p * n_limbs, 0, ap + (size_t)p * n_limbs);
        INTT_<true, ALGO_SHOUP, INTT_NONE><<<dim3(N / (b2.x * M * 2), n_limbs), b2, s2, s>>>(
            S.d_globals, ap + (size_t)p * n_limbs, 0, dp + (size_t)p * n_limbs);
      }
    }
    return cudaSuccess;
  });
}

// Destination prime ids of digit d (ModUp output row j_ is prime ids[j_]); returns the count.
int ref_modup_dst(int d, int* ids) {
  if (d < 0 || d >= (int)S.to.size()) return -1;
  for (size_t j = 0; j < S.to[d].size(); ++j) ids[j] = S.to[d][j];
  return (int)S.to[d].size();
}

// ModUp conversion of digit d at level n: x holds the n coefficient-domain Q limbs [n][N];
// out [count][N] receives row j_ for destination prime ref_modup_dst(d)[j_] (rows of
// inactive Q primes, >= n, are left untouched).
int ref_modup(const uint64_t* x, int n, int d, uint64_t* out, void* stream) {
  if (!S.d_globals || n < 1 || n > S.nq || d < 0 || d >= S.dnum) return -1;
  const int lo = d * S.alpha, cnt = std::max(0, std::min(n, lo + S.alpha) - lo);
  if (cnt == 0) return -1;
  const int nto = (int)S.to[d].size();
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<void*> h(cnt + nto);
  for (int i = 0; i < cnt; ++i) h[i] = const_cast<uint64_t*>(x) + (size_t)(lo + i) * S.N;
  for (int j = 0; j < nto; ++j) h[cnt + j] = out + (size_t)j * S.N;
  if ((size_t)(cnt + nto) > S.ptr_cap) {
    if (S.d_ptrs) cudaFree(S.d_ptrs);
    if (cudaMalloc(&S.d_ptrs, (cnt + nto) * sizeof(void*)) != cudaSuccess) return -2;
    S.ptr_cap = cnt + nto;
  }
  cudaMemcpyAsync(S.d_ptrs, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, s);
  using namespace FIDESlib;
  return run([&] {
    const dim3 block{64, 2};
    CKKS::DecompAndModUpConv<ALGO_SHOUP><<<dim3(S.N / 64), block, sizeof(uint64_t) * cnt * 64, s>>>(
        S.d_ptrs, n, S.d_ptrs + cnt, d, S.d_globals);
    return cudaSuccess;
  });
}

// ModDown conversion: sp holds the K coefficient-domain special limbs [K][N]; out [n][N]
// receives the conversion to Q limbs 0..n-1.
int ref_moddown(const uint64_t* sp, int n, uint64_t* out, void* stream) {
  if (!S.d_globals || S.K < 1 || n < 1 || n > S.nq) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<void*> h(n + S.K);
  for (int j = 0; j < n; ++j) h[j] = out + (size_t)j * S.N;
  for (int k = 0; k < S.K; ++k) h[n + k] = const_cast<uint64_t*>(sp) + (size_t)k * S.N;
  if ((size_t)(n + S.K) > S.ptr_cap) {
    if (S.d_ptrs) cudaFree(S.d_ptrs);
    if (cudaMalloc(&S.d_ptrs, (n + S.K) * sizeof(void*)) != cudaSuccess) return -2;
    S.ptr_cap = n + S.K;
  }
  cudaMemcpyAsync(S.d_ptrs, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, s);
  using namespace FIDESlib;
  return run([&] {
    const dim3 block{64, 2};
    CKKS::ModDown2<ALGO_SHOUP><<<dim3(S.N / 64), block, sizeof(uint64_t) * S.K * 64, s>>>(S.d_ptrs, n, S.d_ptrs + n,
                                                                                    PARTITION(0, 0), S.d_globals);
    return cudaSuccess;
  });
}

void ref_kernels_free(void) { release(); }

}  // extern "C"
