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
// The reduced-noise variant of both conversions (C_.reduced_noise with the DecompAndModUp_negQ
// table of src/ReducedNoiseConstants.cu) is switched by ref_kernels_set_reduced_noise.
// It also drives the reference's basis conversions with their geometry (block 64 x 2, one
// coefficient column per thread, LimbPartitionMGPU.cu:1296-1303 and :1642-1651):
//   * DecompAndModUpConv<ALGO_SHOUP> (src/CKKS/Conv.cu:274-423) for one digit at one level;
//   * ModDown2<ALGO_SHOUP> (src/CKKS/Conv.cu:27-133), special limbs -> Q limbs;
// with the digit metadata of the __constant__ block (contiguous digits of alpha = ceil(L /
// dnum) primes) and the Q-hat tables in the reference's index layouts (MODUPIDX_SCALE,
// MODUPIDX_MATRIX, MODDOWN_MATRIX), computed here from the primes.
// And the key-switch and elementwise kernels with their launch geometry (grid N/128 x limbs,
// 128 threads):
//   * fusedDotKSK_2_ (src/CKKS/ElemenwiseBatchKernels.cu:202-274), the KSK inner product, over
//     the reference's digit pointer tables (LimbPartitionMGPU.cu:470-503): per digit the ModUp
//     output and the two key halves in DIGIT order (special primes first, then the Q primes of
//     the other digits, Context.cu:157-197), plus the own-digit (DECOMP) limbs;
//   * hoistedRotateDotKSK_2_ (:277-377), the hoisted-rotation inner product with P c0 and the
//     automorphism scatter, over the tables of LimbPartitionMGPU.cu:590-655;
//   * automorph_ (src/Rotation.cu:10-12), SwitchModulus (src/CKKS/Rescale.cu:8-13),
//     binomialMult_ (ElemenwiseBatchKernels.cu:1363-1398), add_ / sub_ / scalar_add_
//     (src/AddSub.cu:31-111), mult_ / scalar_mult_ (src/ModMult.cu:8-21).
// The digit metadata of the __constant__ block follows SetupConstants (src/ConstantsGPU.cu:
// 638-681): primeid_digit (special primes: -1), pos_in_digit (DECOMP position for a digit's own
// primes, DIGIT position otherwise), primeid_digit_to, P and its Shoup companion.
// Outputs are bit-identical to this project's kernels and to the oracle for the same primes,
// root and inputs (tests/test_ref_kernels.py), which is how the harness is validated before
// timing.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "NTT.cu"
#include "CKKS/Conv.cu"
#include "CKKS/ElemenwiseBatchKernels.cu"
#include "Rotation.cu"
#include "CKKS/Rescale.cu"
#include "AddSub.cu"
#include "ModMult.cu"

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
  std::vector<std::vector<int>> to;  // per digit: destination prime ids (primeid_digit_to order:
                                     // special primes first, then the other digits' Q primes)
  Global::Globals* d_globals = nullptr;
  std::vector<void*> d_tables;
  void** d_ptrs = nullptr;  // pointer tables (data, aux)
  size_t ptr_cap = 0;
  void** d_ksk = nullptr;  // pointer tables of the key-switch kernels
  size_t ksk_cap = 0;
  uint64_t* d_scal = nullptr;  // scalar_add_'s per-prime scalars
  std::vector<uint64_t> primes;
} S;

uint64_t S_primes(int id) { return S.primes[id]; }

void release() {
  for (void* p : S.d_tables) cudaFree(p);
  S.d_tables.clear();
  if (S.d_globals) cudaFree(S.d_globals);
  if (S.d_ptrs) cudaFree(S.d_ptrs);
  if (S.d_ksk) cudaFree(S.d_ksk);
  if (S.d_scal) cudaFree(S.d_scal);
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
  S.primes.assign(primes, primes + np);
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
    for (int k = 0; k < K; ++k) S.to[d].push_back(n_q + k);
    for (int i = 0; i < n_q; ++i)
      if (i < lo || i >= hi) S.to[d].push_back(i);
    for (int j = 0; j < (int)S.to[d].size(); ++j) {
      hc.primeid_digit_to[d][j] = S.to[d][j];
      hc.pos_in_digit[d][S.to[d][j]] = j;
    }
    for (int n = 1; n <= n_q; ++n) {
      hc.num_primeid_digit_from[d][n - 1] = std::max(0, std::min(hi, n) - lo);
      int cnt = K;  // special primes, then the other digits' primes active at level n
      for (int i = 0; i < n; ++i)
        if (i < lo || i >= hi) ++cnt;
      hc.num_primeid_digit_to[d][n - 1] = cnt;
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
    hc.P_shoup[j] = shoup_h(P, primes[j]);
    hc.primeid_digit[j] = j / alpha;
  }
  for (int k = 0; k < K; ++k) hc.primeid_digit[n_q + k] = -1;  // special primes belong to no digit
  // reduced-noise ModUp constants (src/ReducedNoiseConstants.cu:16-33): -(product of the first
  // s + 1 primes of digit d) mod p_t at MODUPIDX_SCALE(d, s, t); ModDown's uses P (above)
  for (int d = 0; d < dnum; ++d) {
    const int lo = d * alpha, hi = std::min(n_q, (d + 1) * alpha);
    for (int t = 0; t < np; ++t) {
      uint64_t Qmod = 1 % primes[t];
      for (int sidx = 0; sidx < hi - lo; ++sidx) {
        Qmod = mulm(Qmod, primes[lo + sidx], primes[t]);
        hg.DecompAndModUp_negQ[FIDESlib_MODUPIDX_SCALE(d, sidx, t)] = (primes[t] - Qmod) % primes[t];
      }
    }
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
// Sets the __constant__ block's reduced_noise flag (reference Parameters::reducedNoise), read by
// DecompAndModUpConv and ModDown2 (src/CKKS/Conv.cu:76-87, :356-381).
int ref_kernels_set_reduced_noise(int on) {
  if (!S.d_globals) return -1;
  const bool b = on != 0;
  return run([&] { return cudaMemcpyToSymbol(FIDESlib::constants, &b, sizeof(b), offsetof(Constants, reduced_noise)); });
}

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


}  // extern "C"

namespace {

// Uploads pointer tables into the key-switch table buffer (grown as needed), in order.
void** upload_tables(const std::vector<void*>& h, cudaStream_t s) {
  if (h.size() > S.ksk_cap) {
    if (S.d_ksk) cudaFree(S.d_ksk);
    S.d_ksk = nullptr;
    if (cudaMalloc(&S.d_ksk, h.size() * sizeof(void*)) != cudaSuccess) return nullptr;
    S.ksk_cap = h.size();
  }
  cudaMemcpyAsync(S.d_ksk, h.data(), h.size() * sizeof(void*), cudaMemcpyHostToDevice, s);
  return S.d_ksk;
}

int digits_at(int level) { return (level + S.alpha - 1) / S.alpha; }

// Times `reps` launches of f on s (after one untimed launch): each launch is bracketed by its
// own pair of events, the way this project's profiling mode brackets its launches, and *ms is
// the mean of the bracketed times (so host issue gaps between launches are not counted).
template <typename F>
int timed(F&& f, int reps, float* ms, cudaStream_t s) {
  f();
  if (reps <= 0) return run([] { return cudaSuccess; });
  std::vector<cudaEvent_t> ev(2 * reps);
  for (auto& e : ev) cudaEventCreate(&e);
  for (int r = 0; r < reps; ++r) {
    cudaEventRecord(ev[2 * r], s);
    f();
    cudaEventRecord(ev[2 * r + 1], s);
  }
  cudaEventSynchronize(ev.back());
  float total = 0;
  for (int r = 0; r < reps; ++r) {
    float t = 0;
    cudaEventElapsedTime(&t, ev[2 * r], ev[2 * r + 1]);
    total += t;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (ms) *ms = total / reps;
  return run([] { return cudaSuccess; });
}

// Device pointer tables of one switching key in the reference's layout, for n_q + K primes:
// per digit d the DIGIT-order limbs (at index pos_in_digit[d][id]) of each half, and the
// DECOMP limbs (limb j of the prime's own digit).  Our key is [2][dnum][n_q + K][N].
struct KeyTables {
  std::vector<void*> a_digit[FIDESlib::MAXD], b_digit[FIDESlib::MAXD], a_dec, b_dec;
};
KeyTables key_tables(const uint64_t* key) {
  KeyTables t;
  const size_t N = S.N, np = S.np;
  auto limb = [&](int half, int d, int id) { return (void*)(key + (((size_t)half * S.dnum + d) * np + id) * N); };
  for (int d = 0; d < S.dnum; ++d)
    for (int id : S.to[d]) {
      t.a_digit[d].push_back(limb(0, d, id));
      t.b_digit[d].push_back(limb(1, d, id));
    }
  for (int j = 0; j < S.nq; ++j) {
    t.a_dec.push_back(limb(0, j / S.alpha, j));
    t.b_dec.push_back(limb(1, j / S.alpha, j));
  }
  return t;
}

// DIGIT-order table of a ModUp output digit d at level l in our layout [beta][l + K][N]
// (Q limbs, then special limbs); entries of inactive primes are null (never read).
std::vector<void*> digit_table(const uint64_t* digits, int level, int d) {
  const size_t N = S.N, ext = level + S.K;
  std::vector<void*> v;
  for (int id : S.to[d]) {
    if (id >= S.nq)
      v.push_back((void*)(digits + ((size_t)d * ext + level + (id - S.nq)) * N));
    else if (id < level)
      v.push_back((void*)(digits + ((size_t)d * ext + id) * N));
    else
      v.push_back(nullptr);
  }
  return v;
}

}  // namespace

extern "C" {

// KSK inner product through the reference's fusedDotKSK_2_: digits = the ModUp output of a
// level-`level` polynomial in our layout [beta][level + K][N] (own-digit limbs included), key
// = [2][dnum][n_q + K][N]; out_a / out_b [level + K][N] receive sum_d digit_d * key_(a/b, d).
// reps > 0: *ms = mean time of `reps` further launches (tables uploaded once).
int ref_ksk(const uint64_t* digits, int level, const uint64_t* key, uint64_t* out_a, uint64_t* out_b, int reps,
            float* ms, void* stream) {
  if (!S.d_globals || S.K < 1 || level < 1 || level > S.nq) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int dn = S.dnum, nd = digits_at(level), K = S.K;
  const size_t N = S.N;
  KeyTables kt = key_tables(key);
  // flat host image: [6 dnum table pointers][tables...][4 output tables]
  std::vector<std::vector<void*>> tabs(6 * dn);
  std::vector<void*> src_dec, oa, ob, oas, obs;
  for (int j = 0; j < level; ++j) {
    src_dec.push_back((void*)(digits + ((size_t)(j / S.alpha) * (level + K) + j) * N));
    oa.push_back(out_a + (size_t)j * N);
    ob.push_back(out_b + (size_t)j * N);
  }
  for (int k = 0; k < K; ++k) {
    oas.push_back(out_a + (size_t)(level + k) * N);
    obs.push_back(out_b + (size_t)(level + k) * N);
  }
  for (int d = 0; d < nd; ++d) {
    tabs[d] = digit_table(digits, level, d);
    tabs[d + dn] = kt.a_digit[d];
    tabs[d + 2 * dn] = kt.b_digit[d];
    tabs[d + 3 * dn] = src_dec;
    tabs[d + 4 * dn] = kt.a_dec;
    tabs[d + 5 * dn] = kt.b_dec;
  }
  std::vector<void*> h(6 * dn, nullptr);
  std::vector<size_t> at(6 * dn, 0);
  for (int t = 0; t < 6 * dn; ++t) {
    at[t] = h.size();
    h.insert(h.end(), tabs[t].begin(), tabs[t].end());
  }
  const size_t o_oa = h.size();
  h.insert(h.end(), oa.begin(), oa.end());
  const size_t o_oas = h.size();
  h.insert(h.end(), oas.begin(), oas.end());
  const size_t o_ob = h.size();
  h.insert(h.end(), ob.begin(), ob.end());
  const size_t o_obs = h.size();
  h.insert(h.end(), obs.begin(), obs.end());
  // the table of tables holds device addresses: fix them up before the upload
  void** base = nullptr;
  if (h.size() > S.ksk_cap) {  // grow first so that the final address is known
    if (!upload_tables(h, s)) return -2;
  }
  base = S.d_ksk;
  for (int t = 0; t < 6 * dn; ++t) h[t] = tabs[t].empty() ? nullptr : (void*)(base + at[t]);
  if (!upload_tables(h, s)) return -2;
  using namespace FIDESlib;
  auto launch = [&] {
    CKKS::fusedDotKSK_2_<<<dim3(S.N / 128, K + level), 128, 0, s>>>(base + o_oa, base + o_oas, base + o_ob,
                                                                      base + o_obs, (void***)base, nd, 0, K, 0);
  };
  return timed(launch, reps, ms, s);
}

// Hoisted-rotation inner product through the reference's hoistedRotateDotKSK_2_: one
// ModUp output `digits` of c1 (our layout), c0 [level][N], n rotations with keys[r] and
// automorphism indices ks[r]; out0[r] / out1[r] [level + K][N] receive the automorphism of
// (sum_d digit_d key_(b, d) + P c0) and of sum_d digit_d key_(a, d).
int ref_hoisted_ksk(const uint64_t* digits, const uint64_t* c0, int level, int n, const uint64_t* const* keys,
                    const int* ks, uint64_t* const* out0, uint64_t* const* out1, int reps, float* ms, void* stream) {
  if (!S.d_globals || S.K < 1 || level < 1 || level > S.nq || n < 1) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int dn = S.dnum, nd = digits_at(level), K = S.K;
  const size_t N = S.N;
  // table-of-tables layout (LimbPartitionMGPU.cu:590-655): rotation r's key tables at
  // [r 6 dnum + (1, 2, 4, 5) dnum + d], the c1 digits at offset_c1 (+ 3 dnum for the DECOMP
  // limbs), then per output kind n tables, then the indices.
  const size_t off_c1 = (size_t)n * 6 * dn;
  const size_t off_o1 = off_c1 + 6 * dn, off_o0 = off_o1 + n, off_o1s = off_o0 + n, off_o0s = off_o1s + n;
  const size_t off_idx = off_o0s + n;
  const size_t n_heads = off_idx + (n + 1) / 2 + 1;  // indices packed as ints
  std::vector<std::vector<void*>> tabs(n_heads);
  for (int r = 0; r < n; ++r) {
    KeyTables kt = key_tables(keys[r]);
    for (int d = 0; d < nd; ++d) {
      tabs[r * 6 * dn + d + dn] = kt.a_digit[d];
      tabs[r * 6 * dn + d + 2 * dn] = kt.b_digit[d];
      tabs[r * 6 * dn + d + 4 * dn] = kt.a_dec;
      tabs[r * 6 * dn + d + 5 * dn] = kt.b_dec;
    }
  }
  std::vector<void*> c1_dec, c0_q;
  for (int j = 0; j < level; ++j) {
    c1_dec.push_back((void*)(digits + ((size_t)(j / S.alpha) * (level + K) + j) * N));
    c0_q.push_back((void*)(c0 + (size_t)j * N));
  }
  for (int d = 0; d < nd; ++d) {
    tabs[off_c1 + d] = digit_table(digits, level, d);
    tabs[off_c1 + d + 3 * dn] = c1_dec;
  }
  for (int r = 0; r < n; ++r) {
    std::vector<void*> q1, q0, s1, s0;
    for (int j = 0; j < level; ++j) {
      q1.push_back(out1[r] + (size_t)j * N);
      q0.push_back(out0[r] + (size_t)j * N);
    }
    for (int k = 0; k < K; ++k) {
      s1.push_back(out1[r] + (size_t)(level + k) * N);
      s0.push_back(out0[r] + (size_t)(level + k) * N);
    }
    tabs[off_o1 + r] = q1;
    tabs[off_o0 + r] = q0;
    tabs[off_o1s + r] = s1;
    tabs[off_o0s + r] = s0;
  }
  std::vector<void*> h(n_heads, nullptr);
  std::vector<size_t> at(n_heads, 0);
  for (size_t t = 0; t < n_heads; ++t) {
    at[t] = h.size();
    h.insert(h.end(), tabs[t].begin(), tabs[t].end());
  }
  const size_t o_c0 = h.size();
  h.insert(h.end(), c0_q.begin(), c0_q.end());
  if (h.size() > S.ksk_cap && !upload_tables(h, s)) return -2;
  void** base = S.d_ksk;
  for (size_t t = 0; t < n_heads; ++t) h[t] = tabs[t].empty() ? nullptr : (void*)(base + at[t]);
  std::memset(&h[off_idx], 0, ((n + 1) / 2 + 1) * sizeof(void*));
  std::memcpy(&h[off_idx], ks, n * sizeof(int));
  if (!upload_tables(h, s)) return -2;
  using namespace FIDESlib;
  auto launch = [&] {
    CKKS::hoistedRotateDotKSK_2_<<<dim3(S.N / 128, K + level), 128, sizeof(uint64_t) * 128 * nd, s>>>(
        (void***)(base + off_c1), base + o_c0, (void***)(base + off_o1), (void***)(base + off_o1s),
        (void***)(base + off_o0), (void***)(base + off_o0s), n, (const int*)(base + off_idx), (void***)base, nd, 0, K,
        0, nullptr, false);
  };
  return timed(launch, reps, ms, s);
}

// automorph_ on one limb: out[automorph_slot(j)] = in[j] for automorphism index k.
int ref_automorph(const uint64_t* in, uint64_t* out, int k, void* stream) {
  if (!S.d_globals) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  using namespace FIDESlib;
  return run([&] {
    CKKS::automorph_<uint64_t><<<S.N / 128, 128, 0, s>>>(const_cast<uint64_t*>(in), out, k, 0);
    return cudaSuccess;
  });
}

// SwitchModulus of one coefficient vector (N words) from prime o_pid to prime n_pid.
int ref_switch_modulus(const uint64_t* in, int o_pid, uint64_t* out, int n_pid, void* stream) {
  if (!S.d_globals || o_pid < 0 || o_pid >= S.np || n_pid < 0 || n_pid >= S.np) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  using namespace FIDESlib;
  return run([&] {
    CKKS::SwitchModulus<uint64_t><<<S.N / 128, 128, 0, s>>>(in, o_pid, out, n_pid);
    return cudaSuccess;
  });
}

// Elementwise kernels over `level` Q limbs (limb j under prime j), in place on a:
//   op 0: a += b (add_), 1: a -= b (sub_), 2: a *= b (mult_, Barrett), 3: a *= scalars[j]
//   (scalar_mult_, Shoup), 4: a += scalars[j] (scalar_add_); scalars: host array of level words.
int ref_elementwise(int op, uint64_t* a, const uint64_t* b, const uint64_t* scalars, int level, void* stream) {
  if (!S.d_globals || level < 1 || level > S.nq || op < 0 || op > 4) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N = S.N;
  std::vector<void*> h;
  for (int j = 0; j < level; ++j) h.push_back(a + (size_t)j * N);
  for (int j = 0; j < level; ++j) h.push_back(b ? (void*)(b + (size_t)j * N) : nullptr);
  if (!upload_tables(h, s)) return -2;
  void** base = S.d_ksk;
  if (op == 4) {
    if (!S.d_scal && cudaMalloc(&S.d_scal, MAXP * sizeof(uint64_t)) != cudaSuccess) return -2;
    cudaMemcpyAsync(S.d_scal, scalars, level * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
  }
  using namespace FIDESlib;
  return run([&] {
    const dim3 grid(S.N / 128, level);
    if (op == 0) add_<<<grid, 128, 0, s>>>(base, base + level, PARTITION(0, 0));
    if (op == 1) sub_<<<grid, 128, 0, s>>>(base, base + level, PARTITION(0, 0));
    if (op == 4) scalar_add_<<<grid, 128, 0, s>>>(base, S.d_scal, PARTITION(0, 0));
    for (int j = 0; op == 2 && j < level; ++j)
      mult_<uint64_t, ALGO_BARRETT><<<S.N / 128, 128, 0, s>>>(a + j * N, b + j * N, j);
    for (int j = 0; op == 3 && j < level; ++j) {
      const uint64_t q = S_primes(j);
      const uint64_t w = scalars[j] % q;
      scalar_mult_<uint64_t, ALGO_SHOUP><<<S.N / 128, 128, 0, s>>>(a + j * N, w, j, shoup_h(w, q));
    }
    return cudaSuccess;
  });
}

// binomialMult_ in place: (c0, c1, c2) <- (c0 d0, c0 d1 + c1 d0, c1 d1) over `level` Q limbs.
int ref_tensor(uint64_t* c0, uint64_t* c1, uint64_t* c2, const uint64_t* d0, const uint64_t* d1, int level,
               void* stream) {
  if (!S.d_globals || level < 1 || level > S.nq) return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t N = S.N;
  std::vector<void*> h;
  for (uint64_t* p : {c0, c1, c2})
    for (int j = 0; j < level; ++j) h.push_back(p + (size_t)j * N);
  for (const uint64_t* p : {d0, d1})
    for (int j = 0; j < level; ++j) h.push_back((void*)(p + (size_t)j * N));
  if (!upload_tables(h, s)) return -2;
  void** base = S.d_ksk;
  using namespace FIDESlib;
  return run([&] {
    CKKS::binomialMult_<<<dim3(S.N / 128, level), 128, 0, s>>>(PARTITION(0, 0), base, base + level,
                                                                base + 2 * level, base + 3 * level,
                                                                base + 4 * level);
    return cudaSuccess;
  });
}

void ref_kernels_free(void) { release(); }

}  // extern "C"
