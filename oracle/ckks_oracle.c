/*
 * ckks_oracle.c -- CPU restatement of the reference's CKKS evaluation arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY (the checker): used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU baseline / reference arm.  The GPU product never calls it.
 *
 * Each routine cites the reference code whose semantics it restates.  The code
 * favours plain, obviously-correct arithmetic: exact residues in [0, q) after
 * every operation, 128-bit products, Shoup precomputation only for NTT twiddles
 * (an exact technique, as OpenFHE's NTT uses) so that the oracle is fast enough
 * to act as the timed CPU baseline.
 */
#include "ckks_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* number theory                                                              */
/* ------------------------------------------------------------------------- */

/* reference src/Math.cu:18-21 (modprod) */
uint64_t or_mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

/* reference src/Math.cu:23-33 (modpow) */
uint64_t or_powmod(uint64_t a, uint64_t e, uint64_t q) {
  uint64_t r = 1 % q;
  a %= q;
  while (e) {
    if (e & 1) r = or_mulmod(r, a, q);
    a = or_mulmod(a, a, q);
    e >>= 1;
  }
  return r;
}

/* reference src/Math.cu:35-38 (modinv by Fermat; q prime) */
uint64_t or_invmod(uint64_t a, uint64_t q) { return or_powmod(a, q - 2, q); }

static uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
  uint64_t c = a + b;
  return c >= q ? c - q : c;
}
static uint64_t submod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }

/* Deterministic Miller-Rabin for 64-bit n (first 12 prime bases suffice). */
int or_is_prime(uint64_t n) {
  static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
  if (n < 2) return 0;
  for (int i = 0; i < 12; ++i) {
    if (n == bases[i]) return 1;
    if (n % bases[i] == 0) return 0;
  }
  uint64_t d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  for (int i = 0; i < 12; ++i) {
    uint64_t x = or_powmod(bases[i], d, n);
    if (x == 1 || x == n - 1) continue;
    int comp = 1;
    for (int r = 1; r < s; ++r) {
      x = or_mulmod(x, x, n);
      if (x == n - 1) {
        comp = 0;
        break;
      }
    }
    if (comp) return 0;
  }
  return 1;
}

/* Deterministic NTT-friendly prime search: descending from 2^bits over q = 1 mod 2N.
 * (OpenFHE's own prime choice is not available here; this is the documented synthetic rule.) */
int or_gen_primes(int logN, int bits, int count, const uint64_t* exclude, int n_exclude, uint64_t* out) {
  const uint64_t m = 2ull << logN;
  uint64_t top = (bits >= 64) ? ~0ull : (1ull << bits);
  uint64_t q = (top / m) * m + 1;
  if (q >= top) q -= m;
  int got = 0;
  while (got < count && q > m) {
    int skip = 0;
    for (int i = 0; i < n_exclude; ++i)
      if (exclude[i] == q) skip = 1;
    if (!skip && or_is_prime(q)) out[got++] = q;
    q -= m;
  }
  return got;
}

/* Smallest primitive root of q, reference src/ConstantsGPU.cu:39-59 (`generator`). */
uint64_t or_generator(uint64_t q) {
  uint64_t fact[64];
  int nf = 0;
  uint64_t phi = q - 1, n = phi;
  for (uint64_t i = 2; i * i <= n; ++i) {
    if (n % i == 0) {
      fact[nf++] = i;
      while (n % i == 0) n /= i;
    }
  }
  if (n > 1) fact[nf++] = n;
  for (uint64_t g = 2; g <= q; ++g) {
    int ok = 1;
    for (int i = 0; i < nf && ok; ++i) ok = or_powmod(g, phi / fact[i], q) != 1;
    if (ok) return g;
  }
  return 0;
}

/* Primitive 2N-th root psi = g^((q-1)/2N), reference src/ConstantsGPU.cu:62-69 (`unity_root`). */
uint64_t or_root_2n(uint64_t q, int logN) {
  uint64_t order = 2ull << logN;
  return or_powmod(or_generator(q), (q - 1) / order, q);
}

/* reference src/Math.cu:145-151 */
uint32_t or_bit_reverse(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

/* ------------------------------------------------------------------------- */
/* context                                                                    */
/* ------------------------------------------------------------------------- */

struct or_ctx {
  int logN, N, n_q, n_p, dnum, alpha;
  uint64_t* primes; /* n_q + n_p */
  uint64_t* psi;
  /* per prime: psi_rev, psi_rev_shoup, ipsi_rev, ipsi_rev_shoup (N each), n_inv */
  uint64_t** tw;
  uint64_t* n_inv;
  int reduced_noise; /* reference Parameters::reducedNoise (src/CKKS/Parameters.cuh:31) */
};

static uint64_t shoup_pre(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }
static inline uint64_t shoup_mul(uint64_t x, uint64_t w, uint64_t wp, uint64_t q) {
  uint64_t hi = (uint64_t)(((u128)x * wp) >> 64);
  uint64_t r = x * w - hi * q;
  return r >= q ? r - q : r;
}

/* Twiddle tables: psi_rev[j] = psi^brev(j) (reference src/ConstantsGPU.cu:246-276). */
or_ctx* or_ctx_create(int logN, int n_q, int n_p, const uint64_t* primes, const uint64_t* psi, int dnum) {
  or_ctx* c = (or_ctx*)calloc(1, sizeof(or_ctx));
  int np = n_q + n_p;
  c->logN = logN;
  c->N = 1 << logN;
  c->n_q = n_q;
  c->n_p = n_p;
  c->dnum = dnum;
  c->alpha = (n_q + dnum - 1) / dnum;
  c->primes = (uint64_t*)malloc(sizeof(uint64_t) * np);
  c->psi = (uint64_t*)malloc(sizeof(uint64_t) * np);
  c->tw = (uint64_t**)calloc(np, sizeof(uint64_t*));
  c->n_inv = (uint64_t*)malloc(sizeof(uint64_t) * np);
  memcpy(c->primes, primes, sizeof(uint64_t) * np);
  for (int i = 0; i < np; ++i) c->psi[i] = (psi && psi[i]) ? psi[i] : or_root_2n(primes[i], logN);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < np; ++i) {
    const int N = c->N;
    uint64_t q = c->primes[i];
    uint64_t* t = (uint64_t*)malloc(sizeof(uint64_t) * 4 * N);
    uint64_t* pw = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t* ipw = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t ip = or_invmod(c->psi[i], q);
    pw[0] = 1;
    ipw[0] = 1;
    for (int j = 1; j < N; ++j) {
      pw[j] = or_mulmod(pw[j - 1], c->psi[i], q);
      ipw[j] = or_mulmod(ipw[j - 1], ip, q);
    }
    for (int j = 0; j < N; ++j) {
      uint32_t r = or_bit_reverse((uint32_t)j, logN);
      t[j] = pw[r];
      t[N + j] = shoup_pre(pw[r], q);
      t[2 * N + j] = ipw[r];
      t[3 * N + j] = shoup_pre(ipw[r], q);
    }
    free(pw);
    free(ipw);
    c->tw[i] = t;
    c->n_inv[i] = or_invmod((uint64_t)N % q, q);
  }
  return c;
}

void or_ctx_destroy(or_ctx* c) {
  if (!c) return;
  for (int i = 0; i < c->n_q + c->n_p; ++i) free(c->tw[i]);
  free(c->tw);
  free(c->primes);
  free(c->psi);
  free(c->n_inv);
  free(c);
}

int or_ctx_alpha(const or_ctx* c) { return c->alpha; }
uint64_t or_ctx_psi(const or_ctx* c, int prime_id) { return c->psi[prime_id]; }

void or_set_threads(int n) {
#ifdef _OPENMP
  if (n <= 0) n = omp_get_num_procs();
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* NTT                                                                        */
/* ------------------------------------------------------------------------- */

/* Forward negacyclic NTT into bit-reversed (EVALUATION) order.  Restates the butterfly
 * loop of reference test/cpuNTT_nega.cpp:37-77 (`nega_fft`), stopping before its final
 * natural-order permutation (the GPU/OpenFHE format is bit-reversed, test/NTTtests.cu:447-467). */
static void ntt_fwd_limb(uint64_t* a, int logN, uint64_t q, const uint64_t* tw) {
  const int N = 1 << logN;
  const uint64_t* w = tw;
  const uint64_t* wp = tw + N;
  int t = N >> 1;
  for (int m = 1; m < N; m <<= 1, t >>= 1) {
    for (int i = 0; i < m; ++i) {
      const uint64_t W = w[m + i], Wp = wp[m + i];
      uint64_t* x = a + 2 * i * t;
      for (int j = 0; j < t; ++j) {
        uint64_t u = x[j];
        uint64_t v = shoup_mul(x[j + t], W, Wp, q);
        x[j] = addmod(u, v, q);
        x[j + t] = submod(u, v, q);
      }
    }
  }
}

/* Inverse: Gentleman-Sande from bit-reversed order, then N^-1 (OpenFHE's inverse from
 * bit-reversed order; reference src/NTT.cu:42-327 + src/NTTfusions.cuh:413-496 fold N^-1). */
static void ntt_inv_limb(uint64_t* a, int logN, uint64_t q, const uint64_t* tw, uint64_t n_inv) {
  const int N = 1 << logN;
  const uint64_t* w = tw + 2 * N;
  const uint64_t* wp = tw + 3 * N;
  int t = 1;
  for (int m = N >> 1; m >= 1; m >>= 1, t <<= 1) {
    for (int i = 0; i < m; ++i) {
      const uint64_t W = w[m + i], Wp = wp[m + i];
      uint64_t* x = a + 2 * i * t;
      for (int j = 0; j < t; ++j) {
        uint64_t u = x[j], v = x[j + t];
        x[j] = addmod(u, v, q);
        x[j + t] = shoup_mul(submod(u, v, q), W, Wp, q);
      }
    }
  }
  uint64_t np = shoup_pre(n_inv, q);
  for (int j = 0; j < N; ++j) a[j] = shoup_mul(a[j], n_inv, np, q);
}

void or_ntt(const or_ctx* c, uint64_t* a, int n_limbs, const int* prime_ids, int inverse) {
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < n_limbs; ++i) {
    int p = prime_ids[i];
    uint64_t* x = a + (size_t)i * c->N;
    if (inverse)
      ntt_inv_limb(x, c->logN, c->primes[p], c->tw[p], c->n_inv[p]);
    else
      ntt_fwd_limb(x, c->logN, c->primes[p], c->tw[p]);
  }
}

/* ------------------------------------------------------------------------- */
/* basis conversion                                                           */
/* ------------------------------------------------------------------------- */

/* ApproxSwitchCRTBasis (no overflow correction), as the reference's DecompAndModUpConv
 * (src/CKKS/Conv.cu:274-423) and ModDown2 (src/CKKS/Conv.cu:27-133) compute it:
 *   y_i   = [x_i * (Qhat_i)^-1]_{q_i}                 (pre-scale, Qhat_i = prod_{k != i} q_k)
 *   out_j = [ sum_i y_i * [Qhat_i]_{p_j} ]_{p_j}       (128-bit accumulate, one reduction)
 * Tables as reference src/Math.cu:94-130 (q_hat_inv, p_hat). */
static void switch_basis(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out, int n_dst,
                         const int* dst_ids, int lift);

void or_switch_basis(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out, int n_dst,
                     const int* dst_ids) {
  switch_basis(c, in, n_src, src_ids, out, n_dst, dst_ids, 0);
}

void or_switch_basis_lift(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out,
                          int n_dst, const int* dst_ids) {
  switch_basis(c, in, n_src, src_ids, out, n_dst, dst_ids, 1);
}

/* With lift (the reduced-noise conversion, reference src/CKKS/Conv.cu:76-87 and :356-381,
 * src/CKKS/ReducedNoise.cuh:14-16, tables src/ReducedNoiseConstants.cu:16-33): a pre-scaled
 * y_i above q_i / 2 (q_i >> 1, strictly) stands for y_i - q_i, so out_j gains
 * cnt * [-Q_src]_{p_j}, cnt the number of such y_i of the coefficient. */
static void switch_basis(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out, int n_dst,
                         const int* dst_ids, int lift) {
  const int N = c->N;
  uint64_t* pre = (uint64_t*)malloc(sizeof(uint64_t) * n_src);
  uint64_t* mat = (uint64_t*)malloc(sizeof(uint64_t) * n_src * (n_dst ? n_dst : 1));
  for (int i = 0; i < n_src; ++i) {
    uint64_t qi = c->primes[src_ids[i]];
    uint64_t h = 1;
    for (int k = 0; k < n_src; ++k)
      if (k != i) h = or_mulmod(h, c->primes[src_ids[k]] % qi, qi);
    pre[i] = or_invmod(h, qi);
    for (int j = 0; j < n_dst; ++j) {
      uint64_t pj = c->primes[dst_ids[j]];
      uint64_t hj = 1 % pj;
      for (int k = 0; k < n_src; ++k)
        if (k != i) hj = or_mulmod(hj, c->primes[src_ids[k]] % pj, pj);
      mat[i * n_dst + j] = hj;
    }
  }
  uint64_t* negq = (uint64_t*)malloc(sizeof(uint64_t) * (n_dst ? n_dst : 1));
  for (int j = 0; j < n_dst; ++j) {
    uint64_t pj = c->primes[dst_ids[j]], v = 1 % pj;
    for (int k = 0; k < n_src; ++k) v = or_mulmod(v, c->primes[src_ids[k]] % pj, pj);
    negq[j] = v ? pj - v : 0;
  }
#pragma omp parallel
  {
    uint64_t* y = (uint64_t*)malloc(sizeof(uint64_t) * (n_src ? n_src : 1));
#pragma omp for schedule(static)
    for (int n = 0; n < N; ++n) {
      uint64_t cnt = 0;
      for (int i = 0; i < n_src; ++i) {
        y[i] = or_mulmod(in[(size_t)i * N + n], pre[i], c->primes[src_ids[i]]);
        cnt += y[i] > (c->primes[src_ids[i]] >> 1);
      }
      for (int j = 0; j < n_dst; ++j) {
        u128 acc = 0;
        for (int i = 0; i < n_src; ++i) acc += (u128)y[i] * mat[i * n_dst + j];
        if (lift) acc += (u128)cnt * negq[j];
        out[(size_t)j * N + n] = (uint64_t)(acc % c->primes[dst_ids[j]]);
      }
    }
    free(y);
  }
  free(pre);
  free(mat);
  free(negq);
}

void or_ctx_set_reduced_noise(or_ctx* c, int on) { c->reduced_noise = on != 0; }

/* ------------------------------------------------------------------------- */
/* elementwise                                                                */
/* ------------------------------------------------------------------------- */

void or_poly_mul(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids) {
  const size_t N = (size_t)c->N;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_limbs; ++i) {
    uint64_t q = c->primes[prime_ids[i]];
    for (size_t n = 0; n < N; ++n) out[i * N + n] = or_mulmod(a[i * N + n], b[i * N + n], q);
  }
}

void or_poly_add(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids) {
  const size_t N = (size_t)c->N;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_limbs; ++i) {
    uint64_t q = c->primes[prime_ids[i]];
    for (size_t n = 0; n < N; ++n) out[i * N + n] = addmod(a[i * N + n], b[i * N + n], q);
  }
}

void or_poly_sub(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids) {
  const size_t N = (size_t)c->N;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_limbs; ++i) {
    uint64_t q = c->primes[prime_ids[i]];
    for (size_t n = 0; n < N; ++n) out[i * N + n] = submod(a[i * N + n], b[i * N + n], q);
  }
}

/* Tensor product d0 = a0 b0, d1 = a0 b1 + a1 b0, d2 = a1 b1
 * (reference src/CKKS/ElemenwiseBatchKernels.cu:1363-1510, binomialMult_). */
void or_tensor(const or_ctx* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
               uint64_t* d0, uint64_t* d1, uint64_t* d2) {
  const size_t N = (size_t)c->N;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < l; ++i) {
    uint64_t q = c->primes[i];
    for (size_t n = 0; n < N; ++n) {
      size_t k = i * N + n;
      uint64_t x0 = a0[k], x1 = a1[k], y0 = b0[k], y1 = b1[k];
      d0[k] = or_mulmod(x0, y0, q);
      d1[k] = addmod(or_mulmod(x0, y1, q), or_mulmod(x1, y0, q), q);
      d2[k] = or_mulmod(x1, y1, q);
    }
  }
}

/* automorph_slot, reference src/Rotation.cuh:14-26: j -> brev(((2 brev(j) + 1) k mod 2N) >> 1). */
static uint32_t automorph_slot(int logN, uint32_t k, uint32_t j) {
  uint32_t jr = or_bit_reverse(j, logN);
  uint32_t t = (jr << 1) + 1;
  uint32_t r = (uint32_t)(((uint64_t)t * k) & ((2ull << logN) - 1)) >> 1;
  return or_bit_reverse(r, logN);
}

/* Scatter a_rot[sigma(j)] = a[j], reference src/Rotation.cuh:28-35 (automorph__). */
void or_automorph(const or_ctx* c, const uint64_t* in, uint64_t* out, int n_limbs, uint32_t k) {
  const size_t N = (size_t)c->N;
  uint32_t* map = (uint32_t*)malloc(sizeof(uint32_t) * N);
  for (size_t j = 0; j < N; ++j) map[j] = automorph_slot(c->logN, k, (uint32_t)j);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n_limbs; ++i)
    for (size_t j = 0; j < N; ++j) out[i * N + map[j]] = in[i * N + j];
  free(map);
}

/* Rotation index -> automorphism index.  Rotation amount normalised to [0, N/2)
 * (reference src/CKKS/Context.cu:916-924), then 5^(2N - r) mod 2N
 * (reference src/CKKS/RNSPoly.cpp:656-658); 2N-1 is the conjugation index. */
uint32_t or_rotation_auto_index(int logN, int r) {
  const int64_t N = 1ll << logN;
  if (r == 2 * N - 1) return (uint32_t)(2 * N - 1);
  int64_t h = N / 2;
  int64_t idx = r % h;
  if (idx < 0) idx += h;
  return (uint32_t)or_powmod(5, (uint64_t)(2 * N - idx), (uint64_t)(2 * N));
}

/* ------------------------------------------------------------------------- */
/* hybrid key switching                                                       */
/* ------------------------------------------------------------------------- */

int or_num_digits(const or_ctx* c, int l) { return (l + c->alpha - 1) / c->alpha; }

/* ModUp (reference LimbPartitionMGPU.cu:936-1332 for one digit: INTT of the digit's limbs,
 * DecompAndModUpConv, NTT of the new limbs).  Digit d at level l holds Q primes
 * [d*alpha, min((d+1)*alpha, l)) -- OpenFHE's contiguous partition (Context.cu:268-276).
 * Output digit d is an extended poly [l + K][N] in EVAL format; its own limbs are the
 * input limbs unchanged (the "decomp" limbs of ElemenwiseBatchKernels.cu:247-265). */
void or_modup(const or_ctx* c, const uint64_t* x, int l, uint64_t* digits) {
  const size_t N = (size_t)c->N;
  const int K = c->n_p, ext = l + K;
  const int beta = or_num_digits(c, l);
  for (int d = 0; d < beta; ++d) {
    int s0 = d * c->alpha, s1 = (d + 1) * c->alpha;
    if (s1 > l) s1 = l;
    int ns = s1 - s0;
    int* src = (int*)malloc(sizeof(int) * ns);
    int* dst = (int*)malloc(sizeof(int) * ext);
    int* dpos = (int*)malloc(sizeof(int) * ext);
    int nd = 0;
    for (int i = 0; i < ns; ++i) src[i] = s0 + i;
    for (int i = 0; i < l; ++i)
      if (i < s0 || i >= s1) {
        dst[nd] = i;
        dpos[nd++] = i;
      }
    for (int k = 0; k < K; ++k) {
      dst[nd] = c->n_q + k;
      dpos[nd++] = l + k;
    }
    uint64_t* coeff = (uint64_t*)malloc(sizeof(uint64_t) * ns * N);
    memcpy(coeff, x + (size_t)s0 * N, sizeof(uint64_t) * ns * N);
    or_ntt(c, coeff, ns, src, 1);
    uint64_t* conv = (uint64_t*)malloc(sizeof(uint64_t) * (nd ? nd : 1) * N);
    switch_basis(c, coeff, ns, src, conv, nd, dst, c->reduced_noise);
    or_ntt(c, conv, nd, dst, 0);
    uint64_t* D = digits + (size_t)d * ext * N;
    for (int i = 0; i < ns; ++i) memcpy(D + (size_t)(s0 + i) * N, x + (size_t)(s0 + i) * N, sizeof(uint64_t) * N);
    for (int j = 0; j < nd; ++j) memcpy(D + (size_t)dpos[j] * N, conv + (size_t)j * N, sizeof(uint64_t) * N);
    free(coeff);
    free(conv);
    free(src);
    free(dst);
    free(dpos);
  }
}

/* Key-switch-key inner product, reference src/CKKS/ElemenwiseBatchKernels.cu:202-274
 * (fusedDotKSK_2_): out_a[i] = sum_d D_d[i] a_d[i], out_b[i] = sum_d D_d[i] b_d[i]. */
void or_ksk_ip(const or_ctx* c, const uint64_t* digits, int l, const uint64_t* key, uint64_t* out_a, uint64_t* out_b) {
  const size_t N = (size_t)c->N;
  const int K = c->n_p, ext = l + K, kl = c->n_q + K;
  const int beta = or_num_digits(c, l);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < ext; ++i) {
    int pid = i < l ? i : c->n_q + (i - l);
    uint64_t q = c->primes[pid];
    for (size_t n = 0; n < N; ++n) {
      uint64_t sa = 0, sb = 0;
      for (int d = 0; d < beta; ++d) {
        uint64_t v = digits[((size_t)d * ext + i) * N + n];
        uint64_t ka = key[(((size_t)0 * c->dnum + d) * kl + pid) * N + n];
        uint64_t kb = key[(((size_t)1 * c->dnum + d) * kl + pid) * N + n];
        sa = addmod(sa, or_mulmod(v, ka, q), q);
        sb = addmod(sb, or_mulmod(v, kb, q), q);
      }
      out_a[i * N + n] = sa;
      out_b[i * N + n] = sb;
    }
  }
}

/* ModDown, reference src/CKKS/LimbPartition.cu:2145-2217: INTT of the K special limbs,
 * ModDown2 (Conv.cu:27-133; PHatInvModp / PHatModq), NTT, then the NTT_MODDOWN epilogue
 * out_j = (x_j - conv_j) * P^-1 mod q_j (src/NTTfusions.cuh:237-252). */
void or_moddown(const or_ctx* c, const uint64_t* in_ext, int l, uint64_t* out) {
  const size_t N = (size_t)c->N;
  const int K = c->n_p;
  int* src = (int*)malloc(sizeof(int) * (K ? K : 1));
  int* dst = (int*)malloc(sizeof(int) * l);
  for (int k = 0; k < K; ++k) src[k] = c->n_q + k;
  for (int j = 0; j < l; ++j) dst[j] = j;
  uint64_t* sp = (uint64_t*)malloc(sizeof(uint64_t) * (K ? K : 1) * N);
  memcpy(sp, in_ext + (size_t)l * N, sizeof(uint64_t) * K * N);
  or_ntt(c, sp, K, src, 1);
  uint64_t* conv = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  switch_basis(c, sp, K, src, conv, l, dst, c->reduced_noise);
  or_ntt(c, conv, l, dst, 0);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < l; ++j) {
    uint64_t q = c->primes[j];
    uint64_t P = 1;
    for (int k = 0; k < K; ++k) P = or_mulmod(P, c->primes[c->n_q + k] % q, q);
    uint64_t pinv = or_invmod(P, q);
    for (size_t n = 0; n < N; ++n)
      out[j * N + n] = or_mulmod(submod(in_ext[j * N + n], conv[j * N + n], q), pinv, q);
  }
  free(sp);
  free(conv);
  free(src);
  free(dst);
}

/* Hybrid key switch (reference LimbPartitionMGPU.cu:669-1980, modup_ksk_moddown_mgpu). */
void or_keyswitch(const or_ctx* c, const uint64_t* d, int l, const uint64_t* key, uint64_t* f0, uint64_t* f1) {
  const size_t N = (size_t)c->N;
  const int ext = l + c->n_p, beta = or_num_digits(c, l);
  uint64_t* digits = (uint64_t*)malloc(sizeof(uint64_t) * beta * ext * N);
  uint64_t* A = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* B = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  or_modup(c, d, l, digits);
  or_ksk_ip(c, digits, l, key, A, B);
  or_moddown(c, B, l, f0);
  or_moddown(c, A, l, f1);
  free(digits);
  free(A);
  free(B);
}

/* ------------------------------------------------------------------------- */
/* ciphertext ops                                                             */
/* ------------------------------------------------------------------------- */

/* OpenFHE SwitchModulus, as restated in reference src/CKKS/Rescale.cuh:44-64. */
static uint64_t switch_modulus(uint64_t a, uint64_t om, uint64_t nm) {
  uint64_t half = om >> 1;
  if (nm > om) {
    if (a > half) a += nm - om;
  } else {
    uint64_t diff = nm - (om % nm);
    if (a > half) a += diff;
    if (a >= nm) a %= nm;
  }
  return a;
}

/* SwitchModulus of n coefficients from prime src_id to prime dst_id (reference
 * src/CKKS/Rescale.cuh:44-64, itself OpenFHE's NativeVector::SwitchModulus). */
void or_switch_modulus(const or_ctx* c, const uint64_t* in, int n, int src_id, int dst_id, uint64_t* out) {
  const uint64_t om = c->primes[src_id], nm = c->primes[dst_id];
  for (int i = 0; i < n; ++i) out[i] = switch_modulus(in[i], om, nm);
}

/* Rescale (DropLastElementAndScale), reference src/NTTfusions.cuh:214-235 with
 * LimbPartition.cu:711-797: INTT of the top limb, SwitchModulus to each q_j, NTT, then
 * out_j = qlInv_j * x_j + QlQlInvModqlDivqlModq_j * t_j.  QlQlInvModqlDivqlModq_j
 * = floor(Q' [Q'^-1]_{q_l} / q_l) mod q_j with Q' = prod_{i<l-1} q_i, which equals
 * -q_l^-1 mod q_j because q_j divides Q'. */
void or_rescale(const or_ctx* c, const uint64_t* x, int l, uint64_t* out) {
  const size_t N = (size_t)c->N;
  const int top = l - 1;
  const uint64_t qt = c->primes[top];
  uint64_t* last = (uint64_t*)malloc(sizeof(uint64_t) * N);
  memcpy(last, x + (size_t)top * N, sizeof(uint64_t) * N);
  int tid = top;
  or_ntt(c, last, 1, &tid, 1);
  uint64_t* sw = (uint64_t*)malloc(sizeof(uint64_t) * (top ? top : 1) * N);
  int* ids = (int*)malloc(sizeof(int) * (top ? top : 1));
  for (int j = 0; j < top; ++j) {
    ids[j] = j;
    for (size_t n = 0; n < N; ++n) sw[j * N + n] = switch_modulus(last[n], qt, c->primes[j]);
  }
  or_ntt(c, sw, top, ids, 0);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < top; ++j) {
    uint64_t q = c->primes[j];
    uint64_t qinv = or_invmod(qt % q, q);
    uint64_t m = (q - qinv) % q;
    for (size_t n = 0; n < N; ++n)
      out[j * N + n] = addmod(or_mulmod(qinv, x[j * N + n], q), or_mulmod(m, sw[j * N + n], q), q);
  }
  free(last);
  free(sw);
  free(ids);
}

/* HMult + relinearize (+ rescale): reference src/CKKS/Ciphertext.cpp:660-869 (live branch
 * 846-866: binomialMult, foldKeySwitched = keySwitch(d2) then c0 += f0, c1 += f1) and
 * Ciphertext::rescale (:569-607) for FIXEDMANUAL. */
void or_hmult(const or_ctx* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
              const uint64_t* relin_key, int do_rescale, uint64_t* out0, uint64_t* out1) {
  const size_t N = (size_t)c->N;
  uint64_t* d0 = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  uint64_t* d1 = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  uint64_t* d2 = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  uint64_t* f0 = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  uint64_t* f1 = (uint64_t*)malloc(sizeof(uint64_t) * l * N);
  int* ids = (int*)malloc(sizeof(int) * l);
  for (int i = 0; i < l; ++i) ids[i] = i;
  or_tensor(c, a0, a1, b0, b1, l, d0, d1, d2);
  or_keyswitch(c, d2, l, relin_key, f0, f1);
  or_poly_add(c, d0, f0, d0, l, ids);
  or_poly_add(c, d1, f1, d1, l, ids);
  if (do_rescale) {
    or_rescale(c, d0, l, out0);
    or_rescale(c, d1, l, out1);
  } else {
    memcpy(out0, d0, sizeof(uint64_t) * l * N);
    memcpy(out1, d1, sizeof(uint64_t) * l * N);
  }
  free(d0);
  free(d1);
  free(d2);
  free(f0);
  free(f1);
  free(ids);
}

/* One hoisted rotation from precomputed digits: reference hoistedRotateDotKSK_2_
 * (src/CKKS/ElemenwiseBatchKernels.cu:277-377): A = sum D_d a_d, B = P c0 + sum D_d b_d
 * (P c0 on Q limbs only), both scattered by automorph_slot(k); then Ciphertext::modDown
 * (Ciphertext.cpp:466-476) of both: c0' = ModDown(sigma(B)), c1' = ModDown(sigma(A)). */
static void rotate_from_digits(const or_ctx* c, const uint64_t* digits, const uint64_t* c0, int l, const uint64_t* key,
                               uint32_t k, uint64_t* out0, uint64_t* out1) {
  const size_t N = (size_t)c->N;
  const int K = c->n_p, ext = l + K;
  uint64_t* A = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* B = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* As = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* Bs = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  or_ksk_ip(c, digits, l, key, A, B);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < l; ++j) {
    uint64_t q = c->primes[j];
    uint64_t P = 1;
    for (int kk = 0; kk < K; ++kk) P = or_mulmod(P, c->primes[c->n_q + kk] % q, q);
    for (size_t n = 0; n < N; ++n) B[j * N + n] = addmod(B[j * N + n], or_mulmod(c0[j * N + n], P, q), q);
  }
  or_automorph(c, A, As, ext, k);
  or_automorph(c, B, Bs, ext, k);
  or_moddown(c, Bs, l, out0);
  or_moddown(c, As, l, out1);
  free(A);
  free(B);
  free(As);
  free(Bs);
}

/* HRotate: reference src/CKKS/Ciphertext.cpp:1102-1168 (ModUp of c1, one fused hoisted
 * rotation, ModDown). */
void or_rotate_auto(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, const uint64_t* key, uint32_t k,
                    uint64_t* out0, uint64_t* out1) {
  const size_t N = (size_t)c->N;
  const int ext = l + c->n_p, beta = or_num_digits(c, l);
  uint64_t* digits = (uint64_t*)malloc(sizeof(uint64_t) * beta * ext * N);
  or_modup(c, c1, l, digits);
  rotate_from_digits(c, digits, c0, l, key, k, out0, out1);
  free(digits);
}

/* Rotation sum, reference src/CKKS/AccumulateBroadcast.cu:122-160 (Accumulate) over the hoisted
 * rotations left in the extended basis (Ciphertext.cpp:1221-1300 with ext): rounds t = 1, radix,
 * radix^2, ... < size rotate the running value by stride t k (k < radix, stride t k < stride
 * size).  Each rotation's c0 part is automorph(B_k + x0e), x0e the running extended c0 (P c0
 * before the first round), its c1 part automorph(A_k); x0e gains the c0 parts (ModDown once at
 * the end), P c1 + the c1 parts is brought down every round. */
static const uint64_t* key_for(const int* key_rot, const uint64_t* const* keys, int n_keys, int r) {
  for (int i = 0; i < n_keys; ++i)
    if (key_rot[i] == r) return keys[i];
  return NULL;
}

int or_accumulate(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, int radix, int stride, int size,
                  const int* key_rot, const uint64_t* const* keys, int n_keys, uint64_t* out0, uint64_t* out1) {
  const size_t N = (size_t)c->N;
  const int K = c->n_p, ext = l + K, beta = or_num_digits(c, l);
  if (radix < 2 || (radix & (radix - 1)) || stride < 1 || size < 1) return -1;
  for (long t = 1; t < size; t *= radix)  /* every key first: -2 when one is missing */
    for (int k = 1; k < radix && (long)stride * t * k < (long)stride * size; ++k)
      if (!key_for(key_rot, keys, n_keys, (int)(stride * t * k))) return -2;
  memcpy(out0, c0, sizeof(uint64_t) * l * N);
  memcpy(out1, c1, sizeof(uint64_t) * l * N);
  if (size <= 1) return 0;
  uint64_t* pm = (uint64_t*)malloc(sizeof(uint64_t) * ext);
  int* pid = (int*)malloc(sizeof(int) * ext);
  for (int j = 0; j < ext; ++j) {
    pid[j] = j < l ? j : c->n_q + (j - l);
    uint64_t q = c->primes[pid[j]], P = 1;
    for (int k = 0; k < K; ++k) P = or_mulmod(P, c->primes[c->n_q + k] % q, q);
    pm[j] = j < l ? P : 0;
  }
  uint64_t* x0e = (uint64_t*)calloc((size_t)ext * N, sizeof(uint64_t));
  uint64_t* s0 = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* s1 = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* A = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* B = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* As = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* Bs = (uint64_t*)malloc(sizeof(uint64_t) * ext * N);
  uint64_t* digits = (uint64_t*)malloc(sizeof(uint64_t) * beta * ext * N);
  for (int j = 0; j < l; ++j)
    for (size_t n = 0; n < N; ++n) x0e[j * N + n] = or_mulmod(c0[j * N + n], pm[j], c->primes[pid[j]]);
  for (long t = 1; t < size; t *= radix) {
    or_modup(c, out1, l, digits);
    memcpy(s0, x0e, sizeof(uint64_t) * ext * N);
    memset(s1, 0, sizeof(uint64_t) * ext * N);
    for (int j = 0; j < l; ++j)
      for (size_t n = 0; n < N; ++n) s1[j * N + n] = or_mulmod(out1[j * N + n], pm[j], c->primes[pid[j]]);
    for (int k = 1; k < radix && (long)stride * t * k < (long)stride * size; ++k) {
      const int r = (int)(stride * t * k);
      or_ksk_ip(c, digits, l, key_for(key_rot, keys, n_keys, r), A, B);
      for (int j = 0; j < ext; ++j)
        for (size_t n = 0; n < N; ++n) B[j * N + n] = addmod(B[j * N + n], x0e[j * N + n], c->primes[pid[j]]);
      const uint32_t ka = or_rotation_auto_index(c->logN, r);
      or_automorph(c, A, As, ext, ka);
      or_automorph(c, B, Bs, ext, ka);
      for (int j = 0; j < ext; ++j)
        for (size_t n = 0; n < N; ++n) {
          const uint64_t q = c->primes[pid[j]];
          s0[j * N + n] = addmod(s0[j * N + n], Bs[j * N + n], q);
          s1[j * N + n] = addmod(s1[j * N + n], As[j * N + n], q);
        }
    }
    memcpy(x0e, s0, sizeof(uint64_t) * ext * N);
    or_moddown(c, s1, l, out1);
  }
  or_moddown(c, x0e, l, out0);
  free(pm);
  free(pid);
  free(x0e);
  free(s0);
  free(s1);
  free(A);
  free(B);
  free(As);
  free(Bs);
  free(digits);
  return 0;
}

/* Hoisted rotations: reference src/CKKS/Ciphertext.cpp:1221-1394 (one ModUp, one fused
 * KSK/automorph pass over all indices, ModDown per result). */
void or_rotate_hoisted(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, const uint64_t* const* keys,
                       const uint32_t* ks, int n, uint64_t* const* out0, uint64_t* const* out1) {
  const size_t N = (size_t)c->N;
  const int ext = l + c->n_p, beta = or_num_digits(c, l);
  uint64_t* digits = (uint64_t*)malloc(sizeof(uint64_t) * beta * ext * N);
  or_modup(c, c1, l, digits);
  for (int j = 0; j < n; ++j) rotate_from_digits(c, digits, c0, l, keys[j], ks[j], out0[j], out1[j]);
  free(digits);
}
