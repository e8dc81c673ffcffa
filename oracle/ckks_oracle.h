/*
 * ckks_oracle.h -- CPU restatement of the reference's CKKS evaluation arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls this
 * library: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm use it, as the checker.  The GPU library never falls back to it.
 *
 * Every function states the reference file:line it restates.  All arithmetic is
 * exact unsigned integer arithmetic on uint64 residues (primes < 2^62).
 *
 * Layout conventions (identical to the GPU library's C ABI):
 *   - a polynomial is limb-major: limb i is N = 2^logN consecutive uint64 words;
 *   - EVALUATION format is the negacyclic NTT in bit-reversed order (OpenFHE's
 *     "EVALUATION" format, reference test/NTTtests.cu:447-467);
 *   - an extended (Q u P) polynomial at level l has l Q-limbs followed by K P-limbs;
 *   - a key-switching key is [2][dnum][n_q + K][N]: index 0 = "a" (feeds c1),
 *     index 1 = "b" (feeds c0), reference RawCiphertext.cuh:90-95 and
 *     KeySwitchingKey.cu:19-35; digit d, limb i (Q limbs 0..n_q-1, then P limbs).
 */
#ifndef CKKS_ORACLE_H
#define CKKS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- number theory (reference src/Math.cu:8-38, src/ConstantsGPU.cu:39-69) ---- */
uint64_t or_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t or_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t or_invmod(uint64_t a, uint64_t q);
int or_is_prime(uint64_t n);
/* Largest `count` primes q < 2^bits with q = 1 mod 2N, descending, skipping `exclude`. */
int or_gen_primes(int logN, int bits, int count, const uint64_t* exclude, int n_exclude, uint64_t* out);
uint64_t or_generator(uint64_t q);
uint64_t or_root_2n(uint64_t q, int logN);
uint32_t or_bit_reverse(uint32_t x, int bits);

/* ---- context ---- */
typedef struct or_ctx or_ctx;
/* primes: n_q Q-primes then n_p special primes; psi may be NULL (derived by or_root_2n). */
or_ctx* or_ctx_create(int logN, int n_q, int n_p, const uint64_t* primes, const uint64_t* psi, int dnum);
void or_ctx_destroy(or_ctx* c);
int or_ctx_alpha(const or_ctx* c);
uint64_t or_ctx_psi(const or_ctx* c, int prime_id);
/* Reduced-noise ModUp / ModDown conversions (reference Parameters::reducedNoise): off by default. */
void or_ctx_set_reduced_noise(or_ctx* c, int on);
/* Set the number of OpenMP threads the oracle uses (<=0: all). */
void or_set_threads(int n);
int or_get_threads(void);

/* ---- transforms ---- */
/* In-place negacyclic NTT (inverse != 0: INTT incl. N^-1) of n_limbs limbs; limb i uses prime prime_ids[i]. */
void or_ntt(const or_ctx* c, uint64_t* a, int n_limbs, const int* prime_ids, int inverse);

/* ApproxSwitchCRTBasis: coefficient-domain limbs over src primes -> dst primes. */
void or_switch_basis(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out, int n_dst,
                     const int* dst_ids);
/* The same with the reduced-noise lift: sources above q_i / 2 taken as y_i - q_i. */
void or_switch_basis_lift(const or_ctx* c, const uint64_t* in, int n_src, const int* src_ids, uint64_t* out,
                          int n_dst, const int* dst_ids);

/* ---- elementwise ---- */
void or_poly_mul(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids);
void or_poly_add(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids);
void or_poly_sub(const or_ctx* c, const uint64_t* a, const uint64_t* b, uint64_t* out, int n_limbs, const int* prime_ids);
void or_tensor(const or_ctx* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
               uint64_t* d0, uint64_t* d1, uint64_t* d2);
/* Automorphism on EVALUATION-order limbs: out[sigma_k(j)] = in[j] (reference src/Rotation.cuh:14-35). */
void or_automorph(const or_ctx* c, const uint64_t* in, uint64_t* out, int n_limbs, uint32_t k);
/* Automorphism index for a rotation by r slots (reference RNSPoly.cpp:656-658, Context.cu:916-944). */
uint32_t or_rotation_auto_index(int logN, int r);

/* ---- hybrid key switching ---- */
int or_num_digits(const or_ctx* c, int l);
/* ModUp of an EVAL poly at level l -> beta extended digits [beta][l+K][N] in EVAL format. */
void or_modup(const or_ctx* c, const uint64_t* x, int l, uint64_t* digits);
/* KSK inner product over beta digits -> out_a, out_b extended [(l+K)][N]. */
void or_ksk_ip(const or_ctx* c, const uint64_t* digits, int l, const uint64_t* key, uint64_t* out_a, uint64_t* out_b);
/* ModDown of an extended EVAL poly [(l+K)][N] -> [l][N] EVAL. */
void or_moddown(const or_ctx* c, const uint64_t* in_ext, int l, uint64_t* out);
/* Key switch of d (EVAL, level l): f0 = ModDown(sum d_j b_j), f1 = ModDown(sum d_j a_j). */
void or_keyswitch(const or_ctx* c, const uint64_t* d, int l, const uint64_t* key, uint64_t* f0, uint64_t* f1);

/* SwitchModulus of n coefficients from prime src_id to prime dst_id (Rescale.cuh:44-64). */
void or_switch_modulus(const or_ctx* c, const uint64_t* in, int n, int src_id, int dst_id, uint64_t* out);

/* ---- ciphertext ops (level l = number of active Q limbs) ---- */
/* OpenFHE DropLastElementAndScale: out (l-1 limbs). */
void or_rescale(const or_ctx* c, const uint64_t* x, int l, uint64_t* out);
/* HMult + relinearize (+ rescale if do_rescale): out has l (or l-1) limbs. */
void or_hmult(const or_ctx* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
              const uint64_t* relin_key, int do_rescale, uint64_t* out0, uint64_t* out1);
/* Rotation with an automorphism index (fused hoisted form, n = 1). */
void or_rotate_auto(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, const uint64_t* key, uint32_t k,
                    uint64_t* out0, uint64_t* out1);
/* Hoisted rotations: one ModUp of c1, n automorphism indices / keys. */
/* Rotation sum (reference Accumulate): see ckks_oracle.c. */
int or_accumulate(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, int radix, int stride, int size,
                  const int* key_rot, const uint64_t* const* keys, int n_keys, uint64_t* out0, uint64_t* out1);
void or_rotate_hoisted(const or_ctx* c, const uint64_t* c0, const uint64_t* c1, int l, const uint64_t* const* keys,
                       const uint32_t* ks, int n, uint64_t* const* out0, uint64_t* const* out1);

#ifdef __cplusplus
}
#endif
#endif
