/*
 * fides_b200.h -- C ABI of the B200-native CKKS evaluation core (libfides_b200.so).
 *
 * Plain pointers and sizes only.  Polynomials are limb-major uint64 arrays: limb i is
 * N = 2^logN consecutive words.  Unless a function says "host", every polynomial or
 * key pointer is DEVICE memory on the context's GPU.  Data are in EVALUATION format
 * (negacyclic NTT, bit-reversed order) unless stated otherwise -- the same layout as the
 * reference's RawCipherText limbs (src/CKKS/openfhe-interface/RawCiphertext.cuh:21-37).
 *
 * "level" l = number of active Q limbs of a ciphertext (1 <= l <= n_q).  An extended
 * polynomial at level l has l Q limbs followed by the K special limbs.
 *
 * Key-switching keys are [2][dnum][n_q + K][N] (index 0 = a, feeds c1; index 1 = b,
 * feeds c0), the layout of the reference's RawKeySwitchKey::r_key
 * (RawCiphertext.cuh:90-95, KeySwitchingKey.cu:19-35).
 *
 * Every call returns FIDES_OK (0) or a negative status; fides_last_error() returns the
 * calling thread's message.  `stream` is a cudaStream_t (NULL = legacy default stream).
 * Calls enqueue work and return without synchronising unless stated otherwise.
 */
#ifndef FIDES_B200_H
#define FIDES_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FIDES_OK 0
#define FIDES_ERR_ARG (-1)     /* bad argument (null pointer, size, level) */
#define FIDES_ERR_CUDA (-2)    /* a CUDA runtime call failed */
#define FIDES_ERR_OOM (-3)     /* device allocation failed / over budget */
#define FIDES_ERR_LEVEL (-4)   /* level out of range for the operation */
#define FIDES_ERR_KEY (-5)     /* missing or malformed key */
#define FIDES_ERR_TIMEOUT (-6) /* a bounded device-side wait gave up */
#define FIDES_ERR_STATE (-7)   /* object in the wrong state */

/* Parameters.  Replaces FIDESlib::CKKS::Parameters (src/CKKS/Parameters.cuh:20-129) and
 * the RawParams moduli/roots (RawCiphertext.cuh:53-66).  psi[i] = primitive 2N-th root of
 * primes[i]; NULL (or a zero entry) derives it as g^((q-1)/2N), g the smallest primitive
 * root (reference src/ConstantsGPU.cu:39-69). */
typedef struct fides_params {
  int logN;
  int n_q;       /* L + 1 */
  int n_special; /* K */
  int dnum;
  const uint64_t* primes; /* n_q Q primes then K special primes, each < 2^62 */
  const uint64_t* psi;    /* optional */
  int device;             /* CUDA device ordinal */
} fides_params;

typedef struct fides_ctx fides_ctx;

/* Context: replaces GenCryptoContextGPU + ContextData (src/CKKS/Context.cu:74-138) and
 * SetupConstants (src/ConstantsGPU.cu:132-640). */
int fides_ctx_create(const fides_params* params, fides_ctx** out);
int fides_ctx_destroy(fides_ctx* ctx);
const char* fides_last_error(void);
int fides_ctx_psi(const fides_ctx* ctx, uint64_t* psi_out); /* n_q + K roots */
int fides_ctx_alpha(const fides_ctx* ctx);
/* Bytes of device scratch the context currently holds. */
size_t fides_ctx_scratch_bytes(const fides_ctx* ctx);
/* Cap on scratch growth (0 = unlimited); exceeding it returns FIDES_ERR_OOM. */
int fides_ctx_set_scratch_limit(fides_ctx* ctx, size_t bytes);
/* Grows the device scratch pool to hold at least `bytes` once, up front (the pool keeps
 * freed memory), so that later operations never map new memory on their launch path.
 * fides_server_create calls it with the server's worst case. */
int fides_ctx_reserve_scratch(fides_ctx* ctx, size_t bytes);
/* Count of kernels this context has launched (for launch accounting). */
uint64_t fides_ctx_launch_count(const fides_ctx* ctx);

/* Basis-conversion engine (ModUp / ModDown): 0 = automatic, 1 = 64-bit SIMT, 2 = tensor cores
 * (exact INT8-split product on tcgen05, for conversions of at most 16 source limbs whose byte
 * matrix fits in shared memory; wider ones stay on SIMT).  Results are identical. No reference
 * counterpart: the reference has one conversion kernel family (src/Conv.cu:27-423). */
int fides_ctx_set_conv_engine(fides_ctx* ctx, int engine);
/* Reduced-noise basis conversion (reference Parameters::reducedNoise, src/CKKS/Parameters.cuh:31,
 * read as C_.reduced_noise by ModDown2 / DecompAndModUpConv, src/CKKS/Conv.cu:76-87 and
 * :356-381; ReducedNoise.cuh:14-16; tables as src/ReducedNoiseConstants.cu).  With on = 1 every
 * ModUp and ModDown conversion reads each pre-scaled source residue y_i above q_i / 2 as
 * y_i - q_i: the converted value gains cnt * [-Q_src]_{p_j}, cnt the number of such sources,
 * which removes the conversion's q-overflow term for those coefficients (OpenFHE's
 * WITH_REDUCED_NOISE build).  Off (0) by default, as in the reference.  Applies to operations
 * launched after the call (a CUDA graph keeps the tables it was captured with). */
int fides_ctx_set_reduced_noise(fides_ctx* ctx, int on);
/* NTT tile-shape autotuner.  Each NTT pass groups 4, 8 or 16 sub-transforms per CTA; the
 * context keeps one choice per direction (0 forward, 1 inverse), pass (0 column, 1 row) and
 * launch-size class (limbs per launch <= 8, <= 32, <= 128, more).  fides_ctx_autotune times
 * every shape (and residues per thread, below) on the device from CUDA-graph replays (under a
 * second at N = 2^16) and keeps the fastest; best_ms
 * (optional, 8 floats [inverse][class]) receives one transform's time of each class's
 * representative launch (4, 16, 64, 256 limbs).  Results never depend on the shapes.  Do
 * not run it concurrently with other work on the context.  No reference counterpart: the
 * reference fixes its NTT launch geometry (src/CKKS/LimbPartition.cu:444-472). */
int fides_ctx_autotune(fides_ctx* ctx, float* best_ms);
/* Limbs per NTT launch pair: longer limb lists run as balanced chunks of at most this many
 * limbs, each chunk's two passes back to back, so that a chunk small enough for L2 has its
 * between-pass intermediate served from L2.  set_limbs > 0 sets it, 0 restores the largest
 * launch, < 0 only reads; returns the current value (or a negative status).  fides_ctx_autotune
 * picks it by timing. */
int fides_ctx_ntt_chunk(fides_ctx* ctx, int set_limbs);
/* The 16 shape entries, index [inverse][pass][size class]. */
int fides_ctx_ntt_shapes(fides_ctx* ctx, uint8_t* shapes);
int fides_ctx_set_ntt_shape(fides_ctx* ctx, int inverse, int pass, int size_class, int subs_per_cta);
/* Residues per thread of each pass (16, or 8 = three butterfly stages per register chunk and
 * twice the threads, built for N >= 2^15), in the same [inverse][pass][size class] layout;
 * fides_ctx_autotune times both with every shape.  Results never depend on them.  The
 * reference's counterpart is its fixed per-thread radix (src/NTT.cu:331-756). */
int fides_ctx_ntt_residues(fides_ctx* ctx, uint8_t* residues);
int fides_ctx_set_ntt_residues(fides_ctx* ctx, int inverse, int pass, int size_class, int residues_per_thread);
/* Compute roofline of the NTT: butterflies per second that `device` sustains running the
 * forward NTT butterfly (one 64-bit Shoup product, two 64-bit additions) on register-resident
 * data, with no memory traffic.  Takes about 100 ms.  No reference counterpart. */
int fides_int_peak(int device, double* butterflies_per_s);
/* The same for the FP64 butterfly the NTT uses for primes below 2^50 (its FP64-pipe
 * roofline).  No reference counterpart. */
int fides_f64_peak(int device, double* butterflies_per_s);
/* The architecture the runtime loaded the library's kernels for on `device`, as
 * cudaFuncAttributes::binaryVersion (100 = sm_100a code).  No reference counterpart. */
int fides_kernel_arch(int device, int* binary_version);
/* Limb transforms submitted to the NTT since the context was created, by butterfly form:
 * FP64 (primes below 2^50) and 64-bit integer.  No reference counterpart. */
int fides_ctx_ntt_counts(fides_ctx* ctx, uint64_t* f64_limbs, uint64_t* int_limbs);
/* Synchronises the device and reads the context's device status word: bit 0 = a bounded
 * device-side wait gave up (the affected outputs are incomplete), bit 1 = an encoded
 * coefficient exceeded 2^62 in magnitude.  clear != 0 resets it.  Every call that synchronises with
 * the device on the caller's behalf (fides_ctx_synchronize, the host-buffer entry points,
 * fides_ct_export) returns FIDES_ERR_TIMEOUT while bit 0 is set, until it is cleared here.
 * Counterpart of the reference's CudaCheckErrorMod after a synchronisation
 * (src/CudaUtils.cuh:706-757), for waits that give up instead of hanging. */
int fides_ctx_device_status(fides_ctx* ctx, uint32_t* status, int clear);
/* Synchronises `stream` and checks the device status word (FIDES_ERR_TIMEOUT as above). */
int fides_ctx_synchronize(fides_ctx* ctx, void* stream);
/* Host-side fault injection for tests of the failure path: synchronises the device and ORs
 * `bits` into the device status word, as a kernel whose bounded wait gave up would.  No
 * reference counterpart (the reference has no bounded device waits). */
int fides_ctx_inject_status(fides_ctx* ctx, uint32_t bits);

/* Profiling mode: when enabled, every kernel launch is bracketed by CUDA events on its
 * stream and attributed to a family (0 = NTT passes, 1 = basis conversion, 2 = KSK inner
 * product, 3 = other elementwise).  fides_ctx_profile_read synchronises on the recorded
 * events and returns, for one family, the summed device time, the summed algorithmic
 * bytes (compulsory HBM traffic of each launch) and the launch count, then clears that
 * family's records.  Counterpart of the reference's NVTX ranges (src/CudaUtils.cuh:662-690). */
int fides_ctx_profile(fides_ctx* ctx, int enable);
int fides_ctx_profile_read(fides_ctx* ctx, int kind, double* ms, double* bytes, uint64_t* launches);

/* ---- transforms --------------------------------------------------------------------- */
/* Batched NTT / INTT over an arbitrary list of limbs (each limb: device pointer + prime
 * index into params.primes).  Replaces NTT_/INTT_/NTTBatch_ + ApplyNTT/ApplyINTT
 * (src/NTT.cu:42-802, src/CKKS/LimbPartition.cu:433-550).  In place. */
int fides_ntt_limbs(fides_ctx* ctx, uint64_t* const* limbs, const int* prime_ids, int n_limbs, int inverse,
                    void* stream);
/* n_polys contiguous polynomials of n_limbs Q limbs each (prime ids 0..n_limbs-1). */
int fides_ntt_polys(fides_ctx* ctx, uint64_t* data, int n_polys, int n_limbs, int inverse, void* stream);

/* ---- hybrid key-switching pieces ---------------------------------------------------- */
/* ModUp of an EVAL poly at level l into beta extended digits [beta][l+K][N] (own-digit
 * limbs are copied through).  Replaces RNSPoly::modup / LimbPartition::modupMGPU
 * (src/CKKS/LimbPartitionMGPU.cu:1981+) with DecompAndModUpConv (src/CKKS/Conv.cu:274-423). */
int fides_modup(fides_ctx* ctx, const uint64_t* x, int level, uint64_t* digits, void* stream);
/* KSK inner product over the digits: replaces fusedDotKSK_2_
 * (src/CKKS/ElemenwiseBatchKernels.cu:202-274).  out_a/out_b are [l+K][N]. */
int fides_ksk_inner_product(fides_ctx* ctx, const uint64_t* digits, int level, const uint64_t* key,
                            uint64_t* out_a, uint64_t* out_b, void* stream);
/* ModDown [l+K][N] -> [l][N]: replaces LimbPartition::moddown (src/CKKS/LimbPartition.cu:
 * 2145-2217) with ModDown2 (src/CKKS/Conv.cu:27-133) and NTT_MODDOWN (NTTfusions.cuh:237). */
int fides_moddown(fides_ctx* ctx, const uint64_t* x_ext, int level, uint64_t* out, void* stream);
/* Full key switch of d: f0 = ModDown(sum d_j b_j), f1 = ModDown(sum d_j a_j).  Replaces
 * LimbPartition::modup_ksk_moddown_mgpu (src/CKKS/LimbPartitionMGPU.cu:669-1980). */
int fides_keyswitch(fides_ctx* ctx, const uint64_t* d, int level, const uint64_t* key, uint64_t* f0,
                    uint64_t* f1, void* stream);

/* ---- ciphertext operations (device buffers) ----------------------------------------- */
/* Tensor product: replaces binomialMult_ (ElemenwiseBatchKernels.cu:1363-1510). */
int fides_tensor(fides_ctx* ctx, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1,
                 int level, uint64_t* d0, uint64_t* d1, uint64_t* d2, void* stream);
/* Elementwise RNS add / sub of two polynomials of `level` Q limbs (out may alias an input):
 * replaces add_ / sub_ (src/AddSub.cu:10-123) behind Ciphertext::add / sub
 * (src/CKKS/Ciphertext.cpp:244-330). */
int fides_add(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream);
int fides_sub(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream);
/* Elementwise product of two polynomials (ciphertext component x plaintext, EVAL):
 * replaces Mult_ / multPt (ElemenwiseBatchKernels.cu:83-120, Ciphertext::multPt). */
int fides_mul(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream);
/* Per-limb scalar multiply / add (host array of `level` residues, reduced mod q_i): replaces
 * Scalar_mult_ / scalar_add_ (ElemenwiseBatchKernels.cu, AddSub.cu) behind multScalar /
 * addScalar.  At most 64 limbs. */
int fides_mul_scalar(fides_ctx* ctx, const uint64_t* a, int level, const uint64_t* scalars, uint64_t* out,
                     void* stream);
int fides_add_scalar(fides_ctx* ctx, const uint64_t* a, int level, const uint64_t* scalars, uint64_t* out,
                     void* stream);
/* Plaintext-ciphertext inner product of a linear transform's giant step:
 * out0 = sum_t pts[t] * c0s[t], out1 = sum_t pts[t] * c1s[t] (EVAL, mod q, level limbs),
 * 1 <= n_terms <= 32, one launch (LTdotProductPtBatch, LimbPartitionBatch.cu:266). */
int fides_dot_plain(fides_ctx* ctx, const uint64_t* const* c0s, const uint64_t* const* c1s,
                    const uint64_t* const* pts, int n_terms, int level, uint64_t* out0, uint64_t* out1,
                    void* stream);
/* Every giant step's inner product of a BSGS linear transform in one launch (the reference's
 * DotProductPtInternal over all giant steps, LinearTransform.cu:148): out0s[i] / out1s[i] =
 * sum_k pts[i n_baby + k] * (x0s[k], x1s[k]) for giant steps i < n_giant (1..16) over the baby
 * steps k < n_baby (1..16); a null pts entry is no term (a row of nulls gives zero).  ext != 0:
 * operands and results over Q.P ([level + K][N]), as fides_dot_plain_ext. */
int fides_dot_plain_bsgs(fides_ctx* ctx, const uint64_t* const* x0s, const uint64_t* const* x1s, int n_baby,
                         const uint64_t* const* pts, int n_giant, int level, int ext, uint64_t* const* out0s,
                         uint64_t* const* out1s, void* stream);
/* out = a + b over extended-basis polynomials ([level + K][N]: the level Q limbs, then the K
 * special limbs); Ciphertext::add of two operands still in Q.P (LinearTransform.cu:168-173). */
int fides_add_ext(fides_ctx* ctx, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream);
/* The same over extended-basis operands (level Q limbs followed by the K special limbs): the
 * inner product of hoisted rotations kept in Q.P (fides_rotate_hoisted_ext) with diagonals
 * encoded over Q.P (fides_encode_ext); one ModDown (fides_moddown) per result then replaces one
 * per rotation (the reference's LinearTransformInPlace with ext = true). */
int fides_dot_plain_ext(fides_ctx* ctx, const uint64_t* const* c0s, const uint64_t* const* c1s,
                        const uint64_t* const* pts, int n_terms, int level, uint64_t* out0, uint64_t* out1,
                        void* stream);
/* Ciphertext linear combination with integer constants (EVAL, level limbs), over n_lanes
 * independent operand sets that share the constants:
 *   out0s[a] = sum_t s_t * c0s[a * n_terms + t] + add0,  out1s[a] = sum_t s_t * c1s[a * n_terms + t]
 * where scalars holds n_terms x level residues (row t = s_t mod q_0..q_(level-1)) and add0
 * level residues (or NULL).  1 <= n_terms <= 16, 1 <= n_lanes <= 8, level <= 64; one launch.
 * The scalar steps of the Chebyshev series evaluation (evalPartialLinearWSum,
 * src/CKKS/ApproxModEval.cu:328; multConst / addConst per term in the reference). */
int fides_lincomb(fides_ctx* ctx, int n_lanes, const uint64_t* const* c0s, const uint64_t* const* c1s,
                  const uint64_t* scalars, const uint64_t* add0, int n_terms, int level, uint64_t* const* out0s,
                  uint64_t* const* out1s, void* stream);
/* Rescale of n polynomials, polynomial i at levels[i] limbs -> levels[i] - 1 limbs, in one
 * launch sequence (a batched fides_rescale; Ciphertext::rescale per ciphertext in the
 * reference, src/CKKS/Ciphertext.cpp:569-607).  An output may not overlap another input. */
int fides_rescale_batch(fides_ctx* ctx, const uint64_t* const* xs, const int* levels, uint64_t* const* outs, int n,
                        void* stream);
/* CKKS slot encode on the device (replaces Plaintext::loadSlotsBatch / EncodeChunkSlots,
 * src/CKKS/DeviceEncodeBatch.cu:529-828, and the host CKKSPackedEncoding::Encode it mirrors):
 * n_pts plaintexts of n_slots complex slots each (slots = [n_pts][n_slots][re, im] doubles in
 * device memory; n_slots a power of two <= N/2) are multiplied by `scale`, mapped to
 * coefficients by the inverse special FFT (coefficient gap N / (2 n_slots)), rounded to the
 * nearest integer and written as `level` limbs in EVALUATION form, out = [n_pts][level][N].
 * Each limb reduces the signed integer coefficient modulo its own prime, so a coefficient may
 * exceed q_0; every coefficient must stay below 2^62 in magnitude, a larger one is written as 0
 * and sets bit 1 of the device status word (fides_ctx_device_status). */
int fides_encode(fides_ctx* ctx, const double* slots, int n_slots, int n_pts, double scale, int level, uint64_t* out,
                 void* stream);
/* fides_encode over the extended basis (the reference's MakeCKKSPackedPlaintextExtended,
 * api/CryptoContext.hpp:171): out = [n_pts][level + K][N], the level Q limbs followed by the K
 * special limbs of the same integer polynomial. */
int fides_encode_ext(fides_ctx* ctx, const double* slots, int n_slots, int n_pts, double scale, int level,
                     uint64_t* out, void* stream);
/* CKKS slot decode on the device: n_pts plaintexts [n_pts][level][N] in EVALUATION form ->
 * n_slots complex slots each divided by `scale` (slots = [n_pts][n_slots][re, im] doubles in
 * device memory).  Reads limb 0 only, so the coefficients must lie below q_0 / 2 in magnitude
 * (a decrypted message at a scale well below q_0). */
int fides_decode(fides_ctx* ctx, const uint64_t* pts, int level, int n_pts, int n_slots, double scale, double* slots,
                 void* stream);
/* ModRaise of one level-1 polynomial (limb q_0, EVAL) to out_level limbs: INTT, centred
 * SwitchModulus(q_0 -> q_j), NTT (reference Bootstrap.cu ModRaise, src/CKKS/Bootstrap.cu:708+). */
int fides_mod_raise(fides_ctx* ctx, const uint64_t* x, int out_level, uint64_t* out, void* stream);
/* Rescale of n_polys polynomials at level l (FIXEDMANUAL DropLastElementAndScale);
 * out has l-1 limbs per poly.  Replaces Ciphertext::rescale (src/CKKS/Ciphertext.cpp:
 * 569-607) / LimbPartition::rescale (src/CKKS/LimbPartition.cu:711-797). */
int fides_rescale(fides_ctx* ctx, const uint64_t* x, int level, uint64_t* out, void* stream);
/* HMult + relinearize (+ rescale): replaces CKKS::Ciphertext::mult
 * (src/CKKS/Ciphertext.cpp:660-869) behind CudaEngine::evalMult (CudaEngine.cpp:429-437). */
int fides_hmult(fides_ctx* ctx, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1,
                int level, const uint64_t* relin_key, int rescale, uint64_t* out0, uint64_t* out1, void* stream);
/* HRotate by `rotation` slots: replaces CKKS::Ciphertext::rotate (Ciphertext.cpp:1102-1168)
 * behind CudaEngine::evalRotate (CudaEngine.cpp:527-533). */
int fides_rotate(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level, const uint64_t* rot_key,
                 int rotation, uint64_t* out0, uint64_t* out1, void* stream);
/* Same with an explicit automorphism index (2N-1 = conjugation, Ciphertext.cpp:1175-1219). */
int fides_rotate_auto(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level, const uint64_t* key,
                      uint32_t auto_index, uint64_t* out0, uint64_t* out1, void* stream);
/* Hoisted rotations (one ModUp, n rotations): replaces Ciphertext::rotate_hoisted
 * (Ciphertext.cpp:1221-1394) / EvalFastRotation (CudaEngine.cpp:536-585). */
int fides_rotate_hoisted(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level,
                         const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                         uint64_t* const* out1, void* stream);
/* Hoisted rotations left in the extended basis (Ciphertext::rotate_hoisted with ext = true,
 * Ciphertext.cpp:1221-1300): out0[j] / out1[j] = [level + K][N], P times rotation j of (c0, c1)
 * up to the ModDown rounding (the key-switch outputs with P c0 added, automorphism applied, no
 * ModDown); fides_moddown of each gives fides_rotate_hoisted's results.  c0_ext != 0: c0 is
 * already extended ([level + K][N]) and is added as it is instead of P c0 -- a rotation without
 * ModDown of a ciphertext whose c0 stayed in Q.P (Ciphertext::rotate(r, false) after
 * c1.moddown, the giant-step fold of LinearTransform, LinearTransform.cu:164-195). */
int fides_rotate_hoisted_ext(fides_ctx* ctx, const uint64_t* c0, int c0_ext, const uint64_t* c1, int level,
                             const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                             uint64_t* const* out1, void* stream);
/* Rotation sum (replaces Accumulate, src/CKKS/AccumulateBroadcast.cu:122-160, behind
 * CryptoContext::AccumulateSum, api/CryptoContext.hpp:456): x + sum of its rotations by
 * stride t k for rounds t = 1, radix, radix^2, ... < size and k = 1 .. radix - 1 (while
 * stride t k < stride size), i.e. slot i gathers slots i + j stride, j < size.  Each round's
 * rotations are hoisted and summed in the extended basis; as in the reference, c0 stays there
 * until one ModDown at the end and c1 is brought back every round.  radix: a power of two >= 2
 * (the reference's PARTIAL_SUM_RADIX, 4 by default); keys: one device rotation key per index of
 * fides_accumulate_rotations, key_rotations[i] naming the rotation of keys[i].  out0 / out1 may
 * alias c0 / c1. */
int fides_accumulate(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level, int radix, int stride,
                     int size, const int* key_rotations, const uint64_t* const* keys, int n_keys, uint64_t* out0,
                     uint64_t* out1, void* stream);
/* The rotation indices fides_accumulate needs (reference GetAccumulateRotationIndices): writes up
 * to cap of them and returns their count (negative status for bad arguments). */
int fides_accumulate_rotations(int radix, int stride, int size, int* indices, int cap);
/* Hoisted rotations from a ModUp computed earlier: digits = fides_modup(c1) ([beta][level+K][N]),
 * reused for any number of calls.  The reference's EvalFastRotationPrecompute (the ModUp) and
 * EvalFastRotation (KSK with P c0, automorphism, ModDown), CudaEngine.cpp:536-585 over
 * hoistedRotateDotKSK_2_ (ElemenwiseBatchKernels.cu:277-377).  Results equal fides_rotate. */
int fides_rotate_hoisted_digits(fides_ctx* ctx, const uint64_t* c0, const uint64_t* digits, int level,
                                const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                                uint64_t* const* out1, void* stream);
/* Hoisted rotations of a batch of ciphertexts at any levels, each with its own rotation
 * list: one ModUp launch sequence over all c1, one KSK pass over every (ciphertext,
 * rotation) pair, one ModDown over every output.  Replaces fusedHoistedRotateBatch /
 * hoistedRotateDotKSKBatched (LimbPartitionBatch.cu:526+, ElemenwiseBatchKernels.cu:379-634),
 * which require equal levels.  Item k's outputs j are out0[j] / out1[j] of that item. */
typedef struct {
  const uint64_t *c0, *c1;     /* [level][N] each */
  int level;
  int n;                       /* rotations of this ciphertext */
  const uint64_t* const* keys; /* [n] device keys */
  const int* rotations;        /* [n] */
  uint64_t* const* out0;       /* [n] outputs, [level][N] each */
  uint64_t* const* out1;
} fides_hoist_item;
int fides_rotate_hoisted_batch(fides_ctx* ctx, const fides_hoist_item* items, int n_items, void* stream);
/* Rotation index -> automorphism index (Context.cu:916-944 + RNSPoly.cpp:656-658). */
uint32_t fides_rotation_auto_index(int logN, int rotation);

/* ---- batched forms: many ciphertexts at uneven levels per launch -------------------- */
/* Replaces the reference's same-level batches (LimbPartitionBatch.cu:526+,
 * CudaEngine::evalRotateMany, CudaEngine.cpp:656-702) with mixed-level batching. */
typedef struct fides_hmult_item {
  const uint64_t *a0, *a1, *b0, *b1;
  uint64_t *out0, *out1;
  int level;
} fides_hmult_item;
int fides_hmult_batch(fides_ctx* ctx, const fides_hmult_item* items, int n, const uint64_t* relin_key,
                      int rescale, void* stream);

typedef struct fides_rotate_item {
  const uint64_t *c0, *c1;
  uint64_t *out0, *out1;
  const uint64_t* key;
  int level;
  uint32_t auto_index;
} fides_rotate_item;
int fides_rotate_batch(fides_ctx* ctx, const fides_rotate_item* items, int n, void* stream);
/* HMults and rotations in one launch sequence: the stages common to both kinds (the ModUp's
 * conversion and NTT, the KSK inner product, the ModDown's special-limb INTT and conversion) run
 * once over all items, so small stages are launched once instead of twice.  Results equal
 * fides_hmult_batch / fides_rotate_batch item for item.  No reference counterpart (the
 * reference issues each operation kind separately). */
int fides_mixed_batch(fides_ctx* ctx, const fides_hmult_item* hm, int n_hm, const uint64_t* relin_key, int rescale,
                      const fides_rotate_item* rot, int n_rot, void* stream);

/* ---- CUDA graphs ----------------------------------------------------------------------
 * Record everything the library enqueues on `stream` between begin and end into a graph
 * that replays it with one launch (the reference's run_in_graph, src/CudaUtils.cu:953-979,
 * and its optional capture of the key-switch body, LimbPartitionMGPU.cu:811-892).  Scratch
 * taken during capture becomes graph-owned memory, so a replay needs no allocation calls.
 * Pointers and values passed to the captured calls are frozen into the graph. */
typedef struct fides_graph fides_graph;
int fides_capture_begin(fides_ctx* ctx, void* stream);
int fides_capture_end(fides_ctx* ctx, void* stream, fides_graph** out);
int fides_graph_launch(fides_graph* g, void* stream);
int fides_graph_destroy(fides_graph* g);

/* ---- serving: continuous batching over resident keys -------------------------------
 * A scheduler thread admits submitted requests by HBM budget into batches (one operation
 * type per batch, any mix of levels) and runs each batch as one batched launch sequence on
 * one of n_streams streams, so batches admitted while others run overlap on the device.
 * Replaces the reference's concurrent-ops lanes (api/ConcurrentOps.hpp:30-64) and
 * CudaEngine::evalRotateMany batching (CudaEngine.cpp:656-702).  Request buffers are
 * device memory owned by the caller and must stay valid until fides_server_wait returns. */
#define FIDES_OP_HMULT 0           /* HMult + relinearize + rescale: out has level - 1 limbs */
#define FIDES_OP_HMULT_NORESCALE 1 /* HMult + relinearize: out has level limbs */
#define FIDES_OP_ROTATE 2          /* HRotate by `rotation`: out has level limbs */
#define FIDES_OP_BOOTSTRAP 3       /* bootstrap through a registered engine (below): the input
                                    * has the engine's in_level limbs, out its out_level limbs */

typedef struct fides_server fides_server;
typedef struct fides_server_config {
  int n_streams;           /* batches in flight at once (1..16) */
  int max_batch;           /* requests per batch */
  size_t hbm_budget_bytes; /* scratch the in-flight batches may hold (0 = unlimited) */
} fides_server_config;
typedef struct fides_request {
  int op;
  int level;
  const uint64_t *c0, *c1; /* first operand */
  const uint64_t *d0, *d1; /* second operand (HMult) */
  uint64_t *out0, *out1;
  int rotation; /* FIDES_OP_ROTATE */
} fides_request;
typedef struct fides_server_stats {
  uint64_t submitted, completed, rejected, batches, batched_requests, peak_bytes;
} fides_server_stats;

int fides_server_create(fides_ctx* ctx, const fides_server_config* cfg, fides_server** out);
int fides_server_set_relin_key(fides_server* s, const uint64_t* relin_key_dev);
int fides_server_add_rotation_key(fides_server* s, int rotation, const uint64_t* rot_key_dev);
/* Registers one bootstrap engine: an instantiated CUDA graph (cudaGraphExec_t) that
 * bootstraps the ciphertext held in the static device buffers (in0, in1: in_level limbs
 * each) into (out0, out1: out_level limbs each), with every key and intermediate it needs
 * resident.  A FIDES_OP_BOOTSTRAP request copies its input into the static input, launches
 * the graph and copies the static output to its own output, all on the engine's stream,
 * so it overlaps the HMult / HRotate batches; each engine runs one request at a time and
 * several engines run concurrently.  The graph and buffers must outlive the server.  No
 * reference counterpart (the reference has no request loop). */
int fides_server_add_bootstrap(fides_server* s, void* graph_exec, const uint64_t* in0, const uint64_t* in1,
                               int in_level, const uint64_t* out0, const uint64_t* out1, int out_level);
/* A bootstrap engine that holds `capacity` ciphertexts: the graph bootstraps in0[k], in1[k] into
 * out0[k], out1[k] for every k (e.g. one graph with a parallel branch per ciphertext).  The
 * scheduler fills it with up to `capacity` queued bootstrap requests in one launch, preferring
 * the largest idle engine the queue fills.  fides_server_add_bootstrap is capacity 1.  No
 * reference counterpart. */
int fides_server_add_bootstrap_batch(fides_server* s, void* graph_exec, int capacity, const uint64_t* const* in0,
                                     const uint64_t* const* in1, int in_level, const uint64_t* const* out0,
                                     const uint64_t* const* out1, int out_level);
/* At most this many batches of one operation type on the device at once (0 = no limit beyond
 * n_streams, the default).  With 1, requests that arrive while their type's batch runs form the
 * next batch together (batches grow under load), and a type with nothing in flight starts at
 * once.  No reference counterpart. */
int fides_server_set_max_inflight(fides_server* s, int max_inflight_per_op);
/* Thread-safe, non-blocking; rejects malformed requests and missing keys immediately. */
int fides_server_submit(fides_server* s, const fides_request* req, uint64_t* ticket);
/* Blocks until the request completed; *status is its result (FIDES_ERR_OOM when it can
 * never fit the budget), *latency_ms the time from submit to completion. */
int fides_server_wait(fides_server* s, uint64_t ticket, double* latency_ms, int* status);
/* fides_server_wait with a limit: FIDES_ERR_TIMEOUT when the request has not completed within
 * timeout_ms (the ticket stays valid and can be waited for again); a negative timeout waits
 * without limit.  The reference's callers block on stream synchronisation instead. */
int fides_server_wait_timeout(fides_server* s, uint64_t ticket, double timeout_ms, double* latency_ms, int* status);
int fides_server_get_stats(fides_server* s, fides_server_stats* out);
/* Completes in-flight batches, fails requests never started (FIDES_ERR_STATE), frees. */
int fides_server_destroy(fides_server* s);

/* ---- host-buffer entry points (end-to-end path) ------------------------------------- */
/* Upload a key ([2][dnum][n_q + K][N]) into a new device buffer owned by the context; host_key
 * may be host memory or another device buffer on the same GPU (copied either way). */
int fides_key_upload(fides_ctx* ctx, const uint64_t* host_key, uint64_t** dev_key);
/* Interop with the reference's raw host formats (src/CKKS/openfhe-interface/RawCiphertext.cuh:
 * RawCipherText :20-37, RawKeySwitchKey :90-95), replacing Ciphertext::load / store
 * (src/CKKS/Ciphertext.cpp:415-464) and KeySwitchingKey::Initialize (KeySwitchingKey.cu:19-35).
 * limbs: one host array of N residues per limb, [n_polys][level] pointers (sub_0[i].data(),
 * sub_1[i].data(), ... ); moduli (NULL: not checked) must equal the context's primes;
 * format 0 = EVALUATION, 1 = COEFFICIENT (converted by the NTT on import, the INTT on export);
 * natural_order != 0: evaluation vectors in natural order instead of OpenFHE's bit-reversed
 * order (the reference's REV = 0), permuted on the device.  out / in = [n_polys][level][N] device
 * limbs in this library's bit-reversed EVALUATION layout.  Export returns after the copies. */
int fides_ct_import(fides_ctx* ctx, int n_polys, const uint64_t* const* limbs, const uint64_t* moduli, int level,
                    int format, int natural_order, uint64_t* out, void* stream);
int fides_ct_export(fides_ctx* ctx, int n_polys, const uint64_t* in, int level, int format, int natural_order,
                    uint64_t* const* limbs, void* stream);
/* RawKeySwitchKey::r_key -> a device key (as fides_key_upload): limbs = [2][dnum][n_q + K] host
 * pointers (a = [0], b = [1]; NULL = a zero limb), EVALUATION form. */
int fides_key_import(fides_ctx* ctx, const uint64_t* const* limbs, int natural_order, uint64_t** dev_key);
int fides_key_free(fides_ctx* ctx, uint64_t* dev_key);
/* HMult(+rescale) of host ciphertexts: copies in, computes, copies out, synchronises.
 * Mirrors CudaEngine::evalMult's load -> op -> RecoverHostCiphertext cycle
 * (CudaEngine.cpp:429-437, 1156-1227, 1768-1795). */
int fides_hmult_host(fides_ctx* ctx, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
                     const uint64_t* b1, int level, const uint64_t* relin_key_dev, int rescale, uint64_t* out0,
                     uint64_t* out1);
int fides_rotate_host(fides_ctx* ctx, const uint64_t* c0, const uint64_t* c1, int level,
                      const uint64_t* rot_key_dev, int rotation, uint64_t* out0, uint64_t* out1);
/* Pipelined host batches: n independent ops on host buffers.  Item k's host->device copies,
 * its computation and its device->host copies run on three streams ordered by events, so
 * the copies of neighbouring items overlap item k's kernels (pin the host buffers for the
 * copies to be asynchronous).  Returns when every output has arrived in host memory.
 * Results equal fides_hmult_host / fides_rotate_host item by item.  No reference
 * counterpart: CudaEngine loads, computes and recovers one ciphertext at a time
 * (CudaEngine.cpp:1156-1227). */
typedef struct {
  const uint64_t *a0, *a1, *b0, *b1; /* [level][N] each */
  uint64_t *out0, *out1;             /* [level - 1][N] with rescale, else [level][N] */
  int level;
} fides_hmult_host_item;
int fides_hmult_host_batch(fides_ctx* ctx, const fides_hmult_host_item* items, int n,
                           const uint64_t* relin_key_dev, int rescale);
typedef struct {
  const uint64_t *c0, *c1; /* [level][N] each */
  uint64_t *out0, *out1;   /* [level][N] each */
  const uint64_t* rot_key_dev;
  int level;
  int rotation;
} fides_rotate_host_item;
int fides_rotate_host_batch(fides_ctx* ctx, const fides_rotate_host_item* items, int n);
/* Both kinds in one pipeline, alternated (a rotation item, an HMult item, ...): one fill and
 * drain of the pipeline instead of two, and the copy directions stay balanced (an HMult moves
 * twice a rotation's host->device bytes for the same device->host bytes).  Results equal
 * fides_hmult_host_batch / fides_rotate_host_batch on the same items.  No reference
 * counterpart (the reference loads and recovers one ciphertext at a time,
 * CudaEngine.cpp:1156-1227). */
int fides_mixed_host_batch(fides_ctx* ctx, const fides_hmult_host_item* hm, int n_hm, const uint64_t* relin_key_dev,
                           int rescale, const fides_rotate_host_item* rot, int n_rot);
/* fides_mixed_host_batch that returns once its copies and kernels are enqueued.  Consecutive
 * calls continue one pipeline (the context's device slots rotate across calls), so a call's
 * first host->device copies run under the previous call's last kernels instead of after its
 * last device->host copies.  Every host buffer of a call must stay valid and unchanged, and
 * its outputs unread, until fides_host_batch_wait returns.  Enqueueing errors (bad levels,
 * null pointers) are reported by the call; device errors by fides_host_batch_wait. */
int fides_mixed_host_batch_async(fides_ctx* ctx, const fides_hmult_host_item* hm, int n_hm,
                                 const uint64_t* relin_key_dev, int rescale, const fides_rotate_host_item* rot,
                                 int n_rot);
/* Waits for every pipelined host batch enqueued on ctx (copies included) and reports a device
 * error or a bounded wait that gave up. */
int fides_host_batch_wait(fides_ctx* ctx);

/* ---- bootstrapping ---------------------------------------------------------------------
 * CKKS bootstrapping driven from the library's C++ host layer: replaces CKKS::Bootstrap
 * (src/CKKS/Bootstrap.cu:437-648) behind CudaEngine::evalBootstrap and
 * CryptoContext::EvalBootstrapSetup / EvalBootstrapKeyGen / EvalBootstrap
 * (api/CryptoContext.hpp:306-458).  Sequence: optional sparse-secret encapsulation
 * (keySwitchSparse, Bootstrap.cu:257-290: the level-1 input is switched to a sparse secret
 * before ModRaise and back right after it), an optional power-of-two prescale, ModRaise,
 * CoeffsToSlots (level_budget_cts BSGS linear transforms of the special FFT, CoeffsToSlots.cu:
 * 75-151), EvalMod on the real and imaginary parts (Chebyshev series of the scaled cosine by
 * Paterson-Stockmeyer, then r double-angle steps; ApproxModEval.cu:45-167, 527, 873) and
 * SlotsToCoeffs (level_budget_stc transforms).  Full packing: N/2 slots.  Scales follow the
 * FLEXIBLEAUTO chain S_(l-1) = S_l^2 / q_(l-1) from S_(n_q) = top_scale.  The tables (special-FFT
 * diagonals, Chebyshev coefficients) are derived from the mathematics at creation. */
typedef struct fides_boot_params {
  int level_budget_cts, level_budget_stc; /* levels of CoeffsToSlots / SlotsToCoeffs ({3, 3}) */
  int top_level;         /* limbs after ModRaise (<= n_q) */
  double top_scale;      /* S_(n_q): the scale chain's top */
  double msg_scale;      /* scale of the input ciphertexts' slots */
  int K;                 /* EvalMod range: |m + q_0 I| < K q_0 */
  int r;                 /* double-angle steps */
  int degree;            /* Chebyshev degree */
  int baby;              /* BSGS baby steps */
  int prescale_bits;     /* input multiplied by 2^prescale_bits before ModRaise (divided out after) */
  int sparse_encapsulation; /* 1: switch to a sparse secret around ModRaise (keys below) */
  int correction_bits;   /* > 0: the input (at least 2 limbs) is first scaled down by about
                          * 2^correction_bits -- multiplied by round(q_1 / 2^k) and rescaled by q_1 --
                          * so that a message at a scale close to q_0 (scaling primes nearly as
                          * large as q_0) leaves EvalMod room; OpenFHE's correction factor */
  int double_hoist;      /* 1: the linear transforms keep their baby-step rotations and giant-step
                          * outputs in the extended basis Q P (diagonals encoded with the special
                          * limbs too): no ModDown per baby step, one ModDown of c1 per giant step
                          * and one ModDown + rescale per transform.  Results then differ from
                          * the single-hoisted form in the ModDown rounding only. */
} fides_boot_params;
typedef struct fides_boot fides_boot;
int fides_boot_create(fides_ctx* ctx, const fides_boot_params* params, fides_boot** out);
/* Chebyshev series of a ciphertext (replaces evalChebyshevSeries, src/CKKS/ApproxModEval.cu:527,
 * behind CryptoContext::EvalChebyshevSeries, api/CryptoContext.hpp:406): OpenFHE's convention
 * p(x) = c_0 / 2 + sum_(k >= 1) c_k T_k(t), t = (2 x - (lo + hi)) / (hi - lo), for the n_coeffs
 * coefficients c.  Evaluated by Paterson-Stockmeyer in the Chebyshev basis (the bootstrapper's
 * EvalMod evaluator) with the relinearisation key, on the scale chain S_L = top_scale,
 * S_(l-1) = S_l^2 / q_(l-1).  The input (c0, c1) at `level` limbs and `scale` (brought to the
 * canonical S_level one level down if it differs); the result goes to out0 / out1 (room for
 * `level` limbs each) at *out_level = level - ceil(log2 d) - 1 limbs for degree d (one fewer
 * when [lo, hi] != [-1, 1], one fewer again for a non-canonical input scale), at scale
 * *out_scale (that level's canonical scale). */
int fides_eval_chebyshev(fides_ctx* ctx, const uint64_t* relin_key, double top_scale, const uint64_t* c0,
                         const uint64_t* c1, int level, double scale, const double* coeffs, int n_coeffs, double lo,
                         double hi, uint64_t* out0, uint64_t* out1, int* out_level, double* out_scale,
                         void* stream);
int fides_boot_destroy(fides_boot* b);
/* Rotation amounts (slots, in [1, N/2)) whose keys the linear transforms use: writes up to cap
 * of them and returns the count (EvalBootstrapKeyGen's rotation list). */
int fides_boot_rotations(const fides_boot* b, int* out, int cap);
/* Device keys (owned by the caller, kept for the bootstrapper's lifetime): relinearisation,
 * conjugation (automorphism 2N - 1) and, with sparse_encapsulation, the switching keys dense ->
 * sparse and sparse -> dense secret. */
int fides_boot_set_keys(fides_boot* b, const uint64_t* relin_key, const uint64_t* conj_key, const uint64_t* to_sparse,
                        const uint64_t* to_dense);
int fides_boot_set_rotation_key(fides_boot* b, int rotation, const uint64_t* key);
/* Encodes the linear transforms' diagonals on the device (synchronises `stream`). */
int fides_boot_prepare(fides_boot* b, void* stream);
/* Level (limbs) and scale of the bootstrapped output. */
int fides_boot_levels(const fides_boot* b, int* out_level, double* out_scale);
/* Bootstraps (c0, c1) (limb q_0 is read; limbs q_0, q_1 with correction_bits) into out0 / out1
 * (out_level limbs each) on `stream`. */
int fides_bootstrap(fides_boot* b, const uint64_t* c0, const uint64_t* c1, uint64_t* out0, uint64_t* out1,
                    void* stream);
/* n bootstraps at once on `stream`: up to 16 ciphertexts go through one launch sequence
 * together (every hoisted rotation, key switch, HMult, plaintext inner product, linear
 * combination and rescale of the batch in the same launches, EvalMod on 2 x 16 lanes).
 * Results equal fides_bootstrap's, ciphertext by ciphertext.  No reference counterpart (the
 * reference bootstraps one ciphertext per call). */
int fides_bootstrap_batch(fides_boot* b, int n, const uint64_t* const* c0s, const uint64_t* const* c1s,
                          uint64_t* const* out0s, uint64_t* const* out1s, void* stream);
/* The derived tables, for inspection and comparison: the Chebyshev coefficients (returns the
 * count); the number of composed matrices of CoeffsToSlots (which = 0) or SlotsToCoeffs (1);
 * matrix m's slot-diagonal offsets and, when diags is not NULL, its diagonals as
 * [count][N/2][re, im] doubles (returns the count; cap bounds what is written). */
int fides_boot_chebyshev(const fides_boot* b, double* coeffs, int cap);
int fides_boot_matrices(const fides_boot* b, int which);
int fides_boot_table(const fides_boot* b, int which, int m, int* offsets, int cap, double* diags);
/* After fides_boot_prepare: copies the encoded diagonal (i, j) (giant step i, baby step j) of
 * matrix m into out (the matrix's level limbs, EVALUATION form). */
int fides_boot_plaintext(const fides_boot* b, int which, int m, int i, int j, uint64_t* out, void* stream);

/* ---- allocation-free entry point ----------------------------------------------------
 * No counterpart in the reference.  fides_rescale_noalloc computes exactly what
 * fides_rescale computes for one polynomial, but takes its scratch (one limb) from a
 * 512 KiB array compiled into the library instead of allocating device memory, for
 * callers that cannot allocate on the call path: hosts whose HBM is entirely reserved
 * by another allocator (every extra cudaMalloc fails) and latency-bound loops that cannot
 * take the synchronisation cudaMalloc / cudaFree bring.  Limits and rules:
 *   - N <= 2^16 (a larger ring returns FIDES_ERR_ARG), 2 <= level <= n_q;
 *   - out (level - 1 limbs) must not overlap x (FIDES_ERR_ARG);
 *   - the array is shared by every call on a device: calls that overlap on the GPU race;
 *   - the first call on a device looks up the array's device address (with that device
 *     current) and caches it; make that first call before any stream capture. */
int fides_rescale_noalloc(fides_ctx* ctx, const uint64_t* x, int level, uint64_t* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
