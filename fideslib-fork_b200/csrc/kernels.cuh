// Elementwise RNS kernels, basis conversion and the key-switch-key inner product.
//
// Every kernel takes a by-value job list so that one launch covers many polynomials at
// uneven levels (blockIdx.z = job, blockIdx.y = limb, blockIdx.x = coefficient tile).
#pragma once
#include <cuda_runtime.h>

#include "context.hpp"

namespace fides {

constexpr int EW_THREADS = 256;  // coefficients per CTA tile

// Architecture of the library's device code as the runtime loaded it on `device`
// (cudaFuncAttributes::binaryVersion of one of its kernels: 100 for sm_100a).
int kernel_binary_version(int device);

// ---- basis conversion (ModUp: DecompAndModUpConv, Conv.cu:274-423; ModDown: ModDown2, Conv.cu:27-133)
struct ConvJob {
  ConvTable t;
  const uint64_t* src;  // source limb i at src + t.src_pos[i] * N (coefficient domain)
  uint64_t* dst;        // output j at dst + t.dst_pos[j] * N
};
constexpr int MAX_CONV_JOBS = 96;
struct ConvJobList {
  int n, max_src, max_dst, pad;
  ConvJob j[MAX_CONV_JOBS];
};
void launch_conv(Context* c, const ConvJob* jobs, int n, cudaStream_t s);

// ---- KSK inner product (fusedDotKSK_2_, ElemenwiseBatchKernels.cu:202-274) with the
// hoisted-rotation extras of hoistedRotateDotKSK_2_ (:277-377): + P c0 on the b side and an
// automorphism scatter of both outputs.
struct KskJob {
  const uint64_t* x;       // EVAL input at level l (own-digit limbs)
  const uint64_t* x2;      // optional: the input is x * x2 (tensor term a1 b1, never materialised)
  const uint64_t* digits;  // [beta][l + K][N] ModUp output (EVAL)
  const uint64_t* key;     // [2][dnum][n_q + K][N]
  const uint64_t* c0;      // optional: add P * c0 to out_b's Q limbs
  uint64_t* out_a;         // [l + K][N]
  uint64_t* out_b;
  int l;
  uint32_t auto_k;  // 0 = no automorphism
  // optional HMult tensor terms (x = a1, x2 = b1): add P a0 b0 to out_b's and
  // P (a0 b1 + a1 b0) to out_a's Q limbs, so that ModDown yields ModDown(.) + d0 / + d1
  const uint64_t* a0 = nullptr;
  const uint64_t* b0 = nullptr;
  // optional extended-basis addend of out_b, every limb, not multiplied by P (the c0 of a
  // ciphertext kept in the extended basis, double-hoisted linear transforms); before the
  // automorphism scatter
  const uint64_t* c0x = nullptr;
};
constexpr int MAX_KSK_JOBS = 64;
// Jobs that share a switching key (one relinearisation or rotation key for a batch) and the
// same level and extras form a group of up to 4; one CTA runs a whole group, reading each key
// tile once for all of its jobs.  (Groups of 8 read the key half as often but measured 20 %
// slower on the bench step: half as many CTAs, each running twice as long, and more spills.)
constexpr int MAX_KSK_GROUP = 4;
struct KskJobList {
  int n, max_ext, ngroups, pad1;
  uint8_t gstart[MAX_KSK_JOBS], gcount[MAX_KSK_JOBS];
  KskJob j[MAX_KSK_JOBS];
};
void launch_ksk(Context* c, const KskJob* jobs, int n, cudaStream_t s);

// ---- ModDown epilogue (NTT_MODDOWN, NTTfusions.cuh:237-252): out = (x - conv) P^-1 (+ add)
struct FinJob {
  const uint64_t* x;     // Q limbs of the extended poly
  const uint64_t* conv;  // converted special part, EVAL
  const uint64_t* add;   // optional addend
  uint64_t* out;
  int l;
  int pad;
};
constexpr int MAX_FIN_JOBS = 128;
struct FinJobList {
  int n, max_l, pad0, pad1;
  FinJob j[MAX_FIN_JOBS];
};
void launch_moddown_finish(Context* c, const FinJob* jobs, int n, cudaStream_t s);

// ---- tensor product (binomialMult_, ElemenwiseBatchKernels.cu:1363-1510)
struct TensorJob {
  const uint64_t *a0, *a1, *b0, *b1;
  uint64_t *d0, *d1, *d2;
  int l;
  int pad;
};
constexpr int MAX_TENSOR_JOBS = 64;
struct TensorJobList {
  int n, max_l, pad0, pad1;
  TensorJob j[MAX_TENSOR_JOBS];
};
void launch_tensor(Context* c, const TensorJob* jobs, int n, cudaStream_t s);

// ---- rescale (rescale_fusion, NTTfusions.cuh:214-235; SwitchModulus, Rescale.cuh:44-64)
struct SwitchJob {
  const uint64_t* top;  // top limb, coefficient domain
  uint64_t* out;        // l - 1 limbs
  int l;
  int pad;
};
struct RescaleJob {
  const uint64_t* x;  // EVAL, level l
  const uint64_t* t;  // NTT(SwitchModulus(top)), l - 1 limbs
  uint64_t* out;      // l - 1 limbs
  int l;
  int pad;
};
constexpr int MAX_RS_JOBS = 128;
struct SwitchJobList {
  int n, max_l, pad0, pad1;
  SwitchJob j[MAX_RS_JOBS];
};
struct RescaleJobList {
  int n, max_l, pad0, pad1;
  RescaleJob j[MAX_RS_JOBS];
};
void launch_switch_modulus(Context* c, const SwitchJob* jobs, int n, cudaStream_t s);
void launch_rescale_finish(Context* c, const RescaleJob* jobs, int n, cudaStream_t s);

// ---- RNS elementwise ops (reference add_ / sub_, src/AddSub.cu:10-123; Mult_ /
// Scalar_mult_ / scalar_add_, src/CKKS/ElemenwiseBatchKernels.cu:14-200, src/AddSub.cu)
enum EwOp { EW_ADD = 0, EW_SUB = 1, EW_MUL = 2, EW_MUL_SCALAR = 3, EW_ADD_SCALAR = 4 };
struct AddSubJob {
  const uint64_t *a, *b;  // b: second operand (ADD/SUB/MUL) or per-limb scalars (device, *_SCALAR)
  uint64_t* out;
  int l;
  int sub;  // EwOp
  int lq = 0, nq = 0;  // extended-basis operands (ext_prime); lq = 0: Q limbs only
};
constexpr int MAX_ADDSUB_JOBS = 128;
struct AddSubJobList {
  int n, max_l, pad0, pad1;
  AddSubJob j[MAX_ADDSUB_JOBS];
};
void launch_addsub(Context* c, const AddSubJob* jobs, int n, cudaStream_t s);

// Per-limb scalar ops: out_i = a_i * s_i or a_i + s_i (mod q_i), scalars passed by value.
constexpr int MAX_SCALAR_LIMBS = 64;
struct ScalarJob {
  const uint64_t* a;
  uint64_t* out;
  int l;
  int op;  // EW_MUL_SCALAR or EW_ADD_SCALAR
  uint64_t s[MAX_SCALAR_LIMBS];
};
constexpr int MAX_SCALAR_JOBS = 8;
struct ScalarJobList {
  int n, max_l, pad0, pad1;
  ScalarJob j[MAX_SCALAR_JOBS];
};
void launch_scalar(Context* c, const ScalarJob* jobs, int n, cudaStream_t s);

// ---- plaintext-ciphertext inner product of a linear transform's giant step
// (LTdotProductPtBatch / dotProductLtBatchedPt___, LimbPartitionBatch.cu:266,
// ElemenwiseBatchKernels.cu:682-1106): out_k = sum_t pt_t * c_k,t mod q, k = 0, 1, with
// 128-bit accumulation, one launch per giant step instead of two products and two sums per
// diagonal.  Up to MAX_DOT_LANES ciphertexts (lanes) share the plaintext diagonals: the
// lanes of one (limb, coefficient tile) are adjacent CTAs, so each diagonal tile is read from
// DRAM once per launch and from L2 by the other lanes.
constexpr int MAX_DOT_TERMS = 32;
constexpr int MAX_DOT_LANES = 8;
struct DotJob {
  const uint64_t* c0[MAX_DOT_LANES][MAX_DOT_TERMS];
  const uint64_t* c1[MAX_DOT_LANES][MAX_DOT_TERMS];
  const uint64_t* pt[MAX_DOT_TERMS];
  uint64_t* out0[MAX_DOT_LANES];
  uint64_t* out1[MAX_DOT_LANES];
  int n, l, lanes;
  int lq = 0, nq = 0;  // extended-basis operands: limbs >= lq are special limb (limb - lq) (lq = 0: none)
};
// Prime id of limb j of an operand whose first lq limbs are Q limbs 0..lq-1 and whose others
// are the special limbs (lq = 0: every limb is a Q limb).
__host__ __device__ inline int ext_prime(int j, int lq, int nq) { return (lq == 0 || j < lq) ? j : nq + (j - lq); }
void launch_dot_plain(Context* c, const DotJob& job, cudaStream_t s);

// ---- every giant step's inner product of a BSGS linear transform in one launch:
// out_i = sum_j pt[i][j] * x_j for all giant steps i, each baby-step ciphertext x_j and each
// diagonal read from DRAM once (one launch per giant step reads each x_j once per giant step);
// lanes (the ciphertexts of a batch) share the diagonals as in DotJob.
constexpr int MAX_BSGS_BABY = 16;
constexpr int MAX_BSGS_GIANT = 16;
constexpr int MAX_BSGS_LANES = 8;
struct BsgsJob {
  const uint64_t* x0[MAX_BSGS_LANES][MAX_BSGS_BABY];
  const uint64_t* x1[MAX_BSGS_LANES][MAX_BSGS_BABY];
  const uint64_t* pt[MAX_BSGS_GIANT][MAX_BSGS_BABY];  // diagonal (i, j), or null (no term)
  uint64_t* out0[MAX_BSGS_LANES][MAX_BSGS_GIANT];
  uint64_t* out1[MAX_BSGS_LANES][MAX_BSGS_GIANT];
  int nb, ng, l, lanes;
  int lq = 0, nq = 0;  // as DotJob
};
void launch_bsgs_dot(Context* c, const BsgsJob& job, cudaStream_t s);

// ---- ciphertext linear combination with per-limb integer constants:
// out0 = sum_t s_t * x0_t + add0, out1 = sum_t s_t * x1_t (mod q_j per limb j).  The scalar
// steps of a Chebyshev series in one launch: the weighted sums of the Paterson-Stockmeyer
// leaves (evalPartialLinearWSumFused, ApproxModEval.cu:272, inside innerEvalChebyshevPS,
// ApproxModEval.cu:341) and the 2 T_a T_b - T_c recurrence combinations, instead of a
// multiply and an add launch per term.  Lanes: the same constants applied to up to 8
// independent sets of operands (one grid z slice each), e.g. the real and imaginary halves
// of EvalMod.
constexpr int MAX_LC_TERMS = 16;
constexpr int MAX_LC_LIMBS = 64;
constexpr int MAX_LC_LANES = 8;
struct LinCombJob {
  const uint64_t* x0[MAX_LC_LANES][MAX_LC_TERMS];
  const uint64_t* x1[MAX_LC_LANES][MAX_LC_TERMS];
  uint64_t* out0[MAX_LC_LANES];
  uint64_t* out1[MAX_LC_LANES];
  uint64_t s[MAX_LC_TERMS][MAX_LC_LIMBS];
  uint64_t add0[MAX_LC_LIMBS];
  int n, l, lanes;
  int lq = 0, nq = 0;  // as DotJob (s and add0 hold residues modulo each limb's own prime)
};
void launch_lincomb(Context* c, const LinCombJob& job, cudaStream_t s);

}  // namespace fides
