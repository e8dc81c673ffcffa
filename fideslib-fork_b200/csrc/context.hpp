// Internal context of the CKKS evaluation core: parameters, device-resident tables and
// the scratch allocator.  Replaces the reference's ContextData (src/CKKS/Context.cu:74-138)
// and the __constant__ Constants / Global::Globals tables (src/ConstantsGPU.cuh:49-198):
// every table lives in global memory sized to the parameter set, so there is no
// MAXP/MAXD ceiling (ConstantsGPU.cuh:12-32).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "modarith.cuh"

namespace fides {

// Error carried from the internals to the C ABI.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define FIDES_CUDA(call)                                                                           \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      throw ::fides::Error(-2, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + __FILE__ + \
                                   ":" + std::to_string(__LINE__));                                \
  } while (0)

// A Shoup-precomputed constant.
struct __align__(16) ShoupConst {
  uint64_t w, ws;
};

// Destination-prime constants of the tensor-core conversion epilogue.
struct __align__(16) TcDest {
  uint64_t q;
  uint64_t qinv;  // bits of the double nearest 1 / q
};

// Table of one approximate basis conversion (ApproxSwitchCRTBasis):
//   y_i = [x_i * pre_i]_{q_src_i};  out_j = [sum_i y_i * mat[i][j]]_{q_dst_j}.
struct ConvTable {
  int n_src = 0, n_dst = 0;
  const int* src_pos = nullptr;    // limb index of source i in the input poly
  const int* src_prime = nullptr;  // prime id of source i
  const ShoupConst* pre = nullptr; // [n_src]
  const int* dst_pos = nullptr;    // limb index of output j in the output poly
  const int* dst_prime = nullptr;  // prime id of output j
  const uint64_t* mat = nullptr;   // [n_src][n_dst]
  // Tensor-core form (conv_tc.cu); tc_b == nullptr when the table does not fit it.
  //   tc_b: the MMA B operand, byte (n, k) = byte (n mod 8) of mat[k/8][n/8] * 2^(8 (k mod 8))
  //         mod q_dst, stored as its shared-memory image: 16-byte K slices, slice s of row n at
  //         (s * nd_pad * 8 + n) * 16.
  const uint8_t* tc_b = nullptr;
  const TcDest* tc_dst = nullptr;  // [nd_pad]
  int tc_kpad = 0;                 // K = 8 (n_src + lift) rounded up to a multiple of 32
  int tc_nd_pad = 0;               // n_dst rounded up to even
  // Reduced-noise lift (reference src/CKKS/Conv.cu:76-87 and :356-381, ReducedNoise.cuh:14-16):
  // with lift = 1 the conversion also adds cnt * [-Q_src]_{p_j}, cnt = the number of pre-scaled
  // sources y_i above q_i / 2, i.e. it converts the centred representatives y_i - q_i.  Row
  // n_src of mat (and of the B image) holds [-Q_src]_{p_j}.
  int lift = 0;
};

// Basis-conversion engine: tensor cores (INT8 split on tcgen05) or 64-bit SIMT.
enum ConvEngine { CONV_AUTO = 0, CONV_SIMT = 1, CONV_TENSOR = 2 };

// FP64 constants of a prime below 2^50 for the floating-point NTT butterflies: q, 1/q, and
// the inverse transform's last-stage factors N^-1 and psi_rev^-1[1] N^-1 with their
// quotients by q.
struct F64Prime {
  double q, qinv, ninv, ninv_q, last, last_q;
};

struct RescaleConst {
  uint64_t qinv, qinv_s;  // q_top^-1 mod q_j
  uint64_t m, m_s;        // QlQlInvModqlDivqlModq_j = -q_top^-1 mod q_j
};

// Kernel families timed by the profiling mode (fides_ctx_profile).
enum KernelKind { KK_NTT = 0, KK_CONV = 1, KK_KSK = 2, KK_ELEM = 3, KK_COUNT = 4 };

struct ProfileRec {
  int kind;
  cudaEvent_t beg, end;
  double bytes;  // algorithmic bytes of this launch
};

struct Context {
  int device = 0;
  int logN = 0, N = 0, n_q = 0, K = 0, dnum = 0, alpha = 0;
  std::vector<uint64_t> primes, psi;

  // device tables
  DevPrime* d_prime = nullptr;       // [n_q + K]
  ShoupConst* d_tw_fwd = nullptr;    // [n_q + K][N]: psi_rev (bit-reversed powers of psi)
  ShoupConst* d_tw_inv = nullptr;    // [n_q + K][N]: psi^-1 bit-reversed
  ShoupConst* d_inv_last = nullptr;  // [n_q + K]: psi_rev^-1[1] * N^-1 (last GS stage)
  double2* d_twf_fwd = nullptr;      // [n_q + K][N]: (w, w / q) of d_tw_fwd as doubles (q < 2^50)
  double2* d_twf_inv = nullptr;      // [n_q + K][N]: the same for d_tw_inv
  double* d_tww_fwd = nullptr;       // [n_q + K][N]: w / q alone, correctly rounded (row passes derive w)
  double* d_tww_inv = nullptr;
  F64Prime* d_f64 = nullptr;         // [n_q + K]
  ShoupConst* d_pinv = nullptr;      // [n_q]: P^-1 mod q_j
  ShoupConst* d_pmod = nullptr;      // [n_q]: P mod q_j
  RescaleConst* d_rescale = nullptr; // [n_q + 1][n_q]: row l = rescale from level l
  ShoupConst* d_pqinv = nullptr;     // [n_q + 1][n_q]: row l = (P q_(l-1))^-1 mod q_j
  void* d_tables = nullptr;          // backing store of the conversion tables
  std::vector<std::vector<ConvTable>> modup_tab;  // [l][d]
  std::vector<ConvTable> moddown_tab;              // [l]
  // The same tables with the reduced-noise lift; used while reduced_noise is set (reference
  // Parameters::reducedNoise, src/CKKS/Parameters.cuh:31, off by default).
  std::vector<std::vector<ConvTable>> modup_tab_rn;
  std::vector<ConvTable> moddown_tab_rn;
  bool reduced_noise = false;
  const ConvTable& modup_table(int l, int d) const { return (reduced_noise ? modup_tab_rn : modup_tab)[l][d]; }
  const ConvTable& moddown_table(int l) const { return (reduced_noise ? moddown_tab_rn : moddown_tab)[l]; }
  int conv_engine = CONV_AUTO;
  // NTT tile shapes: sub-transforms per CTA (4, 8 or 16) of each pass, by direction (0 =
  // forward, 1 = inverse), pass (0 = column, 1 = row) and launch-size class (limbs in the
  // launch: <= 8, <= 32, <= 128, more).  Defaults keep every SM busy on small launches;
  // fides_ctx_autotune replaces them with timed choices.
  uint8_t ntt_g[2][2][4] = {{{4, 8, 16, 16}, {4, 8, 16, 16}}, {{4, 8, 16, 16}, {4, 8, 16, 16}}};
  static int ntt_size_class(int limbs) { return limbs <= 8 ? 0 : limbs <= 32 ? 1 : limbs <= 128 ? 2 : 3; }
  // Limbs per transform launch pair: a list longer than this runs as balanced chunks, each chunk's
  // column and row passes back to back, so that a chunk that fits in L2 has its intermediate read
  // by the second pass from L2 (and overwritten there in place, never written to DRAM).  0 = the
  // largest launch (MAX_NTT_LIMBS); fides_ctx_autotune picks it by timing.
  int ntt_chunk = 0;
  int ntt_shape(bool inverse, int pass, int limbs) const { return ntt_g[inverse][pass][ntt_size_class(limbs)]; }
  // Residues per thread (16 or 8) of each pass, indexed like ntt_g.  8 exists at N >= 2^15 only
  // (elsewhere 16 is used whatever the table holds); 16 by default, fides_ctx_autotune times both.
  uint8_t ntt_r[2][2][4] = {{{16, 16, 16, 16}, {16, 16, 16, 16}}, {{16, 16, 16, 16}, {16, 16, 16, 16}}};
  int ntt_residues(bool inverse, int pass, int limbs) const { return ntt_r[inverse][pass][ntt_size_class(limbs)]; }
  uint32_t* d_status = nullptr;  // device word: bit 0 = a bounded device wait gave up,
                                 // bit 1 = an encoded coefficient exceeded 2^62
  // special-FFT twiddles of the slot encoder, [N/2] (double, double) pairs: entry h + j
  // (h = len / 2, j < h) = exp(-2 pi i (5^j mod 4 len) / (4 len))
  void* d_sfft = nullptr;

  // scratch: stream-ordered allocations from the device's memory pool
  cudaMemPool_t pool = nullptr;
  std::atomic<size_t> scratch_in_use{0};
  std::atomic<size_t> scratch_peak{0};
  size_t scratch_limit = 0;
  std::atomic<uint64_t> launches{0};
  // limb transforms submitted to the NTT, by butterfly form: [0] FP64 (q < 2^50), [1] integer
  std::atomic<uint64_t> ntt_limbs_by_form[2] = {0, 0};
  // profiling mode: CUDA events around every launch, per kernel family
  bool profiling = false;
  std::mutex prof_mu;
  std::vector<ProfileRec> prof;
  std::vector<cudaEvent_t> ev_pool;
  std::mutex host_mu;                // guards the pinned staging buffers of the host entry points
  void* pinned = nullptr;
  size_t pinned_bytes = 0;

  int beta(int l) const { return (l + alpha - 1) / alpha; }
  size_t limb_bytes() const { return sizeof(uint64_t) * (size_t)N; }
};

// RAII stream-ordered scratch buffer.
struct Scratch {
  Context* ctx = nullptr;
  cudaStream_t s = nullptr;
  void* p = nullptr;
  size_t bytes = 0;
  Scratch(Context* c, size_t b, cudaStream_t st);
  ~Scratch();
  uint64_t* u64() const { return static_cast<uint64_t*>(p); }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
};

// Grows the scratch pool to hold at least `bytes` (allocate, free, synchronise): the pool
// keeps freed memory (release threshold unbounded), so later stream-ordered allocations up to
// that size never map new memory on the launch path.
void reserve_scratch(Context* c, size_t bytes);

Context* create_context(int logN, int n_q, int K, int dnum, const uint64_t* primes, const uint64_t* psi, int device);
void destroy_context(Context* c);

// Launch bracket: counts the launch and, in profiling mode, records events around it.
struct LaunchScope {
  Context* c;
  cudaStream_t s;
  int idx = -1;
  LaunchScope(Context* ctx, cudaStream_t st, int kind, double bytes);
  ~LaunchScope();
};

// host number theory (same rules as the reference's Math.cu / ConstantsGPU.cu)
uint64_t h_mulmod(uint64_t a, uint64_t b, uint64_t q);
uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q);
uint64_t h_invmod(uint64_t a, uint64_t q);
uint64_t h_root_2n(uint64_t q, int logN);
ShoupConst h_shoup(uint64_t w, uint64_t q);
uint32_t h_auto_index(int logN, int rotation);

}  // namespace fides
