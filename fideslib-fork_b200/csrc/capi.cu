// extern "C" boundary (include/fides_b200.h).  Converts exceptions into status codes and
// a thread-local message, the C counterpart of the reference's OPENFHE_THROW / CudaError
// (api/engine/cuda/CudaEngine.cpp, src/CudaUtils.cuh:706-757).
#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fides_b200.h"
#include "autotune.hpp"
#include "capi_internal.hpp"
#include "context.hpp"
#include "encode.hpp"
#include "interop.hpp"
#include "kernels.cuh"
#include "ntt.cuh"
#include "ops.hpp"

namespace {
thread_local std::string g_err;

// Entry-point bracket: an NVTX range named after the entry point (the counterpart of the
// reference's CudaNvtxRange on every operation, src/CudaUtils.cuh:662-690), exceptions turned
// into status codes, and the caller's current device restored on return (entry points make the
// context's device current while they run).
struct EntryScope {
  int prev_device = -1;
  explicit EntryScope(const char* name) {
    nvtxRangePushA(name);
    if (cudaGetDevice(&prev_device) != cudaSuccess) prev_device = -1;
  }
  ~EntryScope() {
    if (prev_device >= 0) cudaSetDevice(prev_device);
    nvtxRangePop();
  }
};

template <typename F>
int guard_named(const char* name, F&& f) {
  EntryScope scope(name);
  try {
    f();
    return FIDES_OK;
  } catch (const fides::Error& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "host allocation failed";
    return FIDES_ERR_OOM;
  } catch (const std::exception& e) {
    g_err = e.what();
    return FIDES_ERR_STATE;
  }
}
#define guard(...) guard_named(__func__, __VA_ARGS__)

// After a synchronisation: a bounded device-side wait that gave up (status bit 0) makes the
// call fail with FIDES_ERR_TIMEOUT.  The bit stays set (every later synchronising call fails
// too) until fides_ctx_device_status clears it, since the affected outputs are incomplete.
void check_device_status(fides::Context* c) {
  uint32_t st = 0;
  FIDES_CUDA(cudaMemcpy(&st, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (st & 1u)
    throw fides::Error(FIDES_ERR_TIMEOUT,
                       "a bounded device-side wait gave up: outputs since the last status clear are incomplete");
}

fides::Context* C(fides_ctx* x) {
  if (!x || !x->c) throw fides::Error(FIDES_ERR_ARG, "null context");
  FIDES_CUDA(cudaSetDevice(x->c->device));
  return x->c;
}

void need(const void* p, const char* what) {
  if (!p) throw fides::Error(FIDES_ERR_ARG, std::string("null pointer: ") + what);
}

cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }
}  // namespace

void fides::set_last_error(const std::string& msg) { g_err = msg; }

namespace fides {
double measure_bf_peak(int device);      // calibrate.cu
double measure_bf_peak_f64(int device);  // calibrate.cu
}

extern "C" {

const char* fides_last_error(void) { return g_err.c_str(); }

int fides_ctx_create(const fides_params* p, fides_ctx** out) {
  return guard([&] {
    need(p, "params");
    need(out, "out");
    need(p->primes, "primes");
    auto* x = new fides_ctx{nullptr, nullptr};
    try {
      x->c = fides::create_context(p->logN, p->n_q, p->n_special, p->dnum, p->primes, p->psi, p->device);
      FIDES_CUDA(cudaStreamCreateWithFlags(&x->host_stream, cudaStreamNonBlocking));
      FIDES_CUDA(cudaStreamCreateWithFlags(&x->h2d_stream, cudaStreamNonBlocking));
      FIDES_CUDA(cudaStreamCreateWithFlags(&x->d2h_stream, cudaStreamNonBlocking));
    } catch (...) {
      if (x->host_stream) cudaStreamDestroy(x->host_stream);
      if (x->h2d_stream) cudaStreamDestroy(x->h2d_stream);
      if (x->c) fides::destroy_context(x->c);
      delete x;
      throw;
    }
    *out = x;
  });
}

int fides_ctx_destroy(fides_ctx* x) {
  return guard([&] {
    if (!x) return;
    if (x->h2d_stream) cudaStreamSynchronize(x->h2d_stream);
    if (x->host_stream) cudaStreamSynchronize(x->host_stream);
    if (x->d2h_stream) cudaStreamSynchronize(x->d2h_stream);
    if (x->pipe_mem) cudaFree(x->pipe_mem);
    for (int i = 0; i < fides_ctx::kPipeSlots; ++i)
      for (cudaEvent_t e : {x->pipe_free[i], x->pipe_in_ready[i], x->pipe_computed[i]})
        if (e) cudaEventDestroy(e);
    if (x->host_stream) cudaStreamDestroy(x->host_stream);
    if (x->h2d_stream) cudaStreamDestroy(x->h2d_stream);
    if (x->d2h_stream) cudaStreamDestroy(x->d2h_stream);
    fides::destroy_context(x->c);
    delete x;
  });
}

int fides_ctx_psi(const fides_ctx* x, uint64_t* psi_out) {
  return guard([&] {
    need(x, "ctx");
    need(psi_out, "psi_out");
    std::memcpy(psi_out, x->c->psi.data(), sizeof(uint64_t) * x->c->psi.size());
  });
}

int fides_ctx_alpha(const fides_ctx* x) { return x && x->c ? x->c->alpha : FIDES_ERR_ARG; }

size_t fides_ctx_scratch_bytes(const fides_ctx* x) { return x && x->c ? x->c->scratch_in_use.load() : 0; }

int fides_ctx_set_scratch_limit(fides_ctx* x, size_t bytes) {
  return guard([&] { C(x)->scratch_limit = bytes; });
}

uint64_t fides_ctx_launch_count(const fides_ctx* x) { return x && x->c ? x->c->launches.load() : 0; }

int fides_int_peak(int device, double* butterflies_per_s) {
  return guard([&] {
    need(butterflies_per_s, "butterflies_per_s");
    *butterflies_per_s = fides::measure_bf_peak(device);
  });
}

int fides_f64_peak(int device, double* butterflies_per_s) {
  return guard([&] {
    need(butterflies_per_s, "butterflies_per_s");
    *butterflies_per_s = fides::measure_bf_peak_f64(device);
  });
}

int fides_kernel_arch(int device, int* binary_version) {
  return guard([&] {
    need(binary_version, "binary_version");
    *binary_version = fides::kernel_binary_version(device);
  });
}

int fides_ctx_ntt_counts(fides_ctx* x, uint64_t* f64_limbs, uint64_t* int_limbs) {
  return guard([&] {
    auto* c = C(x);
    need(f64_limbs, "f64_limbs");
    need(int_limbs, "int_limbs");
    *f64_limbs = c->ntt_limbs_by_form[0].load();
    *int_limbs = c->ntt_limbs_by_form[1].load();
  });
}

int fides_ctx_reserve_scratch(fides_ctx* x, size_t bytes) {
  return guard([&] { fides::reserve_scratch(C(x), bytes); });
}

int fides_ctx_autotune(fides_ctx* x, float* best_ms) {
  return guard([&] { fides::autotune_ntt(C(x), best_ms); });
}

int fides_ctx_ntt_shapes(fides_ctx* x, uint8_t* shapes) {
  return guard([&] {
    auto* c = C(x);
    need(shapes, "shapes");
    std::memcpy(shapes, &c->ntt_g[0][0][0], 16);
  });
}

int fides_ctx_set_ntt_shape(fides_ctx* x, int inverse, int pass, int size_class, int subs_per_cta) {
  return guard([&] {
    auto* c = C(x);
    if (inverse < 0 || inverse > 1 || pass < 0 || pass > 1 || size_class < 0 || size_class > 3 ||
        (subs_per_cta != 4 && subs_per_cta != 8 && subs_per_cta != 16))
      throw fides::Error(FIDES_ERR_ARG, "bad NTT shape");
    c->ntt_g[inverse][pass][size_class] = (uint8_t)subs_per_cta;
  });
}

int fides_ctx_ntt_residues(fides_ctx* x, uint8_t* residues) {
  return guard([&] {
    auto* c = C(x);
    need(residues, "residues");
    std::memcpy(residues, &c->ntt_r[0][0][0], 16);
  });
}

int fides_ctx_set_ntt_residues(fides_ctx* x, int inverse, int pass, int size_class, int residues_per_thread) {
  return guard([&] {
    auto* c = C(x);
    if (inverse < 0 || inverse > 1 || pass < 0 || pass > 1 || size_class < 0 || size_class > 3 ||
        (residues_per_thread != 8 && residues_per_thread != 16))
      throw fides::Error(FIDES_ERR_ARG, "bad NTT residues per thread");
    if (residues_per_thread == 8 && c->logN < 15)
      throw fides::Error(FIDES_ERR_ARG, "8 residues per thread are built for N >= 2^15 only");
    c->ntt_r[inverse][pass][size_class] = (uint8_t)residues_per_thread;
  });
}

int fides_ctx_ntt_chunk(fides_ctx* x, int set_limbs) {
  int out = 0;
  const int rc = guard([&] {
    auto* c = C(x);
    if (set_limbs > 0) c->ntt_chunk = std::min(set_limbs, fides::MAX_NTT_LIMBS);
    if (set_limbs == 0) c->ntt_chunk = 0;
    out = c->ntt_chunk > 0 ? c->ntt_chunk : fides::MAX_NTT_LIMBS;
  });
  return rc == FIDES_OK ? out : rc;
}

int fides_ctx_set_conv_engine(fides_ctx* x, int engine) {
  return guard([&] {
    if (engine < fides::CONV_AUTO || engine > fides::CONV_TENSOR) throw fides::Error(FIDES_ERR_ARG, "bad engine");
    C(x)->conv_engine = engine;
  });
}

int fides_ctx_set_reduced_noise(fides_ctx* x, int on) {
  return guard([&] {
    if (on != 0 && on != 1) throw fides::Error(FIDES_ERR_ARG, "reduced_noise must be 0 or 1");
    auto* c = C(x);
    if (on && c->K == 0) throw fides::Error(FIDES_ERR_ARG, "reduced noise needs special primes");
    c->reduced_noise = on != 0;
  });
}

int fides_ctx_device_status(fides_ctx* x, uint32_t* status, int clear) {
  return guard([&] {
    auto* c = C(x);
    if (!status) throw fides::Error(FIDES_ERR_ARG, "null status");
    FIDES_CUDA(cudaSetDevice(c->device));
    FIDES_CUDA(cudaDeviceSynchronize());
    FIDES_CUDA(cudaMemcpy(status, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (clear) FIDES_CUDA(cudaMemset(c->d_status, 0, sizeof(uint32_t)));
  });
}

int fides_ctx_synchronize(fides_ctx* x, void* stream) {
  return guard([&] {
    auto* c = C(x);
    FIDES_CUDA(cudaStreamSynchronize(S(stream)));
    check_device_status(c);
  });
}

int fides_ctx_inject_status(fides_ctx* x, uint32_t bits) {
  return guard([&] {
    auto* c = C(x);
    FIDES_CUDA(cudaDeviceSynchronize());
    uint32_t st = 0;
    FIDES_CUDA(cudaMemcpy(&st, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    st |= bits;
    FIDES_CUDA(cudaMemcpy(c->d_status, &st, sizeof(uint32_t), cudaMemcpyHostToDevice));
  });
}

int fides_ctx_profile(fides_ctx* x, int enable) {
  return guard([&] {
    auto* c = C(x);
    std::lock_guard<std::mutex> g(c->prof_mu);
    c->profiling = enable != 0;
  });
}

int fides_ctx_profile_read(fides_ctx* x, int kind, double* ms, double* bytes, uint64_t* launches) {
  return guard([&] {
    auto* c = C(x);
    if (kind < 0 || kind >= fides::KK_COUNT) throw fides::Error(FIDES_ERR_ARG, "bad kernel family");
    std::lock_guard<std::mutex> g(c->prof_mu);
    double t = 0, b = 0;
    uint64_t n = 0;
    std::vector<fides::ProfileRec> keep;
    for (auto& r : c->prof) {
      if (r.kind != kind) {
        keep.push_back(r);
        continue;
      }
      FIDES_CUDA(cudaEventSynchronize(r.end));
      float e = 0;
      FIDES_CUDA(cudaEventElapsedTime(&e, r.beg, r.end));
      t += e;
      b += r.bytes;
      ++n;
      c->ev_pool.push_back(r.beg);
      c->ev_pool.push_back(r.end);
    }
    c->prof.swap(keep);
    if (ms) *ms = t;
    if (bytes) *bytes = b;
    if (launches) *launches = n;
  });
}

uint32_t fides_rotation_auto_index(int logN, int rotation) { return fides::h_auto_index(logN, rotation); }

int fides_ntt_limbs(fides_ctx* x, uint64_t* const* limbs, const int* prime_ids, int n_limbs, int inverse,
                    void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(limbs, "limbs");
    need(prime_ids, "prime_ids");
    std::vector<fides::LimbRef> v(n_limbs);
    for (int i = 0; i < n_limbs; ++i) {
      need(limbs[i], "limb");
      if (prime_ids[i] < 0 || prime_ids[i] >= c->n_q + c->K) throw fides::Error(FIDES_ERR_ARG, "bad prime id");
      v[i] = fides::lref(limbs[i], prime_ids[i]);
    }
    fides::ntt_limbs(c, v.data(), n_limbs, inverse != 0, S(stream));
  });
}

int fides_ntt_polys(fides_ctx* x, uint64_t* data, int n_polys, int n_limbs, int inverse, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(data, "data");
    if (n_polys < 0 || n_limbs < 1 || n_limbs > c->n_q) throw fides::Error(FIDES_ERR_ARG, "bad poly shape");
    std::vector<int> ids(n_limbs);
    for (int i = 0; i < n_limbs; ++i) ids[i] = i;
    fides::ntt_polys(c, data, n_polys, n_limbs, ids.data(), inverse != 0, S(stream));
  });
}

int fides_modup(fides_ctx* x, const uint64_t* in, int level, uint64_t* digits, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(in, "x");
    need(digits, "digits");
    fides::op_modup(c, in, level, digits, S(stream));
  });
}

int fides_ksk_inner_product(fides_ctx* x, const uint64_t* digits, int level, const uint64_t* key, uint64_t* out_a,
                            uint64_t* out_b, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(digits, "digits");
    need(out_a, "out_a");
    need(out_b, "out_b");
    fides::op_ksk_ip(c, nullptr, digits, level, key, out_a, out_b, S(stream));
  });
}

int fides_moddown(fides_ctx* x, const uint64_t* x_ext, int level, uint64_t* out, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(x_ext, "x_ext");
    need(out, "out");
    fides::op_moddown(c, x_ext, level, out, S(stream));
  });
}

int fides_keyswitch(fides_ctx* x, const uint64_t* d, int level, const uint64_t* key, uint64_t* f0, uint64_t* f1,
                    void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(d, "d");
    need(f0, "f0");
    need(f1, "f1");
    fides::KeySwitchItem it{d, level, key, f0, f1};
    fides::op_keyswitch_batch(c, &it, 1, S(stream));
  });
}

int fides_tensor(fides_ctx* x, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1,
                 int level, uint64_t* d0, uint64_t* d1, uint64_t* d2, void* stream) {
  return guard([&] {
    auto* c = C(x);
    for (const void* p : {(const void*)a0, (const void*)a1, (const void*)b0, (const void*)b1, (const void*)d0,
                          (const void*)d1, (const void*)d2})
      need(p, "tensor operand");
    fides::op_tensor(c, a0, a1, b0, b1, level, d0, d1, d2, S(stream));
  });
}

static int addsub(fides_ctx* x, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream,
                  int sub) {
  return guard([&] {
    auto* c = C(x);
    need(a, "a");
    need(b, "b");
    need(out, "out");
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    fides::AddSubJob j{a, b, out, level, sub};
    fides::launch_addsub(c, &j, 1, S(stream));
  });
}

int fides_mul(fides_ctx* x, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream) {
  return addsub(x, a, b, level, out, stream, fides::EW_MUL);
}

int fides_add_ext(fides_ctx* x, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(a, "a");
    need(b, "b");
    need(out, "out");
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (c->K < 1) throw fides::Error(FIDES_ERR_ARG, "extended basis needs special primes");
    fides::AddSubJob j{a, b, out, level + c->K, fides::EW_ADD, level, c->n_q};
    fides::launch_addsub(c, &j, 1, S(stream));
  });
}

static int dot_plain_impl(fides_ctx* x, const uint64_t* const* c0s, const uint64_t* const* c1s,
                          const uint64_t* const* pts, int n_terms, int level, uint64_t* out0, uint64_t* out1,
                          void* stream, bool ext) {
  return guard([&] {
    auto* c = C(x);
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (n_terms < 1 || n_terms > fides::MAX_DOT_TERMS) throw fides::Error(FIDES_ERR_ARG, "need 1..32 terms");
    need(c0s, "c0s");
    need(c1s, "c1s");
    need(pts, "pts");
    need(out0, "out0");
    need(out1, "out1");
    fides::DotJob j{};
    for (int t = 0; t < n_terms; ++t) {
      need(c0s[t], "c0s[t]");
      need(c1s[t], "c1s[t]");
      need(pts[t], "pts[t]");
      j.c0[0][t] = c0s[t];
      j.c1[0][t] = c1s[t];
      j.pt[t] = pts[t];
    }
    j.out0[0] = out0;
    j.out1[0] = out1;
    j.n = n_terms;
    j.l = ext ? level + c->K : level;
    if (ext) {
      if (c->K < 1) throw fides::Error(FIDES_ERR_ARG, "extended basis needs special primes");
      j.lq = level;
      j.nq = c->n_q;
    }
    j.lanes = 1;
    fides::launch_dot_plain(c, j, S(stream));
  });
}

int fides_dot_plain(fides_ctx* x, const uint64_t* const* c0s, const uint64_t* const* c1s, const uint64_t* const* pts,
                    int n_terms, int level, uint64_t* out0, uint64_t* out1, void* stream) {
  return dot_plain_impl(x, c0s, c1s, pts, n_terms, level, out0, out1, stream, false);
}

int fides_dot_plain_ext(fides_ctx* x, const uint64_t* const* c0s, const uint64_t* const* c1s,
                        const uint64_t* const* pts, int n_terms, int level, uint64_t* out0, uint64_t* out1,
                        void* stream) {
  return dot_plain_impl(x, c0s, c1s, pts, n_terms, level, out0, out1, stream, true);
}

int fides_dot_plain_bsgs(fides_ctx* x, const uint64_t* const* x0s, const uint64_t* const* x1s, int n_baby,
                         const uint64_t* const* pts, int n_giant, int level, int ext, uint64_t* const* out0s,
                         uint64_t* const* out1s, void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (n_baby < 1 || n_baby > fides::MAX_BSGS_BABY || n_giant < 1 || n_giant > fides::MAX_BSGS_GIANT)
      throw fides::Error(FIDES_ERR_ARG, "need 1..16 baby steps and 1..16 giant steps");
    if (ext && c->K < 1) throw fides::Error(FIDES_ERR_ARG, "extended basis needs special primes");
    need(x0s, "x0s");
    need(x1s, "x1s");
    need(pts, "pts");
    need(out0s, "out0s");
    need(out1s, "out1s");
    fides::BsgsJob j{};
    for (int k = 0; k < n_baby; ++k) {
      need(x0s[k], "x0s[k]");
      need(x1s[k], "x1s[k]");
      j.x0[0][k] = x0s[k];
      j.x1[0][k] = x1s[k];
    }
    for (int i = 0; i < n_giant; ++i) {
      need(out0s[i], "out0s[i]");
      need(out1s[i], "out1s[i]");
      j.out0[0][i] = out0s[i];
      j.out1[0][i] = out1s[i];
      for (int k = 0; k < n_baby; ++k) j.pt[i][k] = pts[(size_t)i * n_baby + k];
    }
    j.nb = n_baby;
    j.ng = n_giant;
    j.lanes = 1;
    j.l = ext ? level + c->K : level;
    if (ext) {
      j.lq = level;
      j.nq = c->n_q;
    }
    fides::launch_bsgs_dot(c, j, S(stream));
  });
}

int fides_lincomb(fides_ctx* x, int n_lanes, const uint64_t* const* c0s, const uint64_t* const* c1s,
                  const uint64_t* scalars, const uint64_t* add0, int n_terms, int level, uint64_t* const* out0s,
                  uint64_t* const* out1s, void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (level < 1 || level > c->n_q || level > fides::MAX_LC_LIMBS)
      throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (n_terms < 1 || n_terms > fides::MAX_LC_TERMS) throw fides::Error(FIDES_ERR_ARG, "need 1..16 terms");
    if (n_lanes < 1 || n_lanes > fides::MAX_LC_LANES) throw fides::Error(FIDES_ERR_ARG, "need 1..8 lanes");
    need(c0s, "c0s");
    need(c1s, "c1s");
    need(scalars, "scalars");
    need(out0s, "out0s");
    need(out1s, "out1s");
    static thread_local fides::LinCombJob j;
    j.lq = j.nq = 0;  // Q limbs only
    for (int a = 0; a < n_lanes; ++a) {
      need(out0s[a], "out0s[lane]");
      need(out1s[a], "out1s[lane]");
      j.out0[a] = out0s[a];
      j.out1[a] = out1s[a];
      for (int t = 0; t < n_terms; ++t) {
        const int k = a * n_terms + t;
        need(c0s[k], "c0s[lane * n_terms + t]");
        need(c1s[k], "c1s[lane * n_terms + t]");
        j.x0[a][t] = c0s[k];
        j.x1[a][t] = c1s[k];
      }
    }
    for (int t = 0; t < n_terms; ++t)
      for (int i = 0; i < level; ++i) {
        const uint64_t v = scalars[(size_t)t * level + i];
        if (v >= c->primes[i]) throw fides::Error(FIDES_ERR_ARG, "scalar not reduced mod q_i");
        j.s[t][i] = v;
      }
    for (int i = 0; i < level; ++i) {
      const uint64_t v = add0 ? add0[i] : 0;
      if (v >= c->primes[i]) throw fides::Error(FIDES_ERR_ARG, "add0 not reduced mod q_i");
      j.add0[i] = v;
    }
    j.n = n_terms;
    j.l = level;
    j.lanes = n_lanes;
    fides::launch_lincomb(c, j, S(stream));
  });
}

int fides_rescale_batch(fides_ctx* x, const uint64_t* const* xs, const int* levels, uint64_t* const* outs, int n,
                        void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "n < 0");
    if (n == 0) return;
    need(xs, "xs");
    need(levels, "levels");
    need(outs, "outs");
    for (int i = 0; i < n; ++i) {
      need(xs[i], "xs[i]");
      need(outs[i], "outs[i]");
      if (levels[i] < 2 || levels[i] > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    }
    fides::op_rescale_batch(c, xs, levels, outs, n, S(stream));
  });
}

int fides_encode(fides_ctx* x, const double* slots, int n_slots, int n_pts, double scale, int level, uint64_t* out,
                 void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(slots, "slots");
    need(out, "out");
    fides::op_encode(c, slots, n_slots, n_pts, scale, level, out, S(stream));
  });
}

int fides_encode_ext(fides_ctx* x, const double* slots, int n_slots, int n_pts, double scale, int level, uint64_t* out,
                     void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(slots, "slots");
    need(out, "out");
    if (c->K < 1) throw fides::Error(FIDES_ERR_ARG, "extended basis needs special primes");
    fides::op_encode_ext(c, slots, n_slots, n_pts, scale, level, c->K, out, S(stream));
  });
}

int fides_decode(fides_ctx* x, const uint64_t* pts, int level, int n_pts, int n_slots, double scale, double* slots,
                 void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(pts, "pts");
    need(slots, "slots");
    fides::op_decode(c, pts, level, n_pts, n_slots, scale, slots, S(stream));
  });
}

int fides_ct_import(fides_ctx* x, int n_polys, const uint64_t* const* limbs, const uint64_t* moduli, int level,
                    int format, int natural_order, uint64_t* out, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(limbs, "limbs");
    need(out, "out");
    if (format != 0 && format != 1) throw fides::Error(FIDES_ERR_ARG, "format must be 0 (EVAL) or 1 (COEFF)");
    fides::op_ct_import(c, n_polys, limbs, moduli, level, format, natural_order != 0, out, S(stream));
  });
}

int fides_ct_export(fides_ctx* x, int n_polys, const uint64_t* in, int level, int format, int natural_order,
                    uint64_t* const* limbs, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(in, "in");
    need(limbs, "limbs");
    if (format != 0 && format != 1) throw fides::Error(FIDES_ERR_ARG, "format must be 0 (EVAL) or 1 (COEFF)");
    fides::op_ct_export(c, n_polys, in, level, format, natural_order != 0, limbs, S(stream));
    check_device_status(c);
  });
}

int fides_key_import(fides_ctx* x, const uint64_t* const* limbs, int natural_order, uint64_t** dev_key) {
  return guard([&] {
    auto* c = C(x);
    need(limbs, "limbs");
    need(dev_key, "dev_key");
    *dev_key = fides::op_key_import(c, limbs, natural_order != 0, nullptr);
  });
}

static int scalar_op(fides_ctx* x, const uint64_t* a, int level, const uint64_t* scalars, uint64_t* out,
                     void* stream, int op) {
  return guard([&] {
    auto* c = C(x);
    need(a, "a");
    need(scalars, "scalars");
    need(out, "out");
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (level > fides::MAX_SCALAR_LIMBS) throw fides::Error(FIDES_ERR_ARG, "scalar ops support at most 64 limbs");
    fides::ScalarJob j{};
    j.a = a;
    j.out = out;
    j.l = level;
    j.op = op;
    for (int i = 0; i < level; ++i) j.s[i] = scalars[i] % c->primes[i];
    fides::launch_scalar(c, &j, 1, S(stream));
  });
}

int fides_mul_scalar(fides_ctx* x, const uint64_t* a, int level, const uint64_t* scalars, uint64_t* out,
                     void* stream) {
  return scalar_op(x, a, level, scalars, out, stream, fides::EW_MUL_SCALAR);
}

int fides_add_scalar(fides_ctx* x, const uint64_t* a, int level, const uint64_t* scalars, uint64_t* out,
                     void* stream) {
  return scalar_op(x, a, level, scalars, out, stream, fides::EW_ADD_SCALAR);
}

int fides_mod_raise(fides_ctx* x, const uint64_t* in, int out_level, uint64_t* out, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(in, "x");
    need(out, "out");
    if (out == in) throw fides::Error(FIDES_ERR_ARG, "out must not alias the input limb");
    fides::op_mod_raise(c, in, out_level, out, S(stream));
  });
}

int fides_add(fides_ctx* x, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream) {
  return addsub(x, a, b, level, out, stream, fides::EW_ADD);
}

int fides_sub(fides_ctx* x, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, void* stream) {
  return addsub(x, a, b, level, out, stream, fides::EW_SUB);
}

int fides_rescale(fides_ctx* x, const uint64_t* in, int level, uint64_t* out, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(in, "x");
    need(out, "out");
    uint64_t* o = out;
    fides::op_rescale_batch(c, &in, &level, &o, 1, S(stream));
  });
}

int fides_hmult(fides_ctx* x, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1,
                int level, const uint64_t* relin_key, int rescale, uint64_t* out0, uint64_t* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    for (const void* p : {(const void*)a0, (const void*)a1, (const void*)b0, (const void*)b1, (const void*)out0,
                          (const void*)out1})
      need(p, "hmult operand");
    fides::HMultItem it{a0, a1, b0, b1, out0, out1, level};
    fides::op_hmult_batch(c, &it, 1, relin_key, rescale != 0, S(stream));
  });
}

int fides_rotate_auto(fides_ctx* x, const uint64_t* c0, const uint64_t* c1, int level, const uint64_t* key,
                      uint32_t auto_index, uint64_t* out0, uint64_t* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(c0, "c0");
    need(c1, "c1");
    need(out0, "out0");
    need(out1, "out1");
    if ((auto_index & 1) == 0 || auto_index >= 2u * (uint32_t)c->N)
      throw fides::Error(FIDES_ERR_ARG, "automorphism index must be odd and < 2N");
    fides::RotateItem it{c0, c1, out0, out1, key, level, auto_index};
    fides::op_rotate_batch(c, &it, 1, S(stream));
  });
}

int fides_rotate(fides_ctx* x, const uint64_t* c0, const uint64_t* c1, int level, const uint64_t* rot_key,
                 int rotation, uint64_t* out0, uint64_t* out1, void* stream) {
  if (!x || !x->c) {
    g_err = "null context";
    return FIDES_ERR_ARG;
  }
  return fides_rotate_auto(x, c0, c1, level, rot_key, fides::h_auto_index(x->c->logN, rotation), out0, out1,
                           stream);
}

int fides_rotate_hoisted(fides_ctx* x, const uint64_t* c0, const uint64_t* c1, int level,
                         const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                         uint64_t* const* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(c0, "c0");
    need(c1, "c1");
    need(keys, "keys");
    need(rotations, "rotations");
    need(out0, "out0");
    need(out1, "out1");
    fides::HoistItem it;
    it.c0 = c0;
    it.c1 = c1;
    it.l = level;
    for (int j = 0; j < n; ++j) {
      need(out0[j], "out0[j]");
      need(out1[j], "out1[j]");
      it.keys.push_back(keys[j]);
      it.ks.push_back(fides::h_auto_index(c->logN, rotations[j]));
      it.out0.push_back(out0[j]);
      it.out1.push_back(out1[j]);
    }
    fides::op_hoisted(c, it, S(stream));
  });
}

int fides_rotate_hoisted_ext(fides_ctx* x, const uint64_t* c0, int c0_ext, const uint64_t* c1, int level,
                             const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                             uint64_t* const* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(c0, "c0");
    need(c1, "c1");
    need(keys, "keys");
    need(rotations, "rotations");
    need(out0, "out0");
    need(out1, "out1");
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (n < 1) throw fides::Error(FIDES_ERR_ARG, "need at least one rotation");
    fides::HoistItem it;
    it.c0 = c0_ext ? nullptr : c0;
    it.c0x = c0_ext ? c0 : nullptr;
    it.c1 = c1;
    it.l = level;
    for (int j = 0; j < n; ++j) {
      need(out0[j], "out0[j]");
      need(out1[j], "out1[j]");
      need(keys[j], "keys[j]");
      it.keys.push_back(keys[j]);
      it.ks.push_back(fides::h_auto_index(c->logN, rotations[j]));
      it.out0.push_back(out0[j]);
      it.out1.push_back(out1[j]);
    }
    fides::op_hoisted_ext_batch(c, &it, 1, S(stream));
  });
}

int fides_accumulate_rotations(int radix, int stride, int size, int* indices, int cap) {
  if (radix < 2 || (radix & (radix - 1)) || stride < 1 || size < 1 || (cap > 0 && !indices)) return FIDES_ERR_ARG;
  int n = 0;
  for (long t = 1; t < size; t *= radix)
    for (int k = 1; k < radix && (long)stride * t * k < (long)stride * size; ++k) {
      if (n < cap) indices[n] = (int)(stride * t * k);
      ++n;
    }
  return n;
}

int fides_accumulate(fides_ctx* x, const uint64_t* c0, const uint64_t* c1, int level, int radix, int stride, int size,
                     const int* key_rotations, const uint64_t* const* keys, int n_keys, uint64_t* out0,
                     uint64_t* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(c0, "c0");
    need(c1, "c1");
    need(out0, "out0");
    need(out1, "out1");
    if (n_keys < 0 || (n_keys > 0 && (!key_rotations || !keys))) throw fides::Error(FIDES_ERR_ARG, "bad key table");
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    std::vector<std::pair<int, const uint64_t*>> kt;
    for (int i = 0; i < n_keys; ++i) {
      need(keys[i], "key");
      kt.push_back({key_rotations[i], keys[i]});
    }
    fides::op_accumulate(c, c0, c1, level, radix, stride, size, kt, out0, out1, S(stream));
  });
}

int fides_rotate_hoisted_digits(fides_ctx* x, const uint64_t* c0, const uint64_t* digits, int level,
                                const uint64_t* const* keys, const int* rotations, int n, uint64_t* const* out0,
                                uint64_t* const* out1, void* stream) {
  return guard([&] {
    auto* c = C(x);
    need(c0, "c0");
    need(digits, "digits");
    need(keys, "keys");
    need(rotations, "rotations");
    need(out0, "out0");
    need(out1, "out1");
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    std::vector<uint32_t> ks(n);
    for (int j = 0; j < n; ++j) {
      need(out0[j], "out0[j]");
      need(out1[j], "out1[j]");
      ks[j] = fides::h_auto_index(c->logN, rotations[j]);
    }
    fides::op_hoisted_digits(c, c0, digits, level, keys, ks.data(), n, out0, out1, S(stream));
  });
}

int fides_rotate_hoisted_batch(fides_ctx* x, const fides_hoist_item* items, int n_items, void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (n_items < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    if (n_items > 0) need(items, "items");
    std::vector<fides::HoistItem> v(n_items);
    for (int i = 0; i < n_items; ++i) {
      const fides_hoist_item& h = items[i];
      need(h.c0, "c0");
      need(h.c1, "c1");
      if (h.n < 0) throw fides::Error(FIDES_ERR_ARG, "negative rotation count");
      if (h.n > 0) {
        need(h.keys, "keys");
        need(h.rotations, "rotations");
        need(h.out0, "out0");
        need(h.out1, "out1");
      }
      v[i].c0 = h.c0;
      v[i].c1 = h.c1;
      v[i].l = h.level;
      for (int j = 0; j < h.n; ++j) {
        need(h.out0[j], "out0[j]");
        need(h.out1[j], "out1[j]");
        v[i].keys.push_back(h.keys[j]);
        v[i].ks.push_back(fides::h_auto_index(c->logN, h.rotations[j]));
        v[i].out0.push_back(h.out0[j]);
        v[i].out1.push_back(h.out1[j]);
      }
    }
    fides::op_hoisted_batch(c, v.data(), n_items, S(stream));
  });
}

int fides_hmult_batch(fides_ctx* x, const fides_hmult_item* items, int n, const uint64_t* relin_key, int rescale,
                      void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative batch");
    if (n && !items) throw fides::Error(FIDES_ERR_ARG, "null items");
    std::vector<fides::HMultItem> v(n);
    for (int i = 0; i < n; ++i) {
      const fides_hmult_item& s = items[i];
      for (const void* p : {(const void*)s.a0, (const void*)s.a1, (const void*)s.b0, (const void*)s.b1,
                            (const void*)s.out0, (const void*)s.out1})
        need(p, "hmult item operand");
      v[i] = fides::HMultItem{s.a0, s.a1, s.b0, s.b1, s.out0, s.out1, s.level};
    }
    fides::op_hmult_batch(c, v.data(), n, relin_key, rescale != 0, S(stream));
  });
}

int fides_mixed_batch(fides_ctx* x, const fides_hmult_item* hm, int n_hm, const uint64_t* relin_key, int rescale,
                      const fides_rotate_item* rot, int n_rot, void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (n_hm < 0 || n_rot < 0) throw fides::Error(FIDES_ERR_ARG, "negative batch");
    if ((n_hm && !hm) || (n_rot && !rot)) throw fides::Error(FIDES_ERR_ARG, "null items");
    std::vector<fides::HMultItem> vh(n_hm);
    for (int i = 0; i < n_hm; ++i) {
      const fides_hmult_item& s = hm[i];
      for (const void* p : {(const void*)s.a0, (const void*)s.a1, (const void*)s.b0, (const void*)s.b1,
                            (const void*)s.out0, (const void*)s.out1})
        need(p, "hmult item operand");
      vh[i] = fides::HMultItem{s.a0, s.a1, s.b0, s.b1, s.out0, s.out1, s.level};
    }
    std::vector<fides::RotateItem> vr(n_rot);
    for (int i = 0; i < n_rot; ++i) {
      const fides_rotate_item& s = rot[i];
      for (const void* p : {(const void*)s.c0, (const void*)s.c1, (const void*)s.out0, (const void*)s.out1})
        need(p, "rotate item operand");
      if ((s.auto_index & 1) == 0 || s.auto_index >= 2u * (uint32_t)c->N)
        throw fides::Error(FIDES_ERR_ARG, "automorphism index must be odd and < 2N");
      vr[i] = fides::RotateItem{s.c0, s.c1, s.out0, s.out1, s.key, s.level, s.auto_index};
    }
    fides::op_mixed_batch(c, vh.data(), n_hm, relin_key, rescale != 0, vr.data(), n_rot, S(stream));
  });
}

int fides_rotate_batch(fides_ctx* x, const fides_rotate_item* items, int n, void* stream) {
  return guard([&] {
    auto* c = C(x);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative batch");
    if (n && !items) throw fides::Error(FIDES_ERR_ARG, "null items");
    std::vector<fides::RotateItem> v(n);
    for (int i = 0; i < n; ++i) {
      const fides_rotate_item& s = items[i];
      for (const void* p : {(const void*)s.c0, (const void*)s.c1, (const void*)s.out0, (const void*)s.out1})
        need(p, "rotate item operand");
      if ((s.auto_index & 1) == 0 || s.auto_index >= 2u * (uint32_t)c->N)
        throw fides::Error(FIDES_ERR_ARG, "automorphism index must be odd and < 2N");
      v[i] = fides::RotateItem{s.c0, s.c1, s.out0, s.out1, s.key, s.level, s.auto_index};
    }
    fides::op_rotate_batch(c, v.data(), n, S(stream));
  });
}

int fides_key_upload(fides_ctx* x, const uint64_t* host_key, uint64_t** dev_key) {
  return guard([&] {
    auto* c = C(x);
    need(host_key, "host_key");
    need(dev_key, "dev_key");
    size_t bytes = sizeof(uint64_t) * 2 * (size_t)c->dnum * (c->n_q + c->K) * c->N;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw fides::Error(FIDES_ERR_OOM, std::string("key allocation failed: ") + cudaGetErrorString(e));
    }
    e = cudaMemcpy(p, host_key, bytes, cudaMemcpyDefault);  // host or device source (unified addressing)
    if (e != cudaSuccess) {
      cudaFree(p);
      throw fides::Error(FIDES_ERR_CUDA, std::string("key upload failed: ") + cudaGetErrorString(e));
    }
    *dev_key = static_cast<uint64_t*>(p);
  });
}

int fides_key_free(fides_ctx* x, uint64_t* dev_key) {
  return guard([&] {
    C(x);
    if (dev_key) FIDES_CUDA(cudaFree(dev_key));
  });
}

}  // extern "C"

namespace {
// Host-buffer round trip: H2D inputs, op on device scratch, D2H outputs, synchronise.
template <typename Op>
void host_roundtrip(fides_ctx* x, const std::vector<const uint64_t*>& ins, int in_limbs, int n_out, int out_limbs,
                    const std::vector<uint64_t*>& outs, Op&& op) {
  auto* c = C(x);
  const size_t N = c->N;
  cudaStream_t s = x->host_stream;
  size_t total = (size_t)ins.size() * in_limbs + (size_t)n_out * out_limbs;
  fides::Scratch sc(c, sizeof(uint64_t) * N * total, s);
  std::vector<uint64_t*> din(ins.size()), dout(n_out);
  uint64_t* p = sc.u64();
  for (size_t i = 0; i < ins.size(); ++i) {
    need(ins[i], "host input");
    din[i] = p;
    p += (size_t)in_limbs * N;
    FIDES_CUDA(cudaMemcpyAsync(din[i], ins[i], sizeof(uint64_t) * N * in_limbs, cudaMemcpyHostToDevice, s));
  }
  for (int i = 0; i < n_out; ++i) {
    need(outs[i], "host output");
    dout[i] = p;
    p += (size_t)out_limbs * N;
  }
  op(din, dout, s);
  for (int i = 0; i < n_out; ++i)
    FIDES_CUDA(cudaMemcpyAsync(outs[i], dout[i], sizeof(uint64_t) * N * out_limbs, cudaMemcpyDeviceToHost, s));
  FIDES_CUDA(cudaStreamSynchronize(s));
  check_device_status(c);
}
// One item of a pipelined host batch: its host inputs and outputs (limb counts each).
struct HostJob {
  std::vector<const uint64_t*> in;
  int in_limbs;
  std::vector<uint64_t*> out;
  int out_limbs;
};

// Waits for every pipelined host batch enqueued on the context and reports its status.
void host_pipeline_wait(fides_ctx* x) {
  cudaError_t e1 = cudaStreamSynchronize(x->h2d_stream), e2 = cudaStreamSynchronize(x->host_stream),
              e3 = cudaStreamSynchronize(x->d2h_stream);
  FIDES_CUDA(e1);
  FIDES_CUDA(e2);
  FIDES_CUDA(e3);
  check_device_status(x->c);
}

// Pipelined host batch: item k's host->device copies (h2d stream), computation (host
// stream) and device->host copies (d2h stream) are ordered by events, so copies of
// neighbouring items run on the copy engines under item k's kernels.  The context's device
// slots rotate across items and across calls; a slot is reused once its previous item's
// device->host copies are done.  With `wait` it returns after the last copy completes;
// otherwise it returns once everything is enqueued (the host buffers must stay valid until
// host_pipeline_wait).  Host buffers should be pinned for the copies to overlap.
template <typename Op>
void host_pipeline(fides_ctx* x, const std::vector<HostJob>& jobs, Op&& op, bool wait = true) {
  auto* c = C(x);
  const size_t N = c->N;
  const int n = (int)jobs.size();
  if (n == 0) {
    if (wait) host_pipeline_wait(x);
    return;
  }
  constexpr int SLOTS = fides_ctx::kPipeSlots;
  size_t slot_limbs = 0;
  for (const auto& j : jobs) {
    for (auto* p : j.in) need(p, "host input");
    for (auto* p : j.out) need(p, "host output");
    slot_limbs = std::max(slot_limbs, j.in.size() * (size_t)j.in_limbs + j.out.size() * (size_t)j.out_limbs);
  }
  cudaStream_t sh = x->h2d_stream, sc = x->host_stream, sd = x->d2h_stream;
  const size_t slot_bytes = sizeof(uint64_t) * N * slot_limbs;
  if (x->pipe_slot_bytes < slot_bytes) {  // grow the slots once the earlier items are done
    host_pipeline_wait(x);
    if (x->pipe_mem) FIDES_CUDA(cudaFree(x->pipe_mem));
    x->pipe_mem = nullptr;
    x->pipe_slot_bytes = 0;
    FIDES_CUDA(cudaMalloc(&x->pipe_mem, slot_bytes * SLOTS));
    x->pipe_slot_bytes = slot_bytes;
    for (bool& u : x->pipe_used) u = false;
  }
  for (int i = 0; i < SLOTS; ++i)
    for (cudaEvent_t* e : {&x->pipe_free[i], &x->pipe_in_ready[i], &x->pipe_computed[i]})
      if (!*e) FIDES_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  try {
    for (int k = 0; k < n; ++k) {
      const HostJob& j = jobs[k];
      const int slot = (int)(x->pipe_next++ % SLOTS);
      uint64_t* base = reinterpret_cast<uint64_t*>(static_cast<char*>(x->pipe_mem) + (size_t)slot * x->pipe_slot_bytes);
      if (x->pipe_used[slot]) FIDES_CUDA(cudaStreamWaitEvent(sh, x->pipe_free[slot], 0));
      std::vector<uint64_t*> din(j.in.size()), dout(j.out.size());
      uint64_t* p = base;
      for (size_t i = 0; i < j.in.size(); ++i, p += (size_t)j.in_limbs * N) {
        din[i] = p;
        FIDES_CUDA(cudaMemcpyAsync(p, j.in[i], sizeof(uint64_t) * N * j.in_limbs, cudaMemcpyHostToDevice, sh));
      }
      for (size_t i = 0; i < j.out.size(); ++i, p += (size_t)j.out_limbs * N) dout[i] = p;
      FIDES_CUDA(cudaEventRecord(x->pipe_in_ready[slot], sh));
      FIDES_CUDA(cudaStreamWaitEvent(sc, x->pipe_in_ready[slot], 0));
      op(k, din, dout, sc);
      FIDES_CUDA(cudaEventRecord(x->pipe_computed[slot], sc));
      FIDES_CUDA(cudaStreamWaitEvent(sd, x->pipe_computed[slot], 0));
      for (size_t i = 0; i < j.out.size(); ++i)
        FIDES_CUDA(cudaMemcpyAsync(j.out[i], dout[i], sizeof(uint64_t) * N * j.out_limbs, cudaMemcpyDeviceToHost,
                                   sd));
      FIDES_CUDA(cudaEventRecord(x->pipe_free[slot], sd));
      x->pipe_used[slot] = true;
    }
  } catch (...) {
    // every stream drains before the error is reported, so no copy outlives the call
    cudaStreamSynchronize(sh);
    cudaStreamSynchronize(sc);
    cudaStreamSynchronize(sd);
    throw;
  }
  if (wait) host_pipeline_wait(x);
}
}  // namespace

extern "C" {

int fides_hmult_host_batch(fides_ctx* x, const fides_hmult_host_item* items, int n, const uint64_t* relin_key_dev,
                           int rescale) {
  return guard([&] {
    auto* c = C(x);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    if (n > 0) need(items, "items");
    std::vector<HostJob> jobs(n);
    for (int k = 0; k < n; ++k) {
      const auto& it = items[k];
      if (it.level < (rescale ? 2 : 1) || it.level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
      jobs[k] = HostJob{{it.a0, it.a1, it.b0, it.b1}, it.level, {it.out0, it.out1}, rescale ? it.level - 1 : it.level};
    }
    host_pipeline(x, jobs, [&](int k, std::vector<uint64_t*>& in, std::vector<uint64_t*>& out, cudaStream_t s) {
      fides::HMultItem h{in[0], in[1], in[2], in[3], out[0], out[1], items[k].level};
      fides::op_hmult_batch(c, &h, 1, relin_key_dev, rescale != 0, s);
    });
  });
}

int fides_rotate_host_batch(fides_ctx* x, const fides_rotate_host_item* items, int n) {
  return guard([&] {
    auto* c = C(x);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    if (n > 0) need(items, "items");
    std::vector<HostJob> jobs(n);
    for (int k = 0; k < n; ++k) {
      const auto& it = items[k];
      if (it.level < 1 || it.level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
      jobs[k] = HostJob{{it.c0, it.c1}, it.level, {it.out0, it.out1}, it.level};
    }
    host_pipeline(x, jobs, [&](int k, std::vector<uint64_t*>& in, std::vector<uint64_t*>& out, cudaStream_t s) {
      const auto& it = items[k];
      fides::RotateItem r{in[0], in[1], out[0], out[1], it.rot_key_dev, it.level,
                          fides::h_auto_index(c->logN, it.rotation)};
      fides::op_rotate_batch(c, &r, 1, s);
    });
  });
}

}  // extern "C"

namespace {
void mixed_host_batch(fides_ctx* x, const fides_hmult_host_item* hm, int n_hm, const uint64_t* relin_key_dev,
                      int rescale, const fides_rotate_host_item* rot, int n_rot, bool wait) {
  {
    auto* c = C(x);
    if (n_hm < 0 || n_rot < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    if (n_hm > 0) {
      need(hm, "hmult items");
      need(relin_key_dev, "relin_key_dev");
    }
    if (n_rot > 0) need(rot, "rotate items");
    // one pipeline, the two kinds interleaved: an HMult moves twice the host->device bytes of
    // a rotation for the same device->host bytes, so alternating them keeps both copy
    // directions busy, and one pipeline fills and drains once; a rotation goes first, so the
    // fill (the first item's host->device copies, which nothing overlaps) is the shorter one
    std::vector<HostJob> jobs;
    std::vector<std::pair<int, int>> which;  // (kind, index)
    for (int i = 0, j = 0; i < n_hm || j < n_rot;) {
      if (j < n_rot) {
        const auto& it = rot[j];
        if (it.level < 1 || it.level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
        need(it.rot_key_dev, "rot_key_dev");
        jobs.push_back(HostJob{{it.c0, it.c1}, it.level, {it.out0, it.out1}, it.level});
        which.push_back({1, j++});
      }
      if (i < n_hm) {
        const auto& it = hm[i];
        if (it.level < (rescale ? 2 : 1) || it.level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
        jobs.push_back(HostJob{{it.a0, it.a1, it.b0, it.b1}, it.level, {it.out0, it.out1},
                               rescale ? it.level - 1 : it.level});
        which.push_back({0, i++});
      }
    }
    host_pipeline(x, jobs, [&](int k, std::vector<uint64_t*>& in, std::vector<uint64_t*>& out, cudaStream_t s) {
      if (which[k].first == 0) {
        fides::HMultItem h{in[0], in[1], in[2], in[3], out[0], out[1], hm[which[k].second].level};
        fides::op_hmult_batch(c, &h, 1, relin_key_dev, rescale != 0, s);
      } else {
        const auto& it = rot[which[k].second];
        fides::RotateItem r{in[0], in[1], out[0], out[1], it.rot_key_dev, it.level,
                            fides::h_auto_index(c->logN, it.rotation)};
        fides::op_rotate_batch(c, &r, 1, s);
      }
    }, wait);
  }
}
}  // namespace

extern "C" {

int fides_mixed_host_batch(fides_ctx* x, const fides_hmult_host_item* hm, int n_hm, const uint64_t* relin_key_dev,
                           int rescale, const fides_rotate_host_item* rot, int n_rot) {
  return guard([&] { mixed_host_batch(x, hm, n_hm, relin_key_dev, rescale, rot, n_rot, true); });
}

int fides_mixed_host_batch_async(fides_ctx* x, const fides_hmult_host_item* hm, int n_hm,
                                 const uint64_t* relin_key_dev, int rescale, const fides_rotate_host_item* rot,
                                 int n_rot) {
  return guard([&] { mixed_host_batch(x, hm, n_hm, relin_key_dev, rescale, rot, n_rot, false); });
}

int fides_host_batch_wait(fides_ctx* x) {
  return guard([&] {
    C(x);
    host_pipeline_wait(x);
  });
}

int fides_hmult_host(fides_ctx* x, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1,
                     int level, const uint64_t* relin_key_dev, int rescale, uint64_t* out0, uint64_t* out1) {
  return guard([&] {
    auto* c = C(x);
    if (level < (rescale ? 2 : 1) || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    host_roundtrip(x, {a0, a1, b0, b1}, level, 2, rescale ? level - 1 : level, {out0, out1},
                   [&](std::vector<uint64_t*>& in, std::vector<uint64_t*>& out, cudaStream_t s) {
                     fides::HMultItem it{in[0], in[1], in[2], in[3], out[0], out[1], level};
                     fides::op_hmult_batch(c, &it, 1, relin_key_dev, rescale != 0, s);
                   });
  });
}

int fides_rotate_host(fides_ctx* x, const uint64_t* c0, const uint64_t* c1, int level, const uint64_t* rot_key_dev,
                      int rotation, uint64_t* out0, uint64_t* out1) {
  return guard([&] {
    auto* c = C(x);
    if (level < 1 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    host_roundtrip(x, {c0, c1}, level, 2, level, {out0, out1},
                   [&](std::vector<uint64_t*>& in, std::vector<uint64_t*>& out, cudaStream_t s) {
                     fides::RotateItem it{in[0], in[1], out[0], out[1], rot_key_dev, level,
                                          fides::h_auto_index(c->logN, rotation)};
                     fides::op_rotate_batch(c, &it, 1, s);
                   });
  });
}

struct fides_graph_impl {
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

int fides_capture_begin(fides_ctx* x, void* stream) {
  return guard([&] {
    C(x);
    if (!stream) throw fides::Error(FIDES_ERR_ARG, "capture needs a non-default stream");
    FIDES_CUDA(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeThreadLocal));
  });
}

int fides_capture_end(fides_ctx* x, void* stream, fides_graph** out) {
  return guard([&] {
    C(x);
    need(out, "out");
    cudaGraph_t g = nullptr;
    FIDES_CUDA(cudaStreamEndCapture(S(stream), &g));
    cudaGraphExec_t e = nullptr;
    cudaError_t rc = cudaGraphInstantiate(&e, g, 0);
    if (rc != cudaSuccess) {
      cudaGraphDestroy(g);
      throw fides::Error(FIDES_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(rc));
    }
    *out = reinterpret_cast<fides_graph*>(new fides_graph_impl{g, e});
  });
}

int fides_graph_launch(fides_graph* g, void* stream) {
  return guard([&] {
    need(g, "graph");
    FIDES_CUDA(cudaGraphLaunch(reinterpret_cast<fides_graph_impl*>(g)->exec, S(stream)));
  });
}

int fides_graph_destroy(fides_graph* g) {
  return guard([&] {
    if (!g) return;
    auto* G = reinterpret_cast<fides_graph_impl*>(g);
    cudaGraphExecDestroy(G->exec);
    cudaGraphDestroy(G->graph);
    delete G;
  });
}

}  // extern "C"

