// fides_rescale_noalloc: rescale without any device allocation.
//
// Some callers of this library cannot allocate device memory on the call path: a host
// whose HBM is entirely reserved up front by another allocator (a framework's caching
// pool, a per-tenant quota) sees every extra cudaMalloc fail even though its own pool
// has room, and a latency-bound serving loop cannot afford the device-wide
// synchronisation and driver locking that cudaMalloc / cudaFree bring.  For them this
// entry point takes its one limb of scratch (the top limb after the inverse NTT) from a
// fixed array compiled into the library instead of from an allocator.
//
// The array is a file-scope __device__ variable, so every GPU that loads the library
// holds it (512 KiB) until the process exits, and every call on a device uses the same
// array: calls that overlap on the GPU (different streams, no ordering between them)
// race on it.  Each call overwrites the whole limb it uses before reading it, so no state
// from an earlier call leaks into a result.
//
// In host code the array's name is only a stand-in; its device address comes from
// cudaGetSymbolAddress, looked up on the first call on each device (with that device
// current) and cached.  That first call should therefore come before any stream capture.
#include <algorithm>
#include <mutex>

#include "../../include/fides_b200.h"
#include "capi_internal.hpp"
#include "ntt.cuh"
#include "ops.hpp"

namespace {

constexpr int kMaxLogN = 16;  // the array holds one limb of up to 2^16 words (512 KiB)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint64_t g_rescale_scratch[size_t(1) << kMaxLogN];

std::mutex g_mu;
uint64_t* g_scratch[kMaxDevices] = {};

// Device address of g_rescale_scratch on `device` (which must be current).
uint64_t* scratch_on(int device) {
  if (device < 0 || device >= kMaxDevices) throw fides::Error(FIDES_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_rescale_scratch);
    if (e != cudaSuccess)
      throw fides::Error(FIDES_ERR_CUDA, std::string("cudaGetSymbolAddress(rescale scratch): ") + cudaGetErrorString(e));
    g_scratch[device] = static_cast<uint64_t*>(p);
  }
  return g_scratch[device];
}

}  // namespace

extern "C" int fides_rescale_noalloc(fides_ctx* x, const uint64_t* in, int level, uint64_t* out, void* stream) {
  // the caller's current device is restored on return, as by every other entry point
  struct RestoreDevice {
    int prev = -1;
    RestoreDevice() {
      if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~RestoreDevice() {
      if (prev >= 0) cudaSetDevice(prev);
    }
  } restore;
  try {
    if (!x || !x->c) throw fides::Error(FIDES_ERR_ARG, "null context");
    fides::Context* c = x->c;
    if (!in || !out) throw fides::Error(FIDES_ERR_ARG, "null polynomial pointer");
    if (c->logN > kMaxLogN)
      throw fides::Error(FIDES_ERR_ARG, "fides_rescale_noalloc supports N <= 2^16 (its static scratch holds one limb of "
                                        "2^16 words); use fides_rescale for larger rings");
    if (level < 2 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    const size_t N = c->N;
    const uint64_t *i0 = in, *i1 = in + (size_t)level * N;
    const uint64_t *o0 = out, *o1 = out + (size_t)(level - 1) * N;
    if (o0 < i1 && i0 < o1)
      throw fides::Error(FIDES_ERR_ARG, "fides_rescale_noalloc: out must not overlap the input");
    FIDES_CUDA(cudaSetDevice(c->device));
    uint64_t* top = scratch_on(c->device);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // INTT of the top limb into the static scratch, then one forward NTT per remaining limb
    // whose prologue applies SwitchModulus to that limb and whose epilogue forms
    // q_l^-1 x_j + QlQlInvModqlDivqlModq_j t_j: the launches fides_rescale makes, built by the
    // same helpers.  The limb descriptors go through a fixed array in chunks, so no level is
    // too large for it and nothing is allocated on the host either.
    fides::LimbRef r = fides::rescale_top_ref(c, in, level, top);
    fides::ntt_limbs(c, &r, 1, true, s);
    constexpr int kChunk = 128;
    fides::LimbRef refs[kChunk];
    for (int j0 = 0; j0 < level - 1; j0 += kChunk) {
      const int m = std::min(kChunk, level - 1 - j0);
      for (int k = 0; k < m; ++k) refs[k] = fides::rescale_limb_ref(c, in, level, top, out + (size_t)(j0 + k) * N, j0 + k);
      fides::ntt_limbs(c, refs, m, false, s, fides::IN_SWITCH, fides::OUT_RESCALE);
    }
    return FIDES_OK;
  } catch (const fides::Error& e) {
    fides::set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    fides::set_last_error(e.what());
    return FIDES_ERR_STATE;
  }
}
