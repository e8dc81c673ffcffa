// NTT tile-shape autotuner.  For each direction, pass and launch-size class, time the
// transform on device-resident synthetic limbs with every supported sub-transforms-per-CTA
// (4, 8, 16) and residues per thread (16; also 8 at N >= 2^15, i.e. three butterfly stages
// per register chunk instead of four) and keep the fastest in the context's tables
// (Context::ntt_g, Context::ntt_r).  Both change only how the butterflies are distributed
// over threads and CTAs, never the arithmetic, so results are identical whatever the tables
// hold.
#include <algorithm>
#include <vector>

#include "autotune.hpp"
#include "ntt.cuh"

namespace fides {
namespace {

// Residues in [0, q) of the limb's prime (a SplitMix64 stream reduced modulo q).
__global__ void fill_residues(uint64_t* x, const DevPrime* primes, const int* prime_of_limb, int logN) {
  const size_t i = (size_t)blockIdx.y << logN | (blockIdx.x * blockDim.x + threadIdx.x);
  uint64_t z = i * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  x[i] = z % primes[prime_of_limb[blockIdx.y]].q;
}

constexpr int SIZES[4] = {4, 16, 64, 256};  // one representative launch per size class
constexpr int SHAPES[3] = {4, 8, 16};
// chunk sizes tried on a list of MAX_NTT_LIMBS limbs (a launch of 224 MB at N = 2^16)
constexpr int CHUNKS[6] = {0, 224, 160, 112, 80, 56};

}  // namespace

void autotune_ntt(Context* c, float* best_ms) {
  const int max_limbs = MAX_NTT_LIMBS;
  const int np = c->n_q + c->K;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FIDES_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  FIDES_CUDA(cudaEventCreate(&e0));
  FIDES_CUDA(cudaEventCreate(&e1));
  uint8_t saved[2][2][4], saved_r[2][2][4];
  std::copy(&c->ntt_g[0][0][0], &c->ntt_g[0][0][0] + 16, &saved[0][0][0]);
  std::copy(&c->ntt_r[0][0][0], &c->ntt_r[0][0][0] + 16, &saved_r[0][0][0]);
  const bool r8 = c->logN >= 15;  // passes with 8 residues per thread exist (ntt_impl.cuh HasLe3)
  const int saved_chunk = c->ntt_chunk;
  c->ntt_chunk = 0;  // the shapes are timed on unsplit launches
  const bool saved_profiling = c->profiling;
  c->profiling = false;  // no profiling events inside the timing graphs
  try {
    Scratch data(c, c->limb_bytes() * max_limbs, s);
    Scratch ids(c, sizeof(int) * max_limbs, s);
    std::vector<int> h_ids(max_limbs);
    for (int i = 0; i < max_limbs; ++i) h_ids[i] = i % np;
    FIDES_CUDA(cudaMemcpyAsync(ids.p, h_ids.data(), sizeof(int) * max_limbs, cudaMemcpyHostToDevice, s));
    const int threads = std::min(256, c->N);
    fill_residues<<<dim3(c->N / threads, max_limbs), threads, 0, s>>>(data.u64(), c->d_prime,
                                                                     static_cast<const int*>(ids.p), c->logN);
    FIDES_CUDA(cudaGetLastError());
    std::vector<LimbRef> refs(max_limbs);
    for (int i = 0; i < max_limbs; ++i) refs[i] = lref(data.u64() + (size_t)i * c->N, h_ids[i]);
    for (int inv = 0; inv < 2; ++inv)
      for (int cls = 0; cls < 4; ++cls) {
        const int n = SIZES[cls];
        // Device time of one transform: kReps round trips (the tuned direction, then the other
        // one, which keeps the data reduced) replayed from a CUDA graph, so that host launch
        // overhead, which exceeds the GPU time of a launch of a few limbs, does not decide
        // between the candidates.  One round trip runs uncaptured first (each kernel's first
        // launch sets its shared-memory attribute).
        auto time_it = [&] {
          constexpr int kReps = 8;
          ntt_limbs(c, refs.data(), n, inv != 0, s);
          ntt_limbs(c, refs.data(), n, inv == 0, s);
          cudaGraph_t graph = nullptr;
          cudaGraphExec_t exec = nullptr;
          FIDES_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
          try {
            for (int k = 0; k < kReps; ++k) {
              ntt_limbs(c, refs.data(), n, inv != 0, s);
              ntt_limbs(c, refs.data(), n, inv == 0, s);
            }
          } catch (...) {
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
          }
          FIDES_CUDA(cudaStreamEndCapture(s, &graph));
          const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
          if (ie != cudaSuccess) {
            cudaGraphDestroy(graph);
            FIDES_CUDA(ie);
          }
          float best = 1e30f;
          cudaError_t err = cudaSuccess;
          for (int rep = 0; rep < 3 && err == cudaSuccess; ++rep) {  // the first replay warms up
            err = cudaEventRecord(e0, s);
            if (err == cudaSuccess) err = cudaGraphLaunch(exec, s);
            if (err == cudaSuccess) err = cudaEventRecord(e1, s);
            if (err == cudaSuccess) err = cudaEventSynchronize(e1);
            float ms = 0;
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
            if (rep && err == cudaSuccess) best = std::min(best, ms);
          }
          cudaGraphExecDestroy(exec);
          cudaGraphDestroy(graph);
          FIDES_CUDA(err);
          return best / (2 * kReps);
        };
        // coordinate descent: the column pass with the row pass at (16, 16), then the row pass
        float best = 0;
        for (int pass = 0; pass < 2; ++pass) {
          int pick = 16, pick_r = 16;
          best = 1e30f;
          for (int r : {16, 8}) {
            if (r == 8 && !r8) continue;
            for (int g : SHAPES) {
              c->ntt_g[inv][pass][cls] = (uint8_t)g;
              c->ntt_r[inv][pass][cls] = (uint8_t)r;
              if (pass == 0) c->ntt_g[inv][1][cls] = 16, c->ntt_r[inv][1][cls] = 16;
              const float t = time_it();
              if (t < best) best = t, pick = g, pick_r = r;
            }
          }
          c->ntt_g[inv][pass][cls] = (uint8_t)pick;
          c->ntt_r[inv][pass][cls] = (uint8_t)pick_r;
        }
        // the other direction of the timing pair uses its current table entries
        if (best_ms) best_ms[inv * 4 + cls] = best;
      }
    // chunk size of long limb lists: a forward + inverse round trip of MAX_NTT_LIMBS limbs
    {
      const int n = max_limbs;
      float best = 1e30f;
      int pick = 0;
      for (int ch : CHUNKS) {
        c->ntt_chunk = ch;
        float t = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {  // the first repetition warms up
          FIDES_CUDA(cudaEventRecord(e0, s));
          ntt_limbs(c, refs.data(), n, false, s);
          ntt_limbs(c, refs.data(), n, true, s);
          FIDES_CUDA(cudaEventRecord(e1, s));
          FIDES_CUDA(cudaEventSynchronize(e1));
          float ms = 0;
          FIDES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if (rep) t = std::min(t, ms);
        }
        if (t < best) best = t, pick = ch;
      }
      c->ntt_chunk = pick;
    }
    FIDES_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    c->profiling = saved_profiling;
    c->ntt_chunk = saved_chunk;
    std::copy(&saved[0][0][0], &saved[0][0][0] + 16, &c->ntt_g[0][0][0]);
    std::copy(&saved_r[0][0][0], &saved_r[0][0][0] + 16, &c->ntt_r[0][0][0]);
    cudaStreamSynchronize(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    throw;
  }
  c->profiling = saved_profiling;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
}

}  // namespace fides
