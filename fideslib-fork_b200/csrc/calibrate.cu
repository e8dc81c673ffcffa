// Butterfly-rate calibration: the rate at which one B200 runs the NTT's butterflies with no
// memory traffic at all (the 64-bit integer form, and the FP64 form used for primes below
// 2^50).  The forward butterfly (ct_bf_small: one 64-bit Shoup product and
// two 64-bit additions) is bound by the FMA-heavy pipe, where the IMAD family executes,
// so this rate -- not HBM bandwidth -- is the compute roofline of the NTT passes.
#include "ntt_impl.cuh"

namespace fides {
namespace {

constexpr int CAL_THREADS = 256;
constexpr int CAL_E = 16;  // values per thread, as in the NTT passes

// Every thread runs `rounds` x 4 stages x 8 butterflies on 16 register values, each
// stage with its own twiddle (held in registers), and writes one checksum word so the
// work cannot be elided.  Values wrap modulo 2^64: only the instruction stream matters.
__global__ void __launch_bounds__(CAL_THREADS) bf_peak_kernel(uint64_t* out, uint64_t q, ShoupConst w0,
                                                             ShoupConst w1, ShoupConst w2, ShoupConst w3,
                                                             int rounds) {
  uint64_t x[CAL_E];
  const uint64_t seed = (uint64_t)(blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B97F4A7C15ull;
#pragma unroll
  for (int r = 0; r < CAL_E; ++r) x[r] = (seed + (uint64_t)r * 0x2545F4914F6CDD1Dull) % q;
  const uint64_t q2 = 2 * q;
  for (int it = 0; it < rounds; ++it) {
#pragma unroll
    for (int b = 3; b >= 0; --b) {
      const ShoupConst w = b == 3 ? w0 : b == 2 ? w1 : b == 1 ? w2 : w3;
#pragma unroll
      for (int r = 0; r < CAL_E; ++r)
        if (!(r & (1 << b))) nttk::ct_bf_small(x[r], x[r | (1 << b)], w, q, q2);
    }
  }
  uint64_t s = 0;
#pragma unroll
  for (int r = 0; r < CAL_E; ++r) s ^= x[r];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// The FP64 forward butterfly of the NTT passes for primes below 2^50 (reduce x, FP64
// modular product of y, x +- r), on register-resident doubles.
__global__ void __launch_bounds__(CAL_THREADS) bf_peak_f64_kernel(uint64_t* out, double q, double qinv, double2 w0,
                                                                 double2 w1, double2 w2, double2 w3, int rounds) {
  double x[CAL_E];
  const uint64_t seed = (uint64_t)(blockIdx.x * blockDim.x + threadIdx.x) * 0x9E3779B97F4A7C15ull;
#pragma unroll
  for (int r = 0; r < CAL_E; ++r) x[r] = (double)((seed + (uint64_t)r * 0x2545F4914F6CDD1Dull) % (uint64_t)q);
  for (int it = 0; it < rounds; ++it) {
#pragma unroll
    for (int b = 3; b >= 0; --b) {
      const double2 w = b == 3 ? w0 : b == 2 ? w1 : b == 1 ? w2 : w3;
#pragma unroll
      for (int r = 0; r < CAL_E; ++r)
        if (!(r & (1 << b))) {
          const int s = r | (1 << b);
          const double a = nttk::f_reduce(x[r], q, qinv);
          const double t = nttk::f_mulmod(x[s], w.x, w.y, q);
          x[r] = __dadd_rn(a, t);
          x[s] = __dsub_rn(a, t);
        }
    }
  }
  uint64_t s = 0;
#pragma unroll
  for (int r = 0; r < CAL_E; ++r) s ^= (uint64_t)__double_as_longlong(x[r]);
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

double measure_bf_peak_f64(int device) {
  FIDES_CUDA(cudaSetDevice(device));
  int sms = 0;
  FIDES_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8;
  const uint64_t q = (1ull << 50) - (1ull << 17) + 1;  // any odd modulus below 2^50
  const double qd = (double)q;
  auto tw = [&](uint64_t w) { return make_double2((double)(w % q), (double)(w % q) / qd); };
  uint64_t* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FIDES_CUDA(cudaMalloc(&out, sizeof(uint64_t) * blocks * CAL_THREADS));
  FIDES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  FIDES_CUDA(cudaEventCreate(&e0));
  FIDES_CUDA(cudaEventCreate(&e1));
  const int rounds = 4096;
  float ms = 0;
  for (int rep = 0; rep < 3; ++rep) {  // the first launch warms up; the last is kept
    FIDES_CUDA(cudaEventRecord(e0, st));
    bf_peak_f64_kernel<<<blocks, CAL_THREADS, 0, st>>>(out, qd, 1.0 / qd, tw(0x1234567890ull), tw(0x0fedcba987ull),
                                                     tw(0x13579bdf02ull), tw(0x2468ace013ull), rounds);
    FIDES_CUDA(cudaGetLastError());
    FIDES_CUDA(cudaEventRecord(e1, st));
    FIDES_CUDA(cudaEventSynchronize(e1));
    FIDES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  const double bf = (double)blocks * CAL_THREADS * rounds * 4 * (CAL_E / 2);
  return bf / (ms * 1e-3);
}

double measure_bf_peak(int device) {
  FIDES_CUDA(cudaSetDevice(device));
  int sms = 0;
  FIDES_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8;
  const uint64_t q = (1ull << 50) - (1ull << 17) + 1;  // any odd modulus below 2^58
  auto sc = [&](uint64_t w) { return h_shoup(w % q, q); };
  uint64_t* out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  FIDES_CUDA(cudaMalloc(&out, sizeof(uint64_t) * blocks * CAL_THREADS));
  FIDES_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  FIDES_CUDA(cudaEventCreate(&e0));
  FIDES_CUDA(cudaEventCreate(&e1));
  const int rounds = 4096;
  float ms = 0;
  for (int rep = 0; rep < 3; ++rep) {  // the first launch warms up; the last is kept
    FIDES_CUDA(cudaEventRecord(e0, st));
    bf_peak_kernel<<<blocks, CAL_THREADS, 0, st>>>(out, q, sc(0x1234567890ull), sc(0x0fedcba987ull),
                                                 sc(0x13579bdf02ull), sc(0x2468ace013ull), rounds);
    FIDES_CUDA(cudaGetLastError());
    FIDES_CUDA(cudaEventRecord(e1, st));
    FIDES_CUDA(cudaEventSynchronize(e1));
    FIDES_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  const double bf = (double)blocks * CAL_THREADS * rounds * 4 * (CAL_E / 2);
  return bf / (ms * 1e-3);
}

}  // namespace fides
