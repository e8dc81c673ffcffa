// Interop with the reference's raw host formats (src/CKKS/openfhe-interface/RawCiphertext.cuh:
// RawCipherText :20-37, RawKeySwitchKey :90-95): limbs arrive as one host array per limb
// (sub_0[i].data(), r_key[a][d][i].data()), in EVALUATION or COEFFICIENT format, and the
// evaluation vectors in OpenFHE's bit-reversed order (the reference's REV = 1) or in natural
// order (REV = 0).  Import gathers them into this library's limb-major device layout and
// brings them to bit-reversed EVALUATION form; export is the way back (Ciphertext::load / store,
// src/CKKS/Ciphertext.cpp:415-464, and KeySwitchingKey::Initialize, KeySwitchingKey.cu:19-35).
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "context.hpp"
#include "interop.hpp"
#include "ntt.cuh"

namespace fides {
namespace {

constexpr int BR_THREADS = 256;

// out[l][j] = in[l][brev_logN(j)] for n limbs (a permutation of each limb; in != out).
__global__ void __launch_bounds__(BR_THREADS) brev_limbs_kernel(const uint64_t* __restrict__ in,
                                                                uint64_t* __restrict__ out, int logN) {
  const size_t base = (size_t)blockIdx.y << logN;
  const uint32_t j = blockIdx.x * BR_THREADS + threadIdx.x;
  out[base + j] = in[base + (__brev(j) >> (32 - logN))];
}

void brev_limbs(Context* c, const uint64_t* in, uint64_t* out, int n_limbs, cudaStream_t s) {
  if (n_limbs <= 0) return;
  dim3 grid(c->N / BR_THREADS, n_limbs);
  LaunchScope ls(c, s, KK_ELEM, 16.0 * c->N * n_limbs);
  brev_limbs_kernel<<<grid, BR_THREADS, 0, s>>>(in, out, c->logN);
  FIDES_CUDA(cudaGetLastError());
}

void check_args(Context* c, int n_polys, int level) {
  if (n_polys < 1) throw Error(-1, "n_polys < 1");
  if (level < 1 || level > c->n_q + c->K) throw Error(-4, "level out of range");
  if (c->N < BR_THREADS) throw Error(-1, "ring too small for the interop kernels");
}

// prime id of limb i: the Q primes come first, then (for level > n_q) the special primes, which
// is the context's own prime order
int limb_prime(Context*, int, int i) { return i; }

}  // namespace

void op_ct_import(Context* c, int n_polys, const uint64_t* const* limbs, const uint64_t* moduli, int level,
                  int format, int natural, uint64_t* out, cudaStream_t s) {
  check_args(c, n_polys, level);
  if (moduli)
    for (int i = 0; i < level; ++i)
      if (moduli[i] != c->primes[limb_prime(c, level, i)]) throw Error(-1, "moduli differ from the context's primes");
  const size_t N = c->N, limb = N * sizeof(uint64_t), total = (size_t)n_polys * level;
  for (size_t k = 0; k < total; ++k)
    if (!limbs[k]) throw Error(-1, "null limb pointer");
  Scratch sc(c, natural ? total * limb : 0, s);
  uint64_t* dst = natural ? sc.u64() : out;
  for (size_t k = 0; k < total; ++k)
    FIDES_CUDA(cudaMemcpyAsync(dst + k * N, limbs[k], limb, cudaMemcpyHostToDevice, s));
  if (natural) brev_limbs(c, dst, out, (int)total, s);
  if (format == 1) {  // COEFFICIENT -> EVALUATION
    std::vector<LimbRef> refs;
    for (int p = 0; p < n_polys; ++p)
      for (int i = 0; i < level; ++i) refs.push_back(lref(out + ((size_t)p * level + i) * N, limb_prime(c, level, i)));
    ntt_limbs(c, refs.data(), (int)refs.size(), false, s);
  }
}

void op_ct_export(Context* c, int n_polys, const uint64_t* in, int level, int format, int natural,
                  uint64_t* const* limbs, cudaStream_t s) {
  check_args(c, n_polys, level);
  const size_t N = c->N, limb = N * sizeof(uint64_t), total = (size_t)n_polys * level;
  for (size_t k = 0; k < total; ++k)
    if (!limbs[k]) throw Error(-1, "null limb pointer");
  Scratch sc(c, (format == 1 || natural) ? (natural && format == 1 ? 2 : 1) * total * limb : 0, s);
  const uint64_t* src = in;
  uint64_t* buf = sc.u64();
  if (format == 1) {  // EVALUATION -> COEFFICIENT into scratch
    std::vector<LimbRef> refs;
    for (int p = 0; p < n_polys; ++p)
      for (int i = 0; i < level; ++i) {
        const size_t k = (size_t)p * level + i;
        LimbRef r = lref(buf + k * N, limb_prime(c, level, i));
        r.src = in + k * N;
        refs.push_back(r);
      }
    ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
    src = buf;
    buf += total * N;
  }
  if (natural) {
    brev_limbs(c, src, buf, (int)total, s);
    src = buf;
  }
  for (size_t k = 0; k < total; ++k)
    FIDES_CUDA(cudaMemcpyAsync(limbs[k], src + k * N, limb, cudaMemcpyDeviceToHost, s));
  FIDES_CUDA(cudaStreamSynchronize(s));
}

uint64_t* op_key_import(Context* c, const uint64_t* const* limbs, int natural, cudaStream_t s) {
  const size_t N = c->N, limb = N * sizeof(uint64_t), ext = (size_t)c->n_q + c->K;
  const size_t total = 2 * (size_t)c->dnum * ext;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, total * limb);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(-3, std::string("key allocation failed: ") + cudaGetErrorString(e));
  }
  uint64_t* key = static_cast<uint64_t*>(p);
  try {
    Scratch sc(c, natural ? total * limb : 0, s);
    uint64_t* dst = natural ? sc.u64() : key;
    for (size_t k = 0; k < total; ++k) {
      if (limbs[k])
        FIDES_CUDA(cudaMemcpyAsync(dst + k * N, limbs[k], limb, cudaMemcpyHostToDevice, s));
      else
        FIDES_CUDA(cudaMemsetAsync(dst + k * N, 0, limb, s));
    }
    if (natural) brev_limbs(c, dst, key, (int)total, s);
    FIDES_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaFree(key);
    throw;
  }
  return key;
}

}  // namespace fides
