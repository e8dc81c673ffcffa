// C++ host API of the B200 CKKS evaluation core, over the C ABI (include/fides_b200.h).
//
// Mirrors the reference's CKKS classes for the evaluation path so that code written against
// FIDESlib::CKKS reads the same: Context (src/CKKS/Context.cuh: AddEvalKey, AddRotationKey,
// GetRotationKey), KeySwitchingKey::Initialize(RawKeySwitchKey&) (src/CKKS/KeySwitchingKey.cuh),
// Ciphertext(cc, RawCipherText) with load/store/mult/square/rescale/rotate/rotate_hoisted/
// conjugate/keySwitch (src/CKKS/Ciphertext.cuh:72-650), and the RawCipherText /
// RawKeySwitchKey exchange formats (src/CKKS/openfhe-interface/RawCiphertext.cuh:21-95) minus
// their OpenFHE object handles.  Errors surface as FIDESlib::B200::Error, a
// std::runtime_error, as the reference's engine throws.
//
// Scale bookkeeping follows FIXEDMANUAL: mult multiplies the scales and raises the noise
// degree; rescale divides by the dropped prime and lowers it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fides_b200.h"

namespace FIDESlib {
namespace B200 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != FIDES_OK) throw Error(rc, fides_last_error());
}
inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(FIDES_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// reference RawCipherText (RawCiphertext.cuh:21-37): limbs in EVALUATION format.
struct RawCipherText {
  std::vector<std::vector<uint64_t>> sub_0, sub_1;
  std::vector<uint64_t> moduli;
  int numRes = 0;
  int N = 0;
  double Noise = 1.0;  // scaling factor
  int NoiseLevel = 1;  // noise (scale) degree
  int slots = 0;
};

// reference RawKeySwitchKey (RawCiphertext.cuh:90-95): r_key[a/b][digit][limb][N].
struct RawKeySwitchKey {
  std::vector<std::vector<std::vector<std::vector<uint64_t>>>> r_key;
};

// reference RawPlainText (RawCiphertext.cuh:39-50), without the OpenFHE object: one polynomial
// of numRes limbs in OpenFHE's layout (bit-reversed EVALUATION, or COEFFICIENT).
enum RawFormat { EVALUATION = 0, COEFFICIENT = 1 };
struct RawPlainText {
  std::vector<std::vector<uint64_t>> sub_0;
  std::vector<uint64_t> moduli;
  int numRes = 0;
  int N = 0;
  RawFormat format = EVALUATION;
  double Noise = 1.0;  // scaling factor
  int slots = 0;
  int NoiseLevel = 1;
};

// reference RawParams (RawCiphertext.cuh:52-88): the fields a context is built from (the
// precomputed tables OpenFHE also exports are rebuilt by the library from the primes).
struct RawParams {
  int N = 0, L = 0, K = 0, logN = 0, dnum = 1;
  std::vector<uint64_t> moduli, root_of_unity;                // Q primes and their 2N-th roots
  std::vector<uint64_t> SPECIALmoduli, SPECIALroot_of_unity;  // special primes and roots
  std::vector<double> ScalingFactorReal;                     // per level (FLEXIBLEAUTO chains)
};

struct Parameters {
  int logN = 0;
  int dnum = 1;
  std::vector<uint64_t> primes;   // Q primes
  std::vector<uint64_t> Sprimes;  // special primes
  std::vector<uint64_t> psi;      // optional roots (Q then special); empty = derived
  int device = 0;
  bool reducedNoise = false;  // reduced-noise ModUp / ModDown (src/CKKS/Parameters.cuh:31)

  // reference Parameters::adaptTo(RawParams&) (src/CKKS/Parameters.cu): the chain, the roots and
  // dnum of an OpenFHE context; device and reducedNoise stay as set here
  Parameters adaptTo(const RawParams& raw) const {
    Parameters p = *this;
    p.logN = raw.logN;
    p.dnum = raw.dnum;
    p.primes = raw.moduli;
    p.Sprimes = raw.SPECIALmoduli;
    p.psi = raw.root_of_unity;
    p.psi.insert(p.psi.end(), raw.SPECIALroot_of_unity.begin(), raw.SPECIALroot_of_unity.end());
    if ((int)p.psi.size() != (int)(p.primes.size() + p.Sprimes.size())) p.psi.clear();  // derive them instead
    return p;
  }
};

// Device buffer of limbs (RAII).
class DeviceLimbs {
  uint64_t* p_ = nullptr;
  size_t n_ = 0;

 public:
  DeviceLimbs() = default;
  explicit DeviceLimbs(size_t words) : n_(words) {
    if (words) check_cuda(cudaMalloc(&p_, words * sizeof(uint64_t)), "cudaMalloc");
  }
  ~DeviceLimbs() {
    if (p_) cudaFree(p_);
  }
  DeviceLimbs(DeviceLimbs&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
  DeviceLimbs& operator=(DeviceLimbs&& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  DeviceLimbs(const DeviceLimbs&) = delete;
  DeviceLimbs& operator=(const DeviceLimbs&) = delete;
  uint64_t* get() const { return p_; }
  size_t words() const { return n_; }
};

class Context;
class CryptoContextImpl;

class KeySwitchingKey {
  Context* cc_;
  uint64_t* dev_ = nullptr;

 public:
  explicit KeySwitchingKey(Context& cc) : cc_(&cc) {}
  KeySwitchingKey(KeySwitchingKey&& o) noexcept : cc_(o.cc_), dev_(o.dev_) { o.dev_ = nullptr; }
  KeySwitchingKey& operator=(KeySwitchingKey&& o) noexcept {
    std::swap(cc_, o.cc_);
    std::swap(dev_, o.dev_);
    return *this;
  }
  KeySwitchingKey(const KeySwitchingKey&) = delete;
  ~KeySwitchingKey();
  // reference KeySwitchingKey::Initialize (KeySwitchingKey.cu:19-35)
  void Initialize(const RawKeySwitchKey& rkk);
  // Flat array [2][dnum][n_q + K][N] in host memory or in device memory on the context's GPU
  // (copied either way).
  void InitializeFlat(const uint64_t* host);
  const uint64_t* device() const { return dev_; }
};

class Context {
  fides_ctx* h_ = nullptr;
  cudaStream_t s_ = nullptr;
  std::unique_ptr<KeySwitchingKey> eval_;
  std::map<int, KeySwitchingKey> rot_;

 public:
  int logN, N, L, K, dnum;
  std::vector<uint64_t> primes;  // Q then special

  explicit Context(const Parameters& p)
      : logN(p.logN), N(1 << p.logN), L((int)p.primes.size()), K((int)p.Sprimes.size()), dnum(p.dnum) {
    primes = p.primes;
    primes.insert(primes.end(), p.Sprimes.begin(), p.Sprimes.end());
    fides_params fp{p.logN, L, K, p.dnum, primes.data(), p.psi.empty() ? nullptr : p.psi.data(), p.device};
    check(fides_ctx_create(&fp, &h_));
    if (p.reducedNoise) check(fides_ctx_set_reduced_noise(h_, 1));
    check_cuda(cudaSetDevice(p.device), "cudaSetDevice");
    check_cuda(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "cudaStreamCreate");
  }
  ~Context() {
    rot_.clear();
    eval_.reset();
    if (s_) cudaStreamDestroy(s_);
    if (h_) fides_ctx_destroy(h_);
  }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;

  fides_ctx* handle() const { return h_; }
  cudaStream_t stream() const { return s_; }
  void synchronize() const { check_cuda(cudaStreamSynchronize(s_), "cudaStreamSynchronize"); }

  // reference ContextData::AddEvalKey / AddRotationKey / GetRotationKey (Context.cu:907-944)
  void AddEvalKey(KeySwitchingKey&& k) { eval_ = std::make_unique<KeySwitchingKey>(std::move(k)); }
  KeySwitchingKey& GetEvalKey() {
    if (!eval_) throw Error(FIDES_ERR_KEY, "no relinearization key");
    return *eval_;
  }
  // index 2N - 1 is the conjugation key (automorphism 2N - 1); other indexes are slot rotations
  void AddRotationKey(int index, KeySwitchingKey&& k) {
    if (index != 2 * N - 1) {
      index %= N / 2;
      if (index < 0) index += N / 2;
    }
    rot_.erase(index);
    rot_.emplace(index, std::move(k));
  }
  KeySwitchingKey& GetRotationKey(int index) {
    if (index != 2 * N - 1) {
      index %= N / 2;
      if (index < 0) index += N / 2;
    }
    auto it = rot_.find(index);
    if (it == rot_.end()) throw Error(FIDES_ERR_KEY, "Rotation index " + std::to_string(index) + " not found");
    return it->second;
  }
};

inline KeySwitchingKey::~KeySwitchingKey() {
  if (dev_) fides_key_free(cc_->handle(), dev_);
}

inline void KeySwitchingKey::InitializeFlat(const uint64_t* host) {
  if (dev_) fides_key_free(cc_->handle(), dev_), dev_ = nullptr;
  check(fides_key_upload(cc_->handle(), host, &dev_));
}

inline void KeySwitchingKey::Initialize(const RawKeySwitchKey& rkk) {
  const Context& c = *cc_;
  const size_t limbs = (size_t)c.L + c.K, N = c.N;
  if (rkk.r_key.size() != 2) throw Error(FIDES_ERR_KEY, "RawKeySwitchKey needs a and b");
  std::vector<uint64_t> flat(2 * (size_t)c.dnum * limbs * N, 0);
  for (int ab = 0; ab < 2; ++ab) {
    if ((int)rkk.r_key[ab].size() > c.dnum) throw Error(FIDES_ERR_KEY, "too many key digits");
    for (size_t d = 0; d < rkk.r_key[ab].size(); ++d) {
      if (rkk.r_key[ab][d].size() != limbs) throw Error(FIDES_ERR_KEY, "key digit has the wrong limb count");
      for (size_t i = 0; i < limbs; ++i) {
        const auto& v = rkk.r_key[ab][d][i];
        if (v.size() != N) throw Error(FIDES_ERR_KEY, "key limb has the wrong length");
        std::copy(v.begin(), v.end(), flat.begin() + (((size_t)ab * c.dnum + d) * limbs + i) * N);
      }
    }
  }
  InitializeFlat(flat.data());
}

class Ciphertext {
  friend class CryptoContextImpl;
  Context* cc_;
  DeviceLimbs c0_, c1_;
  DeviceLimbs c2_;  // third component of an unrelinearised product (CryptoContextImpl::EvalMultNoRelin)
  int level_ = 0;

  void alloc(int level) {
    level_ = level;
    c0_ = DeviceLimbs((size_t)level * cc_->N);
    c1_ = DeviceLimbs((size_t)level * cc_->N);
    c2_ = DeviceLimbs();
  }

 public:
  double NoiseFactor = 1.0;
  int NoiseLevel = 1;
  int slots = 0;

  explicit Ciphertext(Context& cc) : cc_(&cc) {}
  Ciphertext(Context& cc, const RawCipherText& raw) : cc_(&cc) { load(raw); }
  Ciphertext(Ciphertext&&) noexcept = default;
  Ciphertext& operator=(Ciphertext&&) noexcept = default;

  int getLevel() const { return level_; }  // active Q limbs
  uint64_t* c0() const { return c0_.get(); }
  uint64_t* c1() const { return c1_.get(); }
  uint64_t* c2() const { return c2_.get(); }
  bool hasC2() const { return c2_.get() != nullptr; }  // three components (not relinearised)
  void need_two() const {
    if (hasC2()) throw Error(FIDES_ERR_STATE, "three-component ciphertext: relinearize first");
  }

  // reference Ciphertext::load / store (Ciphertext.cpp; CudaEngine.cpp:1768-1795, 1156-1227)
  void load(const RawCipherText& raw) {
    const int l = raw.numRes, N = cc_->N;
    if (l < 1 || l > cc_->L || raw.N != N || (int)raw.sub_0.size() != l || (int)raw.sub_1.size() != l)
      throw Error(FIDES_ERR_ARG, "RawCipherText does not match the context");
    alloc(l);
    for (int i = 0; i < l; ++i) {
      if ((int)raw.sub_0[i].size() != N || (int)raw.sub_1[i].size() != N) throw Error(FIDES_ERR_ARG, "bad limb");
      check_cuda(cudaMemcpyAsync(c0() + (size_t)i * N, raw.sub_0[i].data(), N * 8, cudaMemcpyHostToDevice,
                                 cc_->stream()),
                 "H2D");
      check_cuda(cudaMemcpyAsync(c1() + (size_t)i * N, raw.sub_1[i].data(), N * 8, cudaMemcpyHostToDevice,
                                 cc_->stream()),
                 "H2D");
    }
    NoiseFactor = raw.Noise;
    NoiseLevel = raw.NoiseLevel;
    slots = raw.slots;
    cc_->synchronize();
  }

  void store(RawCipherText& raw) const {
    need_two();
    const int N = cc_->N;
    raw.N = N;
    raw.numRes = level_;
    raw.moduli.assign(cc_->primes.begin(), cc_->primes.begin() + level_);
    raw.sub_0.assign(level_, std::vector<uint64_t>(N));
    raw.sub_1.assign(level_, std::vector<uint64_t>(N));
    for (int i = 0; i < level_; ++i) {
      check_cuda(cudaMemcpyAsync(raw.sub_0[i].data(), c0() + (size_t)i * N, N * 8, cudaMemcpyDeviceToHost,
                                 cc_->stream()),
                 "D2H");
      check_cuda(cudaMemcpyAsync(raw.sub_1[i].data(), c1() + (size_t)i * N, N * 8, cudaMemcpyDeviceToHost,
                                 cc_->stream()),
                 "D2H");
    }
    raw.Noise = NoiseFactor;
    raw.NoiseLevel = NoiseLevel;
    raw.slots = slots;
    cc_->synchronize();
  }

  // reference Ciphertext::mult(b, rescale) (Ciphertext.cpp:660-869): tensor + relinearize
  void mult(const Ciphertext& b, bool rescale = false) {
    need_two();
    if (b.level_ != level_) throw Error(FIDES_ERR_LEVEL, "operands at different levels");
    const int lo = rescale ? level_ - 1 : level_;
    Ciphertext out(*cc_);
    out.alloc(lo);
    check(fides_hmult(cc_->handle(), c0(), c1(), b.c0(), b.c1(), level_, cc_->GetEvalKey().device(), rescale ? 1 : 0,
                      out.c0(), out.c1(), cc_->stream()));
    double f = NoiseFactor * b.NoiseFactor;
    int nl = NoiseLevel + b.NoiseLevel;
    if (rescale) {
      f /= (double)cc_->primes[level_ - 1];
      nl -= 1;
    }
    const int sl = slots;
    *this = std::move(out);
    NoiseFactor = f;
    NoiseLevel = nl;
    slots = sl;
  }
  void square(bool rescale = false) { mult(*this, rescale); }

  // reference Ciphertext::rescale (Ciphertext.cpp:569-607), FIXEDMANUAL
  void rescale() {
    if (level_ < 2) throw Error(FIDES_ERR_LEVEL, "cannot rescale the last limb");
    Ciphertext out(*cc_);
    out.alloc(level_ - 1);
    check(fides_rescale(cc_->handle(), c0(), level_, out.c0(), cc_->stream()));
    check(fides_rescale(cc_->handle(), c1(), level_, out.c1(), cc_->stream()));
    if (hasC2()) {  // every component is divided by the same prime
      out.c2_ = DeviceLimbs((size_t)(level_ - 1) * cc_->N);
      check(fides_rescale(cc_->handle(), c2(), level_, out.c2(), cc_->stream()));
    }
    const double f = NoiseFactor / (double)cc_->primes[level_ - 1];
    const int nl = NoiseLevel - 1, sl = slots;
    cc_->synchronize();  // the old buffers are released below
    *this = std::move(out);
    NoiseFactor = f;
    NoiseLevel = nl;
    slots = sl;
  }

  // reference Ciphertext::rotate(index) (Ciphertext.cpp:1102-1168)
  void rotate(int index) {
    need_two();
    check(fides_rotate(cc_->handle(), c0(), c1(), level_, cc_->GetRotationKey(index).device(), index, c0(), c1(),
                       cc_->stream()));
  }
  // reference Ciphertext::conjugate (Ciphertext.cpp:1175-1219)
  void conjugate() {
    need_two();
    const uint32_t k = 2u * cc_->N - 1;
    check(fides_rotate_auto(cc_->handle(), c0(), c1(), level_, cc_->GetRotationKey(2 * cc_->N - 1).device(), k,
                            c0(), c1(), cc_->stream()));
  }
  // reference Ciphertext::add / sub (Ciphertext.cpp:244-330)
  void add(const Ciphertext& b) {
    need_two();
    if (b.level_ != level_) throw Error(FIDES_ERR_LEVEL, "operands at different levels");
    check(fides_add(cc_->handle(), c0(), b.c0(), level_, c0(), cc_->stream()));
    check(fides_add(cc_->handle(), c1(), b.c1(), level_, c1(), cc_->stream()));
  }
  void sub(const Ciphertext& b) {
    if (b.level_ != level_) throw Error(FIDES_ERR_LEVEL, "operands at different levels");
    check(fides_sub(cc_->handle(), c0(), b.c0(), level_, c0(), cc_->stream()));
    check(fides_sub(cc_->handle(), c1(), b.c1(), level_, c1(), cc_->stream()));
  }

  // reference Ciphertext::keySwitch (Ciphertext.cpp:1893-1907): (c0 + f0, f1)
  void keySwitch(const KeySwitchingKey& ksk) {
    need_two();
    DeviceLimbs f0((size_t)level_ * cc_->N), f1((size_t)level_ * cc_->N);
    check(fides_keyswitch(cc_->handle(), c1(), level_, ksk.device(), f0.get(), f1.get(), cc_->stream()));
    check(fides_add(cc_->handle(), c0(), f0.get(), level_, c0(), cc_->stream()));
    cc_->synchronize();  // f0 is released at scope exit
    c1_ = std::move(f1);
  }

  // reference Ciphertext::rotate_hoisted (Ciphertext.cpp:1221-1394)
  void rotate_hoisted(const std::vector<int>& indexes, std::vector<Ciphertext*> results) const {
    need_two();
    if (results.size() != indexes.size()) throw Error(FIDES_ERR_ARG, "one result per index");
    std::vector<const uint64_t*> keys;
    std::vector<uint64_t*> o0, o1;
    for (size_t j = 0; j < indexes.size(); ++j) {
      keys.push_back(cc_->GetRotationKey(indexes[j]).device());
      results[j]->alloc(level_);
      results[j]->NoiseFactor = NoiseFactor;
      results[j]->NoiseLevel = NoiseLevel;
      results[j]->slots = slots;
      o0.push_back(results[j]->c0());
      o1.push_back(results[j]->c1());
    }
    check(fides_rotate_hoisted(cc_->handle(), c0(), c1(), level_, keys.data(), indexes.data(), (int)indexes.size(),
                               o0.data(), o1.data(), cc_->stream()));
  }
};

}  // namespace B200
}  // namespace FIDESlib
