// The evaluation facade of the B200 CKKS core, shaped like the reference's
// fideslib::CryptoContextImpl<DCRTPoly> (api/CryptoContext.hpp:306-458, bodies in
// api/CryptoContext.cpp:1120-1299 over CudaEngine, api/engine/cuda/CudaEngine.cpp:429-1150):
// MakeCKKSPackedPlaintext (encoded on the device), EvalAdd / EvalSub (ciphertexts, plaintexts and
// real constants), EvalMult (ciphertexts, plaintexts, real constants) / EvalSquare,
// EvalMultNoRelin + Relinearize, EvalNegate, EvalAddMany, EvalRotateMany, EvalChebyshevSeries,
// MultByMonomial, AccumulateSum, LinearTransform(InPlace / Many), Rescale,
// EvalRotate, EvalFastRotationPrecompute + EvalFastRotation, EvalBootstrapSetup +
// EvalBootstrap, with the reference's level and scale management:
//   * FIXEDMANUAL: EvalMult leaves a degree-2 result at the operands' level (scale product);
//     Rescale divides by the top prime and drops it; operands of an addition or a product are
//     brought to the lower level by dropping limbs (Ciphertext::adjustBeforeMult,
//     src/CKKS/Ciphertext.cpp:643-657);
//   * FLEXIBLEAUTO: every level l has the canonical scale S_l of OpenFHE's FLEXIBLE chain,
//     S_(l-1) = S_l^2 / q_(l-1) from the top scale, and operands are adjusted to a common level
//     at its canonical scale before they meet (adjustScaleAndLevel, Ciphertext.cpp:1917-2068:
//     a constant multiple that re-targets the scale, then a rescale).  EvalMult returns the
//     product already rescaled (degree 1, level l - 1, scale S_(l-1)): the library fuses the
//     rescale into the key switch's ModDown, so the product is never held at degree 2; OpenFHE
//     holds it at degree 2 and rescales before the next product, which gives the same value one
//     call later.  Rescale is therefore a copy under FLEXIBLEAUTO, as OpenFHE's is a no-op in its
//     automatic modes.
// OpenFHE types stay out of this header: keys and ciphertexts arrive as the raw formats of
// FIDESlibB200.hpp (RawKeySwitchKey / RawCipherText) or as device arrays, and key generation and
// encryption remain with the caller (OpenFHE in the reference's setting).
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <memory>
#include <vector>

#include "FIDESlibB200.hpp"

namespace FIDESlib {
namespace B200 {

enum ScalingTechnique { FIXEDMANUAL = 0, FLEXIBLEAUTO = 1 };

// An encoded CKKS plaintext (the reference's Plaintext from MakeCKKSPackedPlaintext,
// api/Plaintext.hpp, CKKSPackedEncoding): `level` limbs in EVALUATION form on the device, at
// scale `scale`, holding `slots` slots.
struct Plaintext {
  DeviceLimbs limbs;  // [level][N], or [level + K][N] when ext
  int level = 0;
  double scale = 0;
  int slots = 0;
  // encoded over Q.P as well (MakeCKKSPackedPlaintextExtended): the K special limbs follow the
  // level Q limbs, which are those of the plain encoding
  bool ext = false;
  const uint64_t* data() const { return limbs.get(); }
};

// The ModUp of a ciphertext's c1, kept for any number of EvalFastRotation calls (the
// reference's EvalFastRotationPrecompute result).
struct FastRotationPrecompute {
  DeviceLimbs digits;  // [beta][level + K][N]
  int level = 0;
};

class CryptoContextImpl {
  Context* cc_;
  ScalingTechnique tech_;
  std::vector<double> S_;  // canonical scale of each level (FLEXIBLEAUTO)
  fides_boot* boot_ = nullptr;
  fides_boot_params boot_params_{};
  std::map<int, fides_boot*> short_boot_;  // EvalBootstrapToLevel: bootstrappers on shorter chains
  double boot_msg_scale_ = 0;
  bool boot_double_hoist_ = true;
  std::unique_ptr<KeySwitchingKey> to_sparse_, to_dense_;

  int N() const { return cc_->N; }
  uint64_t q(int i) const { return cc_->primes[i]; }

  static double round_even(double v) { return std::nearbyint(v); }
  // w mod q_i for an integer held exactly in a double (any magnitude)
  uint64_t residue(double w, int i) const {
    const uint64_t qi = q(i);
    const bool neg = w < 0;
    const double a = std::fabs(w);
    uint64_t r;
    if (a < 9223372036854775808.0) {
      r = (uint64_t)a % qi;
    } else {
      int e = 0;
      const double fr = std::frexp(a, &e);
      const uint64_t m = (uint64_t)std::ldexp(fr, 53);
      unsigned __int128 p = 1, b = 2 % qi;
      for (uint64_t k = (uint64_t)(e - 53); k; k >>= 1, b = b * b % qi)
        if (k & 1) p = p * b % qi;
      r = (uint64_t)((unsigned __int128)(m % qi) * p % qi);
    }
    return neg && r ? qi - r : r;
  }
  std::vector<uint64_t> residues(double w, int level) const {
    std::vector<uint64_t> v(level);
    for (int i = 0; i < level; ++i) v[i] = residue(w, i);
    return v;
  }

  Ciphertext fresh(int level, double scale, int degree, int slots) const {
    Ciphertext c(*cc_);
    c.alloc(level);
    c.NoiseFactor = scale;
    c.NoiseLevel = degree;
    c.slots = slots;
    return c;
  }
  static bool same_scale(double a, double b) { return std::abs(a / b - 1) < 1e-12; }

  // a * k (an integer constant) on its first `level` limbs, then rescaled: level - 1 limbs at
  // scale new_scale
  Ciphertext mul_int_rescale(const Ciphertext& a, int level, double k, double new_scale) const {
    const auto s = residues(k, level);
    Ciphertext t = fresh(level, 0, 1, a.slots);
    check(fides_mul_scalar(cc_->handle(), a.c0(), level, s.data(), t.c0(), cc_->stream()));
    check(fides_mul_scalar(cc_->handle(), a.c1(), level, s.data(), t.c1(), cc_->stream()));
    Ciphertext o = fresh(level - 1, new_scale, 1, a.slots);
    check(fides_rescale(cc_->handle(), t.c0(), level, o.c0(), cc_->stream()));
    check(fides_rescale(cc_->handle(), t.c1(), level, o.c1(), cc_->stream()));
    if (a.hasC2()) {  // a third component is scaled the same way
      DeviceLimbs t2((size_t)N() * level);
      o.c2_ = DeviceLimbs((size_t)N() * (level - 1));
      check(fides_mul_scalar(cc_->handle(), a.c2(), level, s.data(), t2.get(), cc_->stream()));
      check(fides_rescale(cc_->handle(), t2.get(), level, o.c2(), cc_->stream()));
      cc_->synchronize();
    }
    cc_->synchronize();  // t is released at scope exit
    return o;
  }

  Ciphertext add_sub_pt(const Ciphertext& a, const Plaintext& p, bool sub) const {
    const int l = std::min(a.getLevel(), p.level);
    Ciphertext A = tech_ == FLEXIBLEAUTO ? AdjustToLevel(a, l) : copy_of(a, l);
    if (!same_scale(A.NoiseFactor, p.scale))
      throw Error(FIDES_ERR_ARG, "the plaintext's scale differs from the ciphertext's");
    Ciphertext o = copy_of(A, l);  // c1 (and c2) as they are
    check((sub ? fides_sub : fides_add)(cc_->handle(), A.c0(), p.data(), l, o.c0(), cc_->stream()));
    cc_->synchronize();  // A is released at scope exit
    return o;
  }

  Ciphertext copy_of(const Ciphertext& a, int level) const {
    Ciphertext o = fresh(level, a.NoiseFactor, a.NoiseLevel, a.slots);
    const size_t bytes = sizeof(uint64_t) * (size_t)N() * level;
    check_cuda(cudaMemcpyAsync(o.c0(), a.c0(), bytes, cudaMemcpyDeviceToDevice, cc_->stream()), "D2D");
    check_cuda(cudaMemcpyAsync(o.c1(), a.c1(), bytes, cudaMemcpyDeviceToDevice, cc_->stream()), "D2D");
    if (a.hasC2()) {
      o.c2_ = DeviceLimbs((size_t)N() * level);
      check_cuda(cudaMemcpyAsync(o.c2(), a.c2(), bytes, cudaMemcpyDeviceToDevice, cc_->stream()), "D2D");
    }
    return o;
  }

 public:
  // top_scale: the scale of the top level (FLEXIBLEAUTO's S_(L+1); under FIXEDMANUAL only the
  // default scale of EvalBootstrap's inputs).
  CryptoContextImpl(Context& cc, ScalingTechnique tech, double top_scale) : cc_(&cc), tech_(tech) {
    const int L = cc.L;
    S_.assign(L + 1, 0.0);
    S_[L] = top_scale;
    for (int l = L; l > 1; --l) S_[l - 1] = S_[l] * S_[l] / (double)cc.primes[l - 1];
  }
  ~CryptoContextImpl() {
    drop_short_boots();
    if (boot_) fides_boot_destroy(boot_);
  }
  CryptoContextImpl(const CryptoContextImpl&) = delete;
  CryptoContextImpl& operator=(const CryptoContextImpl&) = delete;

  ScalingTechnique GetScalingTechnique() const { return tech_; }
  // the canonical scale of `level` limbs (OpenFHE's GetScalingFactorReal)
  double GetScalingFactorReal(int level) const { return S_.at(level); }

  // A ciphertext at `level` limbs with the canonical scale of that level (FLEXIBLEAUTO), or the
  // same value on fewer limbs (FIXEDMANUAL, scale unchanged).
  Ciphertext AdjustToLevel(const Ciphertext& a, int level) const {
    if (level < 1 || level > a.getLevel()) throw Error(FIDES_ERR_LEVEL, "cannot raise a ciphertext's level");
    if (tech_ == FIXEDMANUAL) return copy_of(a, level);  // limbs dropped, scale and degree unchanged
    if (a.NoiseLevel == 2) {
      // an unrescaled product (EvalMultNoRelin / Relinearize): kept as it is at its own level,
      // otherwise rescaled first, as OpenFHE does before the next operation
      if (level == a.getLevel()) return copy_of(a, level);
      return AdjustToLevel(Rescale(a), level);
    }
    if (a.NoiseLevel != 1) throw Error(FIDES_ERR_STATE, "adjust a degree-2 ciphertext after Rescale");
    if (a.getLevel() == level && same_scale(a.NoiseFactor, S_[level])) return copy_of(a, level);
    if (a.getLevel() == level)
      throw Error(FIDES_ERR_LEVEL, "scale differs from the level's canonical scale and no level is left to adjust it");
    const double k = round_even(S_[level] * (double)q(level) / a.NoiseFactor);
    return mul_int_rescale(a, level + 1, k, S_[level]);
  }

  // ---- plaintexts (CryptoContextImpl::MakeCKKSPackedPlaintext, api/CryptoContext.hpp; encoded
  // on the device by fides_encode, the reference's DeviceEncodeBatch.cu path)
  // `z` is padded with zeros to a power of two of slots (at most N/2); level 0 = the top level,
  // scale 0 = that level's canonical scale (OpenFHE's default for the level).
  Plaintext MakeCKKSPackedPlaintext(const std::vector<std::complex<double>>& z, int level = 0,
                                    double scale = 0) const {
    return encode_packed(z, level, scale, false);
  }
  // MakeCKKSPackedPlaintextExtended (api/CryptoContext.hpp:171): the same integer polynomial
  // over Q.P (fides_encode_ext), for the diagonals of a LinearTransform that keeps its baby
  // steps and giant-step sums in the extended basis.
  Plaintext MakeCKKSPackedPlaintextExtended(const std::vector<std::complex<double>>& z, int level = 0,
                                            double scale = 0) const {
    return encode_packed(z, level, scale, true);
  }
  Plaintext MakeCKKSPackedPlaintextExtended(const std::vector<double>& x, int level = 0, double scale = 0) const {
    return encode_packed(std::vector<std::complex<double>>(x.begin(), x.end()), level, scale, true);
  }
  Plaintext encode_packed(const std::vector<std::complex<double>>& z, int level, double scale, bool ext) const {
    const int L = (int)S_.size() - 1;
    if (level == 0) level = L;
    if (level < 1 || level > L) throw Error(FIDES_ERR_LEVEL, "plaintext level out of range");
    if (z.empty() || (int)z.size() > N() / 2) throw Error(FIDES_ERR_ARG, "1..N/2 slots");
    int n = 1;
    while (n < (int)z.size()) n <<= 1;
    std::vector<double> host(2 * (size_t)n, 0.0);
    for (size_t i = 0; i < z.size(); ++i) host[2 * i] = z[i].real(), host[2 * i + 1] = z[i].imag();
    DeviceLimbs dev(2 * (size_t)n);  // n complex slots as doubles
    check_cuda(cudaMemcpyAsync(dev.get(), host.data(), sizeof(double) * host.size(), cudaMemcpyHostToDevice,
                               cc_->stream()),
               "H2D");
    Plaintext p;
    p.level = level;
    p.scale = scale > 0 ? scale : S_[level];
    p.slots = n;
    p.ext = ext;
    p.limbs = DeviceLimbs((size_t)N() * (level + (ext ? cc_->K : 0)));
    check((ext ? fides_encode_ext : fides_encode)(cc_->handle(), reinterpret_cast<const double*>(dev.get()), n, 1,
                                                  p.scale, level, p.limbs.get(), cc_->stream()));
    cc_->synchronize();  // the slot buffer is released at scope exit
    return p;
  }
  Plaintext MakeCKKSPackedPlaintext(const std::vector<double>& x, int level = 0, double scale = 0) const {
    return MakeCKKSPackedPlaintext(std::vector<std::complex<double>>(x.begin(), x.end()), level, scale);
  }
  // A plaintext from / to the reference's raw exchange format (GetRawPlainText /
  // GetOpenFHEPlaintext, RawCiphertext.cuh:106-109): the limbs converted by fides_ct_import /
  // fides_ct_export (COEFFICIENT limbs transformed on the device; OpenFHE's bit-reversed
  // EVALUATION order unless natural_order).
  Plaintext LoadPlaintext(const RawPlainText& raw, bool natural_order = false) const {
    if (raw.numRes < 1 || raw.numRes > (int)S_.size() - 1 || raw.N != N() || (int)raw.sub_0.size() != raw.numRes)
      throw Error(FIDES_ERR_ARG, "RawPlainText does not match the context");
    std::vector<const uint64_t*> limbs;
    for (const auto& v : raw.sub_0) {
      if ((int)v.size() != N()) throw Error(FIDES_ERR_ARG, "bad plaintext limb");
      limbs.push_back(v.data());
    }
    Plaintext p;
    p.level = raw.numRes;
    p.scale = raw.Noise;
    p.slots = raw.slots;
    p.limbs = DeviceLimbs((size_t)N() * raw.numRes);
    check(fides_ct_import(cc_->handle(), 1, limbs.data(), raw.moduli.empty() ? nullptr : raw.moduli.data(),
                          raw.numRes, raw.format == COEFFICIENT ? 1 : 0, natural_order ? 1 : 0, p.limbs.get(),
                          cc_->stream()));
    cc_->synchronize();
    return p;
  }
  void StorePlaintext(const Plaintext& p, RawPlainText& raw, RawFormat format = EVALUATION,
                      bool natural_order = false) const {
    raw.N = N();
    raw.numRes = p.level;
    raw.moduli.assign(cc_->primes.begin(), cc_->primes.begin() + p.level);
    raw.format = format;
    raw.Noise = p.scale;
    raw.slots = p.slots;
    raw.NoiseLevel = 1;
    raw.sub_0.assign(p.level, std::vector<uint64_t>(N()));
    std::vector<uint64_t*> limbs;
    for (auto& v : raw.sub_0) limbs.push_back(v.data());
    check(fides_ct_export(cc_->handle(), 1, p.data(), p.level, format == COEFFICIENT ? 1 : 0, natural_order ? 1 : 0,
                          limbs.data(), cc_->stream()));
  }

  // ---- additive operations (CryptoContextImpl::EvalAdd / EvalSub)
  Ciphertext EvalAdd(const Ciphertext& a, const Ciphertext& b) const { return add_sub(a, b, false); }
  Ciphertext EvalSub(const Ciphertext& a, const Ciphertext& b) const { return add_sub(a, b, true); }
  Ciphertext EvalAdd(const Ciphertext& a, double c) const { return add_const(a, c); }
  Ciphertext EvalSub(const Ciphertext& a, double c) const { return add_const(a, -c); }
  // with a plaintext (Ciphertext::addPt / subPt): the plaintext's scale must equal the
  // ciphertext's (FIXEDMANUAL) or the common level's canonical scale (FLEXIBLEAUTO, where the
  // ciphertext is first brought to the lower of the two levels)
  Ciphertext EvalAdd(const Ciphertext& a, const Plaintext& p) const { return add_sub_pt(a, p, false); }
  Ciphertext EvalSub(const Ciphertext& a, const Plaintext& p) const { return add_sub_pt(a, p, true); }
  // EvalChebyshevSeries (CryptoContextImpl::EvalChebyshevSeries): OpenFHE's convention
  // c_0 / 2 + sum_(k >= 1) c_k T_k on [lo, hi], evaluated on the device (fides_eval_chebyshev)
  // with the relinearisation key; the result sits at its level's canonical scale S_l,
  // ceil(log2 d) + 1 levels below the input for degree d (one more for [lo, hi] != [-1, 1]).
  Ciphertext EvalChebyshevSeries(const Ciphertext& a, const std::vector<double>& coeffs, double lo, double hi) const {
    a.need_two();
    if (a.NoiseLevel == 2) return EvalChebyshevSeries(Rescale(a), coeffs, lo, hi);
    int lvl = 0;
    double sc = 0;
    Ciphertext o = fresh(a.getLevel(), 0, 1, a.slots);
    check(fides_eval_chebyshev(cc_->handle(), cc_->GetEvalKey().device(), S_.back(), a.c0(), a.c1(), a.getLevel(),
                               a.NoiseFactor, coeffs.data(), (int)coeffs.size(), lo, hi, o.c0(), o.c1(), &lvl, &sc,
                               cc_->stream()));
    cc_->synchronize();
    o.level_ = lvl;  // the first lvl limbs of the buffers
    o.NoiseFactor = sc;
    return o;
  }
  // LinearTransform / LinearTransformInPlace (CryptoContextImpl, api/CryptoContext.hpp:460-517):
  // ct <- sum_(k < rowSize) Rot(ct, k stride + offset) * D_k by baby steps and giant steps, with
  // the reference's diagonal contract: diagonals[k] encodes Rot(D_k, r_k), r_k = -bStep (k / bStep)
  // stride - offset (GetLinearTransformPlaintextRotationIndices), at the level the products are
  // taken (ct's, one below for an unrescaled input, which is rescaled first).  The bStep baby
  // rotations by j stride are hoisted (one ModUp); the giant steps' inner products
  // sum_j Rot(ct, j stride) * diagonals[g bStep + j], of every diagonal set, are taken together
  // (dot_giant_steps, the reference's DotProductPtInternal); the giant steps fold from the top, the running sum rotated by
  // bStep stride before each is added, and by offset at the end.  Keys: j stride (1 <= j <= bStep)
  // and offset (GetLinearTransformRotationIndices).  The result keeps the level, at scale
  // ct x diagonal scale and degree + 1 (un-rescaled).
  static std::vector<int> GetLinearTransformRotationIndices(int bStep, int stride = 1, int offset = 0) {
    std::vector<int> r;
    for (int i = 1; i <= bStep; ++i) r.push_back(i * stride);
    if (offset != 0) r.push_back(offset);
    return r;
  }
  static std::vector<int> GetLinearTransformPlaintextRotationIndices(int rowSize, int bStep, int stride = 1,
                                                                    int offset = 0) {
    std::vector<int> r;
    for (int k = 0; k < rowSize; ++k) r.push_back(-bStep * (k / bStep) * stride - offset);
    return r;
  }
  std::vector<Ciphertext> LinearTransformMany(const Ciphertext& ct_in, int rowSize, int bStep,
                                              const std::vector<std::vector<const Plaintext*>>& sets, int stride = 1,
                                              int offset = 0) const {
    ct_in.need_two();
    if (rowSize <= 0 || bStep <= 0) throw Error(FIDES_ERR_ARG, "LinearTransform: rowSize and bStep must be positive");
    if (ct_in.NoiseLevel == 2) return LinearTransformMany(Rescale(ct_in), rowSize, bStep, sets, stride, offset);
    const int l = ct_in.getLevel();
    for (const auto& d : sets) {
      if ((int)d.size() < rowSize) throw Error(FIDES_ERR_ARG, "LinearTransform: fewer diagonals than rowSize");
      for (int k = 0; k < rowSize; ++k) {
        if (!d[k]) throw Error(FIDES_ERR_ARG, "LinearTransform: null diagonal");
        if (d[k]->level != l) throw Error(FIDES_ERR_LEVEL, "LinearTransform: diagonals must be at the ciphertext's level");
      }
    }
    bool ext = cc_->K > 0;  // every diagonal extended: the Q.P path (the reference's ext flag)
    for (const auto& d : sets)
      for (int k = 0; k < rowSize; ++k) ext = ext && d[k]->ext;
    if (ext) return linear_transform_ext(ct_in, rowSize, bStep, sets, stride, offset);
    const int nb = std::min(bStep, rowSize), gs = (rowSize + bStep - 1) / bStep;
    // baby steps: the input and its hoisted rotations by j stride
    std::vector<Ciphertext> baby;
    baby.push_back(copy_of(ct_in, l));
    if (nb > 1) {
      std::vector<int> rots;
      std::vector<const uint64_t*> keys;
      std::vector<uint64_t *> o0, o1;
      for (int j = 1; j < nb; ++j) {
        rots.push_back(j * stride);
        keys.push_back(cc_->GetRotationKey(j * stride).device());
        baby.push_back(fresh(l, ct_in.NoiseFactor, ct_in.NoiseLevel, ct_in.slots));
      }
      for (int j = 1; j < nb; ++j) o0.push_back(baby[j].c0()), o1.push_back(baby[j].c1());
      check(fides_rotate_hoisted(cc_->handle(), ct_in.c0(), ct_in.c1(), l, keys.data(), rots.data(), nb - 1,
                                 o0.data(), o1.data(), cc_->stream()));
    }
    // every giant step's inner product of every set first (fides_dot_plain_bsgs), then the folds
    const int ns = (int)sets.size();
    std::vector<Ciphertext> inner;  // [set][giant step]
    std::vector<const uint64_t *> x0, x1;
    std::vector<uint64_t *> o0, o1;
    for (int j = 0; j < nb; ++j) x0.push_back(baby[j].c0()), x1.push_back(baby[j].c1());
    for (int t = 0; t < ns * gs; ++t) {
      inner.push_back(fresh(l, ct_in.NoiseFactor * sets[t / gs][0]->scale, ct_in.NoiseLevel + 1, ct_in.slots));
      o0.push_back(inner.back().c0());
      o1.push_back(inner.back().c1());
    }
    dot_giant_steps(x0, x1, sets, rowSize, bStep, l, false, o0, o1);
    std::vector<Ciphertext> outs;
    for (int si = 0; si < ns; ++si) {
      Ciphertext acc = std::move(inner[(size_t)si * gs + gs - 1]);
      Ciphertext r = fresh(l, acc.NoiseFactor, acc.NoiseLevel, acc.slots);
      for (int g = gs - 2; g >= 0; --g) {
        const Ciphertext& in = inner[(size_t)si * gs + g];
        check(fides_rotate(cc_->handle(), acc.c0(), acc.c1(), l, cc_->GetRotationKey(bStep * stride).device(),
                           bStep * stride, r.c0(), r.c1(), cc_->stream()));
        check(fides_add(cc_->handle(), r.c0(), in.c0(), l, acc.c0(), cc_->stream()));
        check(fides_add(cc_->handle(), r.c1(), in.c1(), l, acc.c1(), cc_->stream()));
      }
      if (offset != 0) {
        check(fides_rotate(cc_->handle(), acc.c0(), acc.c1(), l, cc_->GetRotationKey(offset).device(), offset, r.c0(),
                           r.c1(), cc_->stream()));
        std::swap(acc, r);
      }
      cc_->synchronize();  // r is released at the end of the iteration
      outs.push_back(std::move(acc));
    }
    cc_->synchronize();  // the baby steps and inner products are released at scope exit
    return outs;
  }
  // Every giant step's inner product of every diagonal set, sets x giant steps outputs in that
  // order: up to 16 giant steps per launch (fides_dot_plain_bsgs, the reference's
  // DotProductPtInternal over all giant steps); more than 16 baby steps: one launch per giant
  // step (fides_dot_plain / fides_dot_plain_ext, up to 32 terms).
  void dot_giant_steps(const std::vector<const uint64_t*>& x0, const std::vector<const uint64_t*>& x1,
                       const std::vector<std::vector<const Plaintext*>>& sets, int rowSize, int bStep, int l, bool ext,
                       const std::vector<uint64_t*>& o0, const std::vector<uint64_t*>& o1) const {
    const int nb = (int)x0.size(), gs = (rowSize + bStep - 1) / bStep, total = (int)sets.size() * gs;
    constexpr int kGiant = 16, kBaby = 16;
    for (int t0 = 0; t0 < total; t0 += (nb <= kBaby ? kGiant : 1)) {
      const int ng = nb <= kBaby ? std::min(kGiant, total - t0) : 1;
      std::vector<const uint64_t*> pts((size_t)ng * nb, nullptr);
      int terms = 0;
      for (int i = 0; i < ng; ++i) {
        const int t = t0 + i, g = t % gs;
        const auto& d = sets[t / gs];
        for (int j = 0; j < nb && g * bStep + j < rowSize; ++j) pts[(size_t)i * nb + j] = d[g * bStep + j]->data();
      }
      if (nb <= kBaby) {
        check(fides_dot_plain_bsgs(cc_->handle(), x0.data(), x1.data(), nb, pts.data(), ng, l, ext ? 1 : 0,
                                   o0.data() + t0, o1.data() + t0, cc_->stream()));
        continue;
      }
      while (terms < nb && pts[terms]) ++terms;  // the last giant step may have fewer terms
      check((ext ? fides_dot_plain_ext : fides_dot_plain)(cc_->handle(), x0.data(), x1.data(), pts.data(), terms, l,
                                                          o0[t0], o1[t0], cc_->stream()));
    }
  }
  // P mod q_i for the first l Q primes (P: the product of the special primes)
  std::vector<uint64_t> p_mod_q(int l) const {
    std::vector<uint64_t> v(l);
    for (int i = 0; i < l; ++i) {
      unsigned __int128 r = 1;
      for (int k = 0; k < cc_->K; ++k) r = r * (cc_->primes[cc_->L + k] % q(i)) % q(i);
      v[i] = (uint64_t)r;
    }
    return v;
  }
  // LinearTransform over extended diagonals (the reference's fused branch with ext = true,
  // LinearTransform.cu:84-196): the baby steps are P ct and the hoisted rotations left in Q.P
  // (fides_rotate_hoisted_ext), each giant step's inner product is taken there
  // (fides_dot_plain_ext), and the giant-step fold keeps c0 in Q.P: before each step the running
  // sum's c1 is brought down and the sum rotated by bStep stride without ModDown, its extended c0
  // added as it is (a rotation by a multiple of N/2 slots is the identity and is skipped, as
  // there).  The transform ends with one ModDown of each component, or of c1 before the rotation
  // by offset, whose ModDown closes it.  Same diagonal contract, keys and result scale as the
  // Q-basis path; the rounding differs (one ModDown per component instead of one per rotation).
  std::vector<Ciphertext> linear_transform_ext(const Ciphertext& ct_in, int rowSize, int bStep,
                                               const std::vector<std::vector<const Plaintext*>>& sets, int stride,
                                               int offset) const {
    const int l = ct_in.getLevel(), e = l + cc_->K;
    const size_t Ne = (size_t)N() * e, Nq = (size_t)N() * l;
    auto* h = cc_->handle();
    auto st = cc_->stream();
    const int nb = std::min(bStep, rowSize), gs = (rowSize + bStep - 1) / bStep;
    std::vector<DeviceLimbs> b0, b1;  // baby steps in Q.P: P ct, then Rot(ct, j stride) before ModDown
    for (int j = 0; j < nb; ++j) b0.emplace_back(Ne), b1.emplace_back(Ne);
    const auto pm = p_mod_q(l);
    check(fides_mul_scalar(h, ct_in.c0(), l, pm.data(), b0[0].get(), st));
    check(fides_mul_scalar(h, ct_in.c1(), l, pm.data(), b1[0].get(), st));
    check_cuda(cudaMemsetAsync(b0[0].get() + Nq, 0, sizeof(uint64_t) * (Ne - Nq), st), "memset");
    check_cuda(cudaMemsetAsync(b1[0].get() + Nq, 0, sizeof(uint64_t) * (Ne - Nq), st), "memset");
    if (nb > 1) {
      std::vector<int> rots;
      std::vector<const uint64_t*> keys;
      std::vector<uint64_t *> o0, o1;
      for (int j = 1; j < nb; ++j) {
        rots.push_back(j * stride);
        keys.push_back(cc_->GetRotationKey(j * stride).device());
        o0.push_back(b0[j].get());
        o1.push_back(b1[j].get());
      }
      check(fides_rotate_hoisted_ext(h, ct_in.c0(), 0, ct_in.c1(), l, keys.data(), rots.data(), nb - 1, o0.data(),
                                     o1.data(), st));
    }
    DeviceLimbs a0(Ne), a1(Ne), t0(Ne), t1(Ne), c1q(Nq);
    // a rotation of the running sum (c0 in Q.P, c1 brought down first), into a0 / a1
    auto rotate_sum = [&](int r) {
      check(fides_moddown(h, a1.get(), l, c1q.get(), st));
      const uint64_t* key = cc_->GetRotationKey(r).device();
      uint64_t* r0 = t0.get();
      uint64_t* r1 = t1.get();
      check(fides_rotate_hoisted_ext(h, a0.get(), 1, c1q.get(), l, &key, &r, 1, &r0, &r1, st));
      std::swap(a0, t0);
      std::swap(a1, t1);
    };
    const int ns = (int)sets.size();
    std::vector<DeviceLimbs> i0, i1;  // every giant step's inner product in Q.P, [set][giant step]
    std::vector<const uint64_t *> x0, x1;
    std::vector<uint64_t *> o0, o1;
    for (int j = 0; j < nb; ++j) x0.push_back(b0[j].get()), x1.push_back(b1[j].get());
    for (int t = 0; t < ns * gs; ++t) {
      i0.emplace_back(Ne), i1.emplace_back(Ne);
      o0.push_back(i0.back().get());
      o1.push_back(i1.back().get());
    }
    dot_giant_steps(x0, x1, sets, rowSize, bStep, l, true, o0, o1);
    std::vector<Ciphertext> outs;
    for (int si = 0; si < ns; ++si) {
      const size_t top = (size_t)si * gs + gs - 1;
      std::swap(a0, i0[top]);
      std::swap(a1, i1[top]);
      for (int g = gs - 2; g >= 0; --g) {
        if ((bStep * stride) % (N() / 2) != 0) rotate_sum(bStep * stride);
        check(fides_add_ext(h, a0.get(), i0[(size_t)si * gs + g].get(), l, a0.get(), st));
        check(fides_add_ext(h, a1.get(), i1[(size_t)si * gs + g].get(), l, a1.get(), st));
      }
      if (offset != 0) rotate_sum(offset);
      Ciphertext o = fresh(l, ct_in.NoiseFactor * sets[si][0]->scale, ct_in.NoiseLevel + 1, ct_in.slots);
      check(fides_moddown(h, a0.get(), l, o.c0(), st));
      check(fides_moddown(h, a1.get(), l, o.c1(), st));
      outs.push_back(std::move(o));
    }
    cc_->synchronize();  // the Q.P buffers are released at scope exit
    return outs;
  }
  Ciphertext LinearTransform(const Ciphertext& ct, int rowSize, int bStep, const std::vector<const Plaintext*>& diagonals,
                             int stride = 1, int offset = 0) const {
    return std::move(LinearTransformMany(ct, rowSize, bStep, {diagonals}, stride, offset).at(0));
  }
  void LinearTransformInPlace(Ciphertext& ct, int rowSize, int bStep, const std::vector<const Plaintext*>& diagonals,
                              int stride = 1, int offset = 0) const {
    ct = LinearTransform(ct, rowSize, bStep, diagonals, stride, offset);
  }
  // In-place forms (CryptoContextImpl::*InPlace): the operand is replaced by the result.
  void EvalAddInPlace(Ciphertext& a, const Ciphertext& b) const { a = EvalAdd(a, b); }
  void EvalAddInPlace(Ciphertext& a, const Plaintext& p) const { a = EvalAdd(a, p); }
  void EvalAddInPlace(Ciphertext& a, double c) const { a = EvalAdd(a, c); }
  void EvalSubInPlace(Ciphertext& a, const Ciphertext& b) const { a = EvalSub(a, b); }
  void EvalSubInPlace(Ciphertext& a, const Plaintext& p) const { a = EvalSub(a, p); }
  void EvalSubInPlace(Ciphertext& a, double c) const { a = EvalSub(a, c); }
  void EvalMultInPlace(Ciphertext& a, const Ciphertext& b) const { a = EvalMult(a, b); }
  void EvalMultInPlace(Ciphertext& a, const Plaintext& p) const { a = EvalMult(a, p); }
  void EvalMultInPlace(Ciphertext& a, double c) const { a = EvalMult(a, c); }
  void EvalSquareInPlace(Ciphertext& a) const { a = EvalSquare(a); }
  void EvalNegateInPlace(Ciphertext& a) const { a = EvalNegate(a); }
  void RelinearizeInPlace(Ciphertext& a) const { a = Relinearize(a); }
  void RescaleInPlace(Ciphertext& a) const { a = Rescale(a); }
  void EvalRotateInPlace(Ciphertext& a, int index) const { a = EvalRotate(a, index); }
  void EvalChebyshevSeriesInPlace(Ciphertext& a, const std::vector<double>& coeffs, double lo, double hi) const {
    a = EvalChebyshevSeries(a, coeffs, lo, hi);
  }
  void MultByMonomialInPlace(Ciphertext& a, uint32_t power) const { a = MultByMonomial(a, power); }
  void AccumulateSumInPlace(Ciphertext& a, int slots, int stride = 1) const { a = AccumulateSum(a, slots, stride); }
  void EvalBootstrapInPlace(Ciphertext& a) const { a = EvalBootstrap(a); }
  void EvalBootstrapToLevelInPlace(Ciphertext& a, uint32_t outputLevel) { a = EvalBootstrapToLevel(a, outputLevel); }
  // AccumulateSum (CryptoContextImpl::AccumulateSum, CudaEngine::accumulateSum): slot i gathers
  // slots i + j stride, j < slots, by rounds of hoisted rotations summed in the extended basis
  // (fides_accumulate, radix 4 as the reference's default PARTIAL_SUM_RADIX); the rotation keys
  // of fides_accumulate_rotations must be registered.  Level and scale unchanged.
  Ciphertext AccumulateSum(const Ciphertext& a, int slots, int stride = 1, int radix = 4) const {
    a.need_two();
    const int n = fides_accumulate_rotations(radix, stride, slots, nullptr, 0);
    if (n < 0) throw Error(n, "AccumulateSum: bad radix, stride or slot count");
    std::vector<int> rots(n);
    fides_accumulate_rotations(radix, stride, slots, rots.data(), n);
    std::vector<const uint64_t*> keys;
    for (int r : rots) keys.push_back(cc_->GetRotationKey(r).device());
    Ciphertext o = fresh(a.getLevel(), a.NoiseFactor, a.NoiseLevel, a.slots);
    check(fides_accumulate(cc_->handle(), a.c0(), a.c1(), a.getLevel(), radix, stride, slots, rots.data(),
                           keys.data(), n, o.c0(), o.c1(), cc_->stream()));
    return o;
  }
  // MultByMonomial (CryptoContextImpl::MultByMonomial): every component times X^power in
  // Z_q[X]/(X^N + 1) (X^N = -1, so power is taken modulo 2N); level, scale and degree unchanged.
  // The monomial's limbs are transformed on the device and multiplied in, one product per limb.
  Ciphertext MultByMonomial(const Ciphertext& a, uint32_t power) const {
    const int l = a.getLevel(), n = N();
    power %= 2u * (uint32_t)n;
    const bool neg = power >= (uint32_t)n;
    std::vector<uint64_t> host((size_t)l * n, 0);
    for (int i = 0; i < l; ++i) host[(size_t)i * n + power % n] = neg ? q(i) - 1 : 1;
    DeviceLimbs mono((size_t)l * n);
    check_cuda(cudaMemcpyAsync(mono.get(), host.data(), sizeof(uint64_t) * host.size(), cudaMemcpyHostToDevice,
                               cc_->stream()),
               "H2D");
    check(fides_ntt_polys(cc_->handle(), mono.get(), 1, l, 0, cc_->stream()));
    Ciphertext o = copy_of(a, l);
    check(fides_mul(cc_->handle(), a.c0(), mono.get(), l, o.c0(), cc_->stream()));
    check(fides_mul(cc_->handle(), a.c1(), mono.get(), l, o.c1(), cc_->stream()));
    if (a.hasC2()) check(fides_mul(cc_->handle(), a.c2(), mono.get(), l, o.c2(), cc_->stream()));
    cc_->synchronize();  // the host and device monomials are released at scope exit
    return o;
  }
  // EvalNegate (CryptoContextImpl::EvalNegate): every component times -1
  Ciphertext EvalNegate(const Ciphertext& a) const {
    const int l = a.getLevel();
    const auto m1 = residues(-1.0, l);
    Ciphertext o = copy_of(a, l);
    check(fides_mul_scalar(cc_->handle(), a.c0(), l, m1.data(), o.c0(), cc_->stream()));
    check(fides_mul_scalar(cc_->handle(), a.c1(), l, m1.data(), o.c1(), cc_->stream()));
    if (a.hasC2()) check(fides_mul_scalar(cc_->handle(), a.c2(), l, m1.data(), o.c2(), cc_->stream()));
    return o;
  }
  // EvalAddMany (CryptoContextImpl::EvalAddMany): the sum of the ciphertexts, left to right
  Ciphertext EvalAddMany(const std::vector<const Ciphertext*>& cts) const {
    if (cts.empty()) throw Error(FIDES_ERR_ARG, "no ciphertexts");
    Ciphertext acc = copy_of(*cts[0], cts[0]->getLevel());
    for (size_t i = 1; i < cts.size(); ++i) acc = EvalAdd(acc, *cts[i]);
    return acc;
  }

  // ---- multiplicative operations (EvalMult, EvalSquare, Rescale)
  Ciphertext EvalMult(const Ciphertext& a, const Ciphertext& b) const {
    a.need_two();
    b.need_two();
    if (tech_ == FIXEDMANUAL) {
      const int l = std::min(a.getLevel(), b.getLevel());
      Ciphertext A = copy_of(a, l), B = copy_of(b, l);
      Ciphertext o = fresh(l, a.NoiseFactor * b.NoiseFactor, a.NoiseLevel + b.NoiseLevel, a.slots);
      check(fides_hmult(cc_->handle(), A.c0(), A.c1(), B.c0(), B.c1(), l, cc_->GetEvalKey().device(), 0, o.c0(),
                        o.c1(), cc_->stream()));
      cc_->synchronize();
      return o;
    }
    const int l = std::min(a.getLevel(), b.getLevel());
    if (l < 2) throw Error(FIDES_ERR_LEVEL, "no level left for the product's rescale");
    Ciphertext A = AdjustToLevel(a, l), B = AdjustToLevel(b, l);
    Ciphertext o = fresh(l - 1, S_[l - 1], 1, a.slots);
    check(fides_hmult(cc_->handle(), A.c0(), A.c1(), B.c0(), B.c1(), l, cc_->GetEvalKey().device(), 1, o.c0(),
                      o.c1(), cc_->stream()));
    cc_->synchronize();
    return o;
  }
  Ciphertext EvalSquare(const Ciphertext& a) const { return EvalMult(a, a); }
  // Multiplication by a plaintext (Ciphertext::multPt): both components times the plaintext on
  // the lower of the two levels.  FIXEDMANUAL: scale product, degree + 1, no rescale.
  // FLEXIBLEAUTO: the ciphertext at its canonical scale, the product rescaled (level l - 1,
  // scale S_l p.scale / q_(l-1), which is S_(l-1) for a plaintext at the canonical S_l).
  Ciphertext EvalMult(const Ciphertext& a, const Plaintext& p) const {
    a.need_two();
    const int l = std::min(a.getLevel(), p.level);
    if (tech_ == FIXEDMANUAL) {
      Ciphertext o = fresh(l, a.NoiseFactor * p.scale, a.NoiseLevel + 1, a.slots);
      check(fides_mul(cc_->handle(), a.c0(), p.data(), l, o.c0(), cc_->stream()));
      check(fides_mul(cc_->handle(), a.c1(), p.data(), l, o.c1(), cc_->stream()));
      return o;
    }
    if (l < 2) throw Error(FIDES_ERR_LEVEL, "no level left for the product's rescale");
    Ciphertext A = AdjustToLevel(a, l);
    Ciphertext t = fresh(l, 0, 1, a.slots);
    check(fides_mul(cc_->handle(), A.c0(), p.data(), l, t.c0(), cc_->stream()));
    check(fides_mul(cc_->handle(), A.c1(), p.data(), l, t.c1(), cc_->stream()));
    Ciphertext o = fresh(l - 1, S_[l] * p.scale / (double)q(l - 1), 1, a.slots);
    check(fides_rescale(cc_->handle(), t.c0(), l, o.c0(), cc_->stream()));
    check(fides_rescale(cc_->handle(), t.c1(), l, o.c1(), cc_->stream()));
    cc_->synchronize();  // t is released at scope exit
    return o;
  }
  // Multiplication by a real constant: FLEXIBLEAUTO lands on level l - 1 at S_(l-1); FIXEDMANUAL
  // multiplies by round(c q_(l-1)) and raises the degree (the next Rescale divides q_(l-1) out).
  Ciphertext EvalMult(const Ciphertext& a, double c) const {
    a.need_two();
    const int l = a.getLevel();
    if (tech_ == FIXEDMANUAL) {
      const double k = round_even(c * (double)q(l - 1));
      const auto s = residues(k, l);
      Ciphertext o = fresh(l, a.NoiseFactor * (double)q(l - 1), a.NoiseLevel + 1, a.slots);
      check(fides_mul_scalar(cc_->handle(), a.c0(), l, s.data(), o.c0(), cc_->stream()));
      check(fides_mul_scalar(cc_->handle(), a.c1(), l, s.data(), o.c1(), cc_->stream()));
      return o;
    }
    if (l < 2) throw Error(FIDES_ERR_LEVEL, "no level left for the product's rescale");
    const double k = round_even(c * S_[l - 1] * (double)q(l - 1) / a.NoiseFactor);
    return mul_int_rescale(a, l, k, S_[l - 1]);
  }
  // FIXEDMANUAL: divides by the top prime and drops it.  FLEXIBLEAUTO: products are already
  // rescaled (a copy), except the unrescaled ones of EvalMultNoRelin, which land on S_(l-1).
  Ciphertext Rescale(const Ciphertext& a) const {
    if (tech_ == FLEXIBLEAUTO && a.NoiseLevel != 2) return copy_of(a, a.getLevel());
    Ciphertext o = copy_of(a, a.getLevel());
    o.rescale();
    return o;
  }

  // EvalMultNoRelin (CryptoContextImpl::EvalMultNoRelin): the tensor product (a0 b0, a0 b1 +
  // a1 b0, a1 b1) of two ciphertexts on the lower level, without key switching: three components
  // until Relinearize.  Scale = product of the operands' (FLEXIBLEAUTO: operands first brought to
  // that level's canonical scale, so S_l^2), degree = sum.
  Ciphertext EvalMultNoRelin(const Ciphertext& a, const Ciphertext& b) const {
    a.need_two();
    b.need_two();
    const int l = std::min(a.getLevel(), b.getLevel());
    Ciphertext A = tech_ == FLEXIBLEAUTO ? AdjustToLevel(a, l) : copy_of(a, l);
    Ciphertext B = tech_ == FLEXIBLEAUTO ? AdjustToLevel(b, l) : copy_of(b, l);
    Ciphertext o = fresh(l, A.NoiseFactor * B.NoiseFactor, A.NoiseLevel + B.NoiseLevel, a.slots);
    o.c2_ = DeviceLimbs((size_t)N() * l);
    check(fides_tensor(cc_->handle(), A.c0(), A.c1(), B.c0(), B.c1(), l, o.c0(), o.c1(), o.c2(), cc_->stream()));
    cc_->synchronize();  // A and B are released at scope exit
    return o;
  }
  // Relinearize (CryptoContextImpl::Relinearize): the third component key-switched with the
  // relinearisation key and added, (c0 + f0, c1 + f1); level, scale and degree unchanged.  Equal
  // residue for residue to EvalMult's product before its rescale.
  Ciphertext Relinearize(const Ciphertext& a) const {
    const int l = a.getLevel();
    if (!a.hasC2()) return copy_of(a, l);
    Ciphertext o = fresh(l, a.NoiseFactor, a.NoiseLevel, a.slots);
    DeviceLimbs f0((size_t)N() * l), f1((size_t)N() * l);
    check(fides_keyswitch(cc_->handle(), a.c2(), l, cc_->GetEvalKey().device(), f0.get(), f1.get(), cc_->stream()));
    check(fides_add(cc_->handle(), a.c0(), f0.get(), l, o.c0(), cc_->stream()));
    check(fides_add(cc_->handle(), a.c1(), f1.get(), l, o.c1(), cc_->stream()));
    cc_->synchronize();  // f0 and f1 are released at scope exit
    return o;
  }

  // ---- rotations (EvalRotate, EvalFastRotationPrecompute, EvalFastRotation)
  Ciphertext EvalRotate(const Ciphertext& a, int index) const {
    a.need_two();
    Ciphertext o = fresh(a.getLevel(), a.NoiseFactor, a.NoiseLevel, a.slots);
    check(fides_rotate(cc_->handle(), a.c0(), a.c1(), a.getLevel(), cc_->GetRotationKey(index).device(), index,
                       o.c0(), o.c1(), cc_->stream()));
    return o;
  }
  std::shared_ptr<FastRotationPrecompute> EvalFastRotationPrecompute(const Ciphertext& a) const {
    a.need_two();
    auto p = std::make_shared<FastRotationPrecompute>();
    const int l = a.getLevel(), beta = (l + fides_ctx_alpha(cc_->handle()) - 1) / fides_ctx_alpha(cc_->handle());
    p->level = l;
    p->digits = DeviceLimbs((size_t)beta * (l + cc_->K) * N());
    check(fides_modup(cc_->handle(), a.c1(), l, p->digits.get(), cc_->stream()));
    return p;
  }
  // `m` (the cyclotomic order 2N) is accepted for signature parity with the reference.
  Ciphertext EvalFastRotation(const Ciphertext& a, int index, uint32_t m,
                              const std::shared_ptr<FastRotationPrecompute>& pre) const {
    (void)m;
    auto v = EvalFastRotation(a, std::vector<int>{index}, pre);
    return std::move(v.at(0));
  }
  // EvalRotateMany (CryptoContextImpl::EvalRotateMany, CudaEngine::evalRotateMany): every
  // ciphertext rotated by the same index, all in one launch sequence (fides_rotate_batch).
  std::vector<Ciphertext> EvalRotateMany(const std::vector<const Ciphertext*>& cts, int index) const {
    std::vector<Ciphertext> outs;
    std::vector<fides_rotate_item> items;
    const uint64_t* key = cc_->GetRotationKey(index).device();
    const uint32_t k = fides_rotation_auto_index(cc_->logN, index);
    for (const Ciphertext* c : cts) {
      c->need_two();
      outs.push_back(fresh(c->getLevel(), c->NoiseFactor, c->NoiseLevel, c->slots));
    }
    for (size_t i = 0; i < cts.size(); ++i)
      items.push_back(fides_rotate_item{cts[i]->c0(), cts[i]->c1(), outs[i].c0(), outs[i].c1(), key,
                                        cts[i]->getLevel(), k});
    if (!items.empty()) check(fides_rotate_batch(cc_->handle(), items.data(), (int)items.size(), cc_->stream()));
    return outs;
  }
  // Several indexes from one precomputation, in one launch sequence.
  std::vector<Ciphertext> EvalFastRotation(const Ciphertext& a, const std::vector<int>& indexes,
                                           const std::shared_ptr<FastRotationPrecompute>& pre) const {
    if (!pre || pre->level != a.getLevel()) throw Error(FIDES_ERR_STATE, "precomputation of another level");
    std::vector<Ciphertext> outs;
    std::vector<const uint64_t*> keys;
    std::vector<uint64_t*> o0, o1;
    for (int r : indexes) {
      outs.push_back(fresh(a.getLevel(), a.NoiseFactor, a.NoiseLevel, a.slots));
      keys.push_back(cc_->GetRotationKey(r).device());
    }
    for (auto& o : outs) {
      o0.push_back(o.c0());
      o1.push_back(o.c1());
    }
    check(fides_rotate_hoisted_digits(cc_->handle(), a.c0(), pre->digits.get(), a.getLevel(), keys.data(),
                                      indexes.data(), (int)indexes.size(), o0.data(), o1.data(), cc_->stream()));
    return outs;
  }

  // ---- bootstrapping (EvalBootstrapSetup, EvalBootstrapKeyGen's key list, EvalBootstrap)
  // levelBudget = {CoeffsToSlots levels, SlotsToCoeffs levels}; dim1 (BSGS baby steps; 0 = 8);
  // numSlots must be N/2 (full packing) or 0; correctionFactor = the input prescale in bits (0 =
  // none).  msgScale = the scale of the inputs' slots (0 = the canonical level-1 scale S_1).
  void EvalBootstrapSetup(std::vector<uint32_t> levelBudget = {3, 3}, std::vector<uint32_t> dim1 = {0, 0},
                          uint32_t numSlots = 0, uint32_t correctionFactor = 0, double msgScale = 0) {
    if (numSlots != 0 && (int)numSlots != N() / 2)
      throw Error(FIDES_ERR_ARG, "bootstrapping supports full packing (N/2 slots) only");
    if (levelBudget.size() != 2) throw Error(FIDES_ERR_ARG, "levelBudget = {CoeffsToSlots, SlotsToCoeffs}");
    drop_short_boots();
    if (boot_) fides_boot_destroy(boot_), boot_ = nullptr;
    boot_msg_scale_ = msgScale > 0 ? msgScale : S_[1];
    fides_boot_params p{(int)levelBudget[0], (int)levelBudget[1], cc_->L, S_[cc_->L], boot_msg_scale_, 12, 3, 31,
                        dim1.empty() || dim1[0] == 0 ? 8 : (int)dim1[0], (int)correctionFactor,
                        to_sparse_ && to_dense_ ? 1 : 0, 0, boot_double_hoist_ ? 1 : 0};
    check(fides_boot_create(cc_->handle(), &p, &boot_));
    boot_params_ = p;
  }
  // Double-hoisted linear transforms in the bootstrap (fides_boot_params::double_hoist; on by
  // default, about 8-10 % faster).  Set before EvalBootstrapSetup; off gives the single-hoisted
  // form's results bit for bit.
  void SetBootstrapDoubleHoisting(bool on) { boot_double_hoist_ = on; }
  // Rotation indexes whose keys EvalBootstrap needs (register them with Context::AddRotationKey,
  // with the conjugation key 2N - 1 and the relinearisation key).
  std::vector<int> GetBootstrapRotations() const {
    if (!boot_) throw Error(FIDES_ERR_STATE, "EvalBootstrapSetup first");
    std::vector<int> r(fides_boot_rotations(boot_, nullptr, 0));
    fides_boot_rotations(boot_, r.data(), (int)r.size());
    return r;
  }
  // Sparse-secret encapsulation keys (dense -> sparse, sparse -> dense), set before
  // EvalBootstrapSetup (the reference's keySwitchSparse, src/CKKS/Bootstrap.cu:257-290).
  void SetSparseEncapsulationKeys(KeySwitchingKey&& to_sparse, KeySwitchingKey&& to_dense) {
    to_sparse_ = std::make_unique<KeySwitchingKey>(std::move(to_sparse));
    to_dense_ = std::make_unique<KeySwitchingKey>(std::move(to_dense));
  }
  // Binds the context's keys and encodes the linear transforms (once, after the keys are in).
  void EvalBootstrapPrepare() {
    if (!boot_) throw Error(FIDES_ERR_STATE, "EvalBootstrapSetup first");
    check(fides_boot_set_keys(boot_, cc_->GetEvalKey().device(), cc_->GetRotationKey(2 * N() - 1).device(),
                              to_sparse_ ? to_sparse_->device() : nullptr, to_dense_ ? to_dense_->device() : nullptr));
    for (int r : GetBootstrapRotations()) check(fides_boot_set_rotation_key(boot_, r, cc_->GetRotationKey(r).device()));
    check(fides_boot_prepare(boot_, cc_->stream()));
  }
  // The input's limb q_0 is bootstrapped; its slots must be at the setup's msgScale.
  Ciphertext EvalBootstrap(const Ciphertext& a) const {
    a.need_two();
    if (!boot_) throw Error(FIDES_ERR_STATE, "EvalBootstrapSetup first");
    int lo = 0;
    double sc = 0;
    check(fides_boot_levels(boot_, &lo, &sc));
    Ciphertext o = fresh(lo, sc, 1, a.slots);
    check(fides_bootstrap(boot_, a.c0(), a.c1(), o.c0(), o.c1(), cc_->stream()));
    cc_->synchronize();
    return o;
  }
  // EvalBootstrapToLevel (CryptoContextImpl::EvalBootstrapToLevel): the refreshed ciphertext at
  // `outputLevel` consumed towers (OpenFHE's level: L minus the limbs kept), or at EvalBootstrap's
  // own level when that consumes at least as many.  A deeper request runs the same circuit on a
  // chain cut short at the top (ModRaise to fewer limbs), so every step moves fewer limbs; that
  // bootstrapper is built and prepared with the same parameters and keys on first use of each
  // depth and kept.  Precision is the bootstrap's own: the scales of the shorter chain are the
  // canonical ones of its levels.
  Ciphertext EvalBootstrapToLevel(const Ciphertext& a, uint32_t outputLevel) {
    a.need_two();
    if (!boot_) throw Error(FIDES_ERR_STATE, "EvalBootstrapSetup first");
    int lo = 0;
    double sc = 0;
    check(fides_boot_levels(boot_, &lo, &sc));
    const int L = cc_->L, consumed = L - lo;
    if ((int)outputLevel <= consumed) return EvalBootstrap(a);
    if ((int)outputLevel >= L) throw Error(FIDES_ERR_LEVEL, "the output level leaves no limb");
    const int top = L - ((int)outputLevel - consumed);
    fides_boot*& b = short_boot_[top];
    if (!b) {
      fides_boot_params p = boot_params_;
      p.top_level = top;  // top_scale stays the chain's S_L: the bootstrapper indexes scales by level
      try {
        check(fides_boot_create(cc_->handle(), &p, &b));
        check(fides_boot_set_keys(b, cc_->GetEvalKey().device(), cc_->GetRotationKey(2 * N() - 1).device(),
                                  to_sparse_ ? to_sparse_->device() : nullptr,
                                  to_dense_ ? to_dense_->device() : nullptr));
        std::vector<int> r(fides_boot_rotations(b, nullptr, 0));
        fides_boot_rotations(b, r.data(), (int)r.size());
        for (int x : r) check(fides_boot_set_rotation_key(b, x, cc_->GetRotationKey(x).device()));
        check(fides_boot_prepare(b, cc_->stream()));
      } catch (...) {
        if (b) fides_boot_destroy(b);
        short_boot_.erase(top);
        throw;
      }
    }
    check(fides_boot_levels(b, &lo, &sc));
    Ciphertext o = fresh(lo, sc, 1, a.slots);
    check(fides_bootstrap(b, a.c0(), a.c1(), o.c0(), o.c1(), cc_->stream()));
    cc_->synchronize();
    return o;
  }
  // Several inputs bootstrapped concurrently (one stream each); results equal EvalBootstrap's.
  std::vector<Ciphertext> EvalBootstrap(const std::vector<const Ciphertext*>& in) const {
    if (!boot_) throw Error(FIDES_ERR_STATE, "EvalBootstrapSetup first");
    int lo = 0;
    double sc = 0;
    check(fides_boot_levels(boot_, &lo, &sc));
    std::vector<Ciphertext> outs;
    std::vector<const uint64_t *> c0, c1;
    std::vector<uint64_t *> o0, o1;
    for (const Ciphertext* a : in) {
      outs.push_back(fresh(lo, sc, 1, a->slots));
      c0.push_back(a->c0());
      c1.push_back(a->c1());
    }
    for (auto& o : outs) {
      o0.push_back(o.c0());
      o1.push_back(o.c1());
    }
    check(fides_bootstrap_batch(boot_, (int)in.size(), c0.data(), c1.data(), o0.data(), o1.data(), cc_->stream()));
    cc_->synchronize();
    return outs;
  }

 private:
  void drop_short_boots() {
    for (auto& kv : short_boot_)
      if (kv.second) fides_boot_destroy(kv.second);
    short_boot_.clear();
  }
  Ciphertext add_sub(const Ciphertext& a, const Ciphertext& b, bool sub) const {
    if (tech_ == FLEXIBLEAUTO && (a.NoiseLevel == 2 || b.NoiseLevel == 2) &&
        !(a.NoiseLevel == 2 && b.NoiseLevel == 2 && a.getLevel() == b.getLevel())) {
      // unrescaled products meet only their like at the same level; otherwise rescale first
      if (a.NoiseLevel == 2 && b.NoiseLevel == 2) return add_sub(Rescale(a), Rescale(b), sub);
      if (a.NoiseLevel == 2) return add_sub(Rescale(a), b, sub);
      return add_sub(a, Rescale(b), sub);
    }
    const int l = std::min(a.getLevel(), b.getLevel());
    Ciphertext A = AdjustToLevel(a, l), B = AdjustToLevel(b, l);
    if (A.NoiseLevel != B.NoiseLevel || !same_scale(A.NoiseFactor, B.NoiseFactor))
      throw Error(FIDES_ERR_STATE, "operands at different scales (rescale first)");
    Ciphertext o = fresh(l, A.NoiseFactor, A.NoiseLevel, a.slots);
    auto f = sub ? fides_sub : fides_add;
    check(f(cc_->handle(), A.c0(), B.c0(), l, o.c0(), cc_->stream()));
    check(f(cc_->handle(), A.c1(), B.c1(), l, o.c1(), cc_->stream()));
    if (A.hasC2() || B.hasC2()) {  // a missing third component is zero
      o.c2_ = DeviceLimbs((size_t)N() * l);
      const size_t bytes = sizeof(uint64_t) * (size_t)N() * l;
      if (A.hasC2() && B.hasC2())
        check(f(cc_->handle(), A.c2(), B.c2(), l, o.c2(), cc_->stream()));
      else if (A.hasC2())
        check_cuda(cudaMemcpyAsync(o.c2(), A.c2(), bytes, cudaMemcpyDeviceToDevice, cc_->stream()), "D2D");
      else if (!sub)
        check_cuda(cudaMemcpyAsync(o.c2(), B.c2(), bytes, cudaMemcpyDeviceToDevice, cc_->stream()), "D2D");
      else
        check(fides_mul_scalar(cc_->handle(), B.c2(), l, residues(-1.0, l).data(), o.c2(), cc_->stream()));
    }
    cc_->synchronize();
    return o;
  }
  Ciphertext add_const(const Ciphertext& a, double c) const {
    const int l = a.getLevel();
    const auto s = residues(round_even(c * a.NoiseFactor), l);
    Ciphertext o = copy_of(a, l);
    check(fides_add_scalar(cc_->handle(), a.c0(), l, s.data(), o.c0(), cc_->stream()));
    return o;
  }
};

}  // namespace B200
}  // namespace FIDESlib
