// Test driver of the C++ evaluation facade (CryptoContextB200.hpp), loaded by the GPU test suite
// (tests/test_bootstrap.py) as a shared library: it builds its own Context from the primes,
// imports the evaluation keys from device arrays (KeySwitchingKey::InitializeFlat), loads host
// ciphertexts through RawCipherText, runs the facade's calls and stores every result back to
// host arrays for the suite to compare with the oracle, the Python driver and the C ABI.
#include <cstdio>
#include <cstring>
#include <vector>

#include "CryptoContextB200.hpp"

using namespace FIDESlib::B200;

namespace {
RawCipherText raw_of(const uint64_t* c0, const uint64_t* c1, int l, int N, double scale) {
  RawCipherText r;
  r.N = N;
  r.numRes = l;
  r.Noise = scale;
  r.NoiseLevel = 1;
  for (int i = 0; i < l; ++i) {
    r.sub_0.emplace_back(c0 + (size_t)i * N, c0 + (size_t)(i + 1) * N);
    r.sub_1.emplace_back(c1 + (size_t)i * N, c1 + (size_t)(i + 1) * N);
  }
  return r;
}
void put(const Ciphertext& ct, uint64_t*& out) {
  RawCipherText r;
  ct.store(r);
  for (auto& v : r.sub_0) out = std::copy(v.begin(), v.end(), out);
  for (auto& v : r.sub_1) out = std::copy(v.begin(), v.end(), out);
}
KeySwitchingKey key_from(Context& cc, const uint64_t* dev) {
  KeySwitchingKey k(cc);
  k.InitializeFlat(dev);
  return k;
}
}  // namespace

extern "C" {

// The facade's bootstrap of n_boot level-1 ciphertexts (host arrays, one limb each): singly
// (EvalBootstrap) into boot_out0/1 and as one batch (the vector form) into batch_out0/1, each
// output of *out_level limbs.  Keys are device arrays of the caller's context; rots lists the
// rotation keys given (every rotation GetBootstrapRotations names must be among them).
int facade_bootstrap(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale,
                     const uint64_t* relin, const uint64_t* conj, int n_rot, const int* rots,
                     const uint64_t* const* rot_keys, const uint64_t* to_sparse, const uint64_t* to_dense,
                     double msg_scale, int prescale_bits, int double_hoist, int n_boot, const uint64_t* const* c0s,
                     const uint64_t* const* c1s, uint64_t* const* out0, uint64_t* const* out1, uint64_t* const* bo0,
                     uint64_t* const* bo1, int* out_level, double* out_scale, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    cc.AddEvalKey(key_from(cc, relin));
    cc.AddRotationKey(2 * N - 1, key_from(cc, conj));
    for (int i = 0; i < n_rot; ++i) cc.AddRotationKey(rots[i], key_from(cc, rot_keys[i]));
    {
      CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
      if (to_sparse && to_dense) ev.SetSparseEncapsulationKeys(key_from(cc, to_sparse), key_from(cc, to_dense));
      ev.SetBootstrapDoubleHoisting(double_hoist != 0);
      ev.EvalBootstrapSetup({3, 3}, {0, 0}, (uint32_t)(N / 2), (uint32_t)prescale_bits, msg_scale);
      ev.EvalBootstrapPrepare();
      std::vector<Ciphertext> in;
      for (int i = 0; i < n_boot; ++i) in.emplace_back(cc, raw_of(c0s[i], c1s[i], 1, N, msg_scale));
      std::vector<const Ciphertext*> ptrs;
      for (auto& c : in) ptrs.push_back(&c);
      auto batch = ev.EvalBootstrap(ptrs);
      for (int i = 0; i < n_boot; ++i) {
        Ciphertext o = ev.EvalBootstrap(in[i]);
        *out_level = o.getLevel();
        *out_scale = o.NoiseFactor;
        uint64_t* w = out0[i];
        RawCipherText r;
        o.store(r);
        for (auto& v : r.sub_0) w = std::copy(v.begin(), v.end(), w);
        w = out1[i];
        for (auto& v : r.sub_1) w = std::copy(v.begin(), v.end(), w);
        RawCipherText rb;
        batch[i].store(rb);
        w = bo0[i];
        for (auto& v : rb.sub_0) w = std::copy(v.begin(), v.end(), w);
        w = bo1[i];
        for (auto& v : rb.sub_1) w = std::copy(v.begin(), v.end(), w);
      }
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// EvalBootstrap and EvalBootstrapToLevel of one level-1 ciphertext (setup as facade_bootstrap,
// dense secret, no encapsulation): out_d0/1 = EvalBootstrap [*lvl_d limbs], out_s0/1 =
// EvalBootstrapToLevel(consumed, the default's consumed towers) [same], out_t0/1 =
// EvalBootstrapToLevel(consumed + extra) [*lvl_t limbs]; *sc_t its scale.
int facade_bootstrap_to_level(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale,
                              const uint64_t* relin, const uint64_t* conj, int n_rot, const int* rots,
                              const uint64_t* const* rot_keys, double msg_scale, int prescale_bits, int extra,
                              const uint64_t* c0, const uint64_t* c1, uint64_t* out_d0, uint64_t* out_d1,
                              uint64_t* out_s0, uint64_t* out_s1, uint64_t* out_t0, uint64_t* out_t1, int* lvl_d,
                              int* lvl_t, double* sc_t, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    cc.AddEvalKey(key_from(cc, relin));
    cc.AddRotationKey(2 * N - 1, key_from(cc, conj));
    for (int i = 0; i < n_rot; ++i) cc.AddRotationKey(rots[i], key_from(cc, rot_keys[i]));
    CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
    ev.EvalBootstrapSetup({3, 3}, {0, 0}, (uint32_t)(N / 2), (uint32_t)prescale_bits, msg_scale);
    ev.EvalBootstrapPrepare();
    Ciphertext in(cc, raw_of(c0, c1, 1, N, msg_scale));
    auto dump = [&](const Ciphertext& o, uint64_t* w0, uint64_t* w1) {
      RawCipherText r;
      o.store(r);
      for (auto& v : r.sub_0) w0 = std::copy(v.begin(), v.end(), w0);
      for (auto& v : r.sub_1) w1 = std::copy(v.begin(), v.end(), w1);
    };
    Ciphertext d = ev.EvalBootstrap(in);
    *lvl_d = d.getLevel();
    dump(d, out_d0, out_d1);
    const uint32_t consumed = (uint32_t)(n_q - d.getLevel());
    dump(ev.EvalBootstrapToLevel(in, consumed), out_s0, out_s1);
    Ciphertext t = ev.EvalBootstrapToLevel(in, consumed + (uint32_t)extra);
    *lvl_t = t.getLevel();
    *sc_t = t.NoiseFactor;
    dump(t, out_t0, out_t1);
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// The facade's arithmetic on a and b (host, level l, scale S_l of a FLEXIBLEAUTO chain from
// top_scale), results packed into out in this order:
//   EvalMult(a, b) [l-1] | EvalRotate(a, rot) [l] | EvalFastRotation(a, rot) from
//   EvalFastRotationPrecompute(a) [l] | EvalAdd(a, b) [l] | EvalSub(a, b) [l] |
//   EvalAdd(a, 0.25) [l] | EvalMult(a, 0.5) [l-1] | EvalSquare(a) [l-1] |
//   EvalMult(EvalMult(a, b), a) [l-2] (operands at different levels, adjusted)
// each as c0 limbs then c1 limbs.  And under FIXEDMANUAL (out_manual):
//   EvalMult(a, b) [l] (degree 2, not rescaled) | Rescale of it [l-1]
int facade_arith(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale, const uint64_t* relin,
                 int rot, const uint64_t* rot_key, int l, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
                 const uint64_t* b1, uint64_t* out, uint64_t* out_manual, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    cc.AddEvalKey(key_from(cc, relin));
    cc.AddRotationKey(rot, key_from(cc, rot_key));
    {
      CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
      const double S = ev.GetScalingFactorReal(l);
      Ciphertext A(cc, raw_of(a0, a1, l, N, S)), B(cc, raw_of(b0, b1, l, N, S));
      uint64_t* w = out;
      Ciphertext M = ev.EvalMult(A, B);
      put(M, w);
      put(ev.EvalRotate(A, rot), w);
      auto pre = ev.EvalFastRotationPrecompute(A);
      put(ev.EvalFastRotation(A, rot, 2 * N, pre), w);
      put(ev.EvalAdd(A, B), w);
      put(ev.EvalSub(A, B), w);
      put(ev.EvalAdd(A, 0.25), w);
      put(ev.EvalMult(A, 0.5), w);
      put(ev.EvalSquare(A), w);
      put(ev.EvalMult(M, A), w);
    }
    {
      CryptoContextImpl man(cc, FIXEDMANUAL, top_scale);
      Ciphertext A(cc, raw_of(a0, a1, l, N, 1.0)), B(cc, raw_of(b0, b1, l, N, 1.0));
      uint64_t* w = out_manual;
      Ciphertext M = man.EvalMult(A, B);
      if (M.NoiseLevel != 2 || M.getLevel() != l) throw Error(FIDES_ERR_STATE, "FIXEDMANUAL product metadata");
      put(M, w);
      Ciphertext R = man.Rescale(M);
      if (R.NoiseLevel != 1 || R.getLevel() != l - 1) throw Error(FIDES_ERR_STATE, "FIXEDMANUAL rescale metadata");
      put(R, w);
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// Plaintext operations of the facade on ciphertext (a0, a1) at l limbs: the plaintext of the
// n complex slots z = [n][re, im] encoded at level l (canonical scale S_l of top_scale), then,
// packed into out in this order: the plaintext's limbs [l] | FLEXIBLEAUTO EvalMult(A, P) [l-1] |
// EvalAdd(A, P) [l] | EvalSub(A, P) [l] | FIXEDMANUAL EvalMult(A, P) [l] (at scale 1 x S_l,
// degree 2), each ciphertext as c0 limbs then c1 limbs.
int facade_plain(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale, int l,
                 const uint64_t* a0, const uint64_t* a1, const double* z, int n, uint64_t* out, char* err,
                 int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    std::vector<std::complex<double>> slots(n);
    for (int i = 0; i < n; ++i) slots[i] = {z[2 * i], z[2 * i + 1]};
    uint64_t* w = out;
    {
      CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
      const double S = ev.GetScalingFactorReal(l);
      Plaintext P = ev.MakeCKKSPackedPlaintext(slots, l);
      if (P.level != l || P.scale != S) throw Error(FIDES_ERR_STATE, "plaintext metadata");
      check_cuda(cudaMemcpy(w, P.data(), sizeof(uint64_t) * (size_t)N * l, cudaMemcpyDeviceToHost), "D2H");
      w += (size_t)N * l;
      Ciphertext A(cc, raw_of(a0, a1, l, N, S));
      Ciphertext M = ev.EvalMult(A, P);
      if (M.getLevel() != l - 1 || std::abs(M.NoiseFactor / ev.GetScalingFactorReal(l - 1) - 1) > 1e-12)
        throw Error(FIDES_ERR_STATE, "EvalMult(plaintext) metadata");
      put(M, w);
      put(ev.EvalAdd(A, P), w);
      put(ev.EvalSub(A, P), w);
      bool refused = false;  // a plaintext at another scale is refused
      try {
        Plaintext Q = ev.MakeCKKSPackedPlaintext(slots, l, 2 * S);
        ev.EvalAdd(A, Q);
      } catch (const Error& e) {
        refused = e.code == FIDES_ERR_ARG;
      }
      if (!refused) throw Error(FIDES_ERR_STATE, "EvalAdd with a mismatched scale was not refused");
    }
    {
      CryptoContextImpl man(cc, FIXEDMANUAL, top_scale);
      Plaintext P = man.MakeCKKSPackedPlaintext(slots, l);
      Ciphertext A(cc, raw_of(a0, a1, l, N, 1.0));
      Ciphertext M = man.EvalMult(A, P);
      if (M.NoiseLevel != 2 || M.getLevel() != l) throw Error(FIDES_ERR_STATE, "FIXEDMANUAL plaintext product");
      put(M, w);
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// Unrelinearised products and the other CryptoContextImpl forms, on ciphertexts a, b at l limbs
// (top_scale as in facade_arith), packed into out in this order, each as c0 then c1 limbs:
//   FIXEDMANUAL Relinearize(EvalMultNoRelin(a, b)) [l] |
//   FIXEDMANUAL Relinearize(EvalAdd(EvalMultNoRelin(a, b), EvalMultNoRelin(a, a))) [l] |
//   FLEXIBLEAUTO Rescale(Relinearize(EvalMultNoRelin(a, b))) [l-1] | EvalNegate(a) [l] |
//   EvalAddMany({a, b, a}) [l] | EvalRotateMany({a, b}, rot) [l] [l] | MultByMonomial(a, N + 5) [l]
int facade_more(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale, const uint64_t* relin,
                int rot, const uint64_t* rot_key, int l, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0,
                const uint64_t* b1, uint64_t* out, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    cc.AddEvalKey(key_from(cc, relin));
    cc.AddRotationKey(rot, key_from(cc, rot_key));
    uint64_t* w = out;
    {
      CryptoContextImpl man(cc, FIXEDMANUAL, top_scale);
      Ciphertext A(cc, raw_of(a0, a1, l, N, 1.0)), B(cc, raw_of(b0, b1, l, N, 1.0));
      Ciphertext X = man.EvalMultNoRelin(A, B);
      if (!X.hasC2() || X.NoiseLevel != 2 || X.getLevel() != l) throw Error(FIDES_ERR_STATE, "EvalMultNoRelin");
      bool refused = false;  // three components go through Relinearize first
      try {
        man.EvalRotate(X, rot);
      } catch (const Error& e) {
        refused = e.code == FIDES_ERR_STATE;
      }
      if (!refused) throw Error(FIDES_ERR_STATE, "a three-component rotation was not refused");
      Ciphertext R = man.Relinearize(X);
      if (R.hasC2()) throw Error(FIDES_ERR_STATE, "Relinearize left a third component");
      {  // the in-place form gives the same residues
        Ciphertext Y = man.EvalMultNoRelin(A, B);
        man.RelinearizeInPlace(Y);
        RawCipherText r1, r2;
        Y.store(r1);
        R.store(r2);
        if (r1.sub_0 != r2.sub_0 || r1.sub_1 != r2.sub_1) throw Error(FIDES_ERR_STATE, "RelinearizeInPlace differs");
      }
      put(R, w);
      put(man.Relinearize(man.EvalAdd(X, man.EvalMultNoRelin(A, A))), w);
    }
    {
      CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
      const double S = ev.GetScalingFactorReal(l);
      Ciphertext A(cc, raw_of(a0, a1, l, N, S)), B(cc, raw_of(b0, b1, l, N, S));
      Ciphertext R = ev.Rescale(ev.Relinearize(ev.EvalMultNoRelin(A, B)));
      if (R.getLevel() != l - 1 || R.NoiseLevel != 1 || std::abs(R.NoiseFactor / ev.GetScalingFactorReal(l - 1) - 1) > 1e-12)
        throw Error(FIDES_ERR_STATE, "FLEXIBLEAUTO relinearised product metadata");
      put(R, w);
      put(ev.EvalNegate(A), w);
      put(ev.EvalAddMany({&A, &B, &A}), w);
      auto rs = ev.EvalRotateMany({&A, &B}, rot);
      put(rs.at(0), w);
      put(rs.at(1), w);
      put(ev.MultByMonomial(A, (uint32_t)N + 5), w);
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// EvalChebyshevSeries under FLEXIBLEAUTO on (a0, a1) at l limbs, canonical scale S_l of
// top_scale: out = the result's c0 then c1 limbs; *out_level / *out_scale its level and scale.
int facade_chebyshev(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale,
                     const uint64_t* relin, int l, const uint64_t* a0, const uint64_t* a1, const double* coeffs,
                     int n_coeffs, double lo, double hi, uint64_t* out, int* out_level, double* out_scale, char* err,
                     int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    cc.AddEvalKey(key_from(cc, relin));
    CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
    Ciphertext A(cc, raw_of(a0, a1, l, N, ev.GetScalingFactorReal(l)));
    Ciphertext R = ev.EvalChebyshevSeries(A, std::vector<double>(coeffs, coeffs + n_coeffs), lo, hi);
    uint64_t* w = out;
    put(R, w);
    *out_level = R.getLevel();
    *out_scale = R.NoiseFactor;
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// AccumulateSum(a, size, stride) under FLEXIBLEAUTO with the rotation keys (rots[i], keys[i]):
// out = the result's c0 then c1 limbs (l each).
int facade_accumulate(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale, int n_keys,
                      const int* rots, const uint64_t* const* keys, int l, const uint64_t* a0, const uint64_t* a1,
                      int size, int stride, uint64_t* out, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    for (int i = 0; i < n_keys; ++i) cc.AddRotationKey(rots[i], key_from(cc, keys[i]));
    CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
    Ciphertext A(cc, raw_of(a0, a1, l, N, ev.GetScalingFactorReal(l)));
    uint64_t* w = out;
    put(ev.AccumulateSum(A, size, stride), w);
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// LinearTransform under FLEXIBLEAUTO of (a0, a1) at l limbs (canonical scale), the rowSize
// diagonals given as slot vectors dz = [rowSize][n][re, im] (already pre-rotated by the caller),
// encoded at level l; and LinearTransformMany with the same diagonals and their negation.
// Each result is rescaled (Rescale: the transform leaves degree 2) and packed into out as c0
// then c1 limbs (l - 1 each): LinearTransform's, then LinearTransformMany's two; *out_scale the
// rescaled scale.  ext != 0: the diagonals are encoded over Q.P (MakeCKKSPackedPlaintextExtended),
// which takes the extended-basis path.
int facade_linear_transform(int logN, int n_q, int K, int dnum, const uint64_t* primes, double top_scale, int n_keys,
                            const int* rots, const uint64_t* const* keys, int l, const uint64_t* a0,
                            const uint64_t* a1, int row_size, int b_step, int stride, int offset, const double* dz,
                            int n, int ext, uint64_t* out, double* out_scale, char* err, int err_len) {
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes, primes + n_q);
    p.Sprimes.assign(primes + n_q, primes + n_q + K);
    Context cc(p);
    const int N = 1 << logN;
    for (int i = 0; i < n_keys; ++i) cc.AddRotationKey(rots[i], key_from(cc, keys[i]));
    CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
    Ciphertext A(cc, raw_of(a0, a1, l, N, ev.GetScalingFactorReal(l)));
    std::vector<Plaintext> pts, neg;
    for (int k = 0; k < row_size; ++k) {
      std::vector<std::complex<double>> v(n), w(n);
      for (int i = 0; i < n; ++i) {
        v[i] = {dz[((size_t)k * n + i) * 2], dz[((size_t)k * n + i) * 2 + 1]};
        w[i] = -v[i];
      }
      pts.push_back(ext ? ev.MakeCKKSPackedPlaintextExtended(v, l) : ev.MakeCKKSPackedPlaintext(v, l));
      neg.push_back(ext ? ev.MakeCKKSPackedPlaintextExtended(w, l) : ev.MakeCKKSPackedPlaintext(w, l));
    }
    std::vector<const Plaintext *> d, dn;
    for (auto& x : pts) d.push_back(&x);
    for (auto& x : neg) dn.push_back(&x);
    uint64_t* w = out;
    Ciphertext R = ev.LinearTransform(A, row_size, b_step, d, stride, offset);
    if (R.NoiseLevel != 2 || R.getLevel() != l) throw Error(FIDES_ERR_STATE, "LinearTransform result metadata");
    Ciphertext Rr = ev.Rescale(R);
    *out_scale = Rr.NoiseFactor;
    put(Rr, w);
    auto many = ev.LinearTransformMany(A, row_size, b_step, {d, dn}, stride, offset);
    put(ev.Rescale(many.at(0)), w);
    put(ev.Rescale(many.at(1)), w);
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

// The reference's raw formats: a context from RawParams (Parameters::adaptTo), a plaintext of the
// n slots z encoded at the top level, exported with StorePlaintext as EVALUATION (eval_out),
// COEFFICIENT (coeff_out) and natural-order EVALUATION (nat_out), each [L][N]; the COEFFICIENT and
// natural-order exports are loaded back with LoadPlaintext and must equal the plaintext.
int facade_raw_plaintext(int logN, int n_q, int K, int dnum, const uint64_t* primes, const uint64_t* psi,
                         double top_scale, const double* z, int n, uint64_t* eval_out, uint64_t* coeff_out,
                         uint64_t* nat_out, char* err, int err_len) {
  try {
    RawParams raw;
    raw.logN = logN;
    raw.N = 1 << logN;
    raw.L = n_q;
    raw.K = K;
    raw.dnum = dnum;
    raw.moduli.assign(primes, primes + n_q);
    raw.SPECIALmoduli.assign(primes + n_q, primes + n_q + K);
    raw.root_of_unity.assign(psi, psi + n_q);
    raw.SPECIALroot_of_unity.assign(psi + n_q, psi + n_q + K);
    Context cc(Parameters{}.adaptTo(raw));
    const int N = 1 << logN;
    CryptoContextImpl ev(cc, FLEXIBLEAUTO, top_scale);
    std::vector<std::complex<double>> v(n);
    for (int i = 0; i < n; ++i) v[i] = {z[2 * i], z[2 * i + 1]};
    Plaintext P = ev.MakeCKKSPackedPlaintext(v);
    const size_t words = (size_t)N * n_q;
    std::vector<uint64_t> dev(words);
    check_cuda(cudaMemcpy(dev.data(), P.data(), words * 8, cudaMemcpyDeviceToHost), "D2H");
    auto flat = [&](const RawPlainText& r, uint64_t* out) {
      for (const auto& limb : r.sub_0) out = std::copy(limb.begin(), limb.end(), out);
    };
    RawPlainText re, rc, rn;
    ev.StorePlaintext(P, re);
    ev.StorePlaintext(P, rc, COEFFICIENT);
    ev.StorePlaintext(P, rn, EVALUATION, true);
    flat(re, eval_out);
    flat(rc, coeff_out);
    flat(rn, nat_out);
    for (const RawPlainText* r : {&rc, &rn}) {
      Plaintext Q = ev.LoadPlaintext(*r, r == &rn);
      std::vector<uint64_t> back(words);
      check_cuda(cudaMemcpy(back.data(), Q.data(), words * 8, cudaMemcpyDeviceToHost), "D2H");
      if (back != dev || Q.level != P.level || Q.scale != P.scale) throw Error(FIDES_ERR_STATE, "plaintext round trip");
    }
    return 0;
  } catch (const std::exception& e) {
    if (err && err_len > 0) snprintf(err, err_len, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
