// CKKS bootstrapping in the library's C++ host layer: ModRaise -> CoeffsToSlots -> EvalMod ->
// SlotsToCoeffs over the internal batched operations, for callers of the C ABI
// (fides_boot_*, include/fides_b200.h).
//
// Follows the reference's CKKS::Bootstrap (src/CKKS/Bootstrap.cu:437-648): sparse-secret
// encapsulation (keySwitchSparse, :257-290), ModRaise (:708+), EvalCoeffsToSlots /
// EvalSlotsToCoeffs as baby-step / giant-step linear transforms over hoisted rotations
// (src/CKKS/CoeffsToSlots.cu:75-151, src/CKKS/LinearTransform.cu), and approxModReduction: a
// Chebyshev series of the scaled cosine then double-angle steps (src/CKKS/ApproxModEval.cu:45-167,
// :527 evalChebyshevSeries, :873 applyDoubleAngleIterations).  OpenFHE's coefficient tables are
// not available here, so every table is derived from the mathematics:
//   * the special FFT z = U0 w (U0[j][k] = zeta^(5^j k), n = N/2 slots) is a radix-2
//     decimation-in-time transform of the bit-reversed input, F = S_(n/2) ... S_1, where S_h
//     pairs entries p and p + h of each block of 2h with the twiddle exp(i pi 5^(p mod h) / 4h);
//     each S_h has the slot diagonals 0, +h, -h.  CoeffsToSlots applies n F^-1 (unnormalised
//     inverse stages 2 S_h^-1), SlotsToCoeffs applies F, each grouped into `level budget`
//     composed matrices evaluated by BSGS;
//   * EvalMod: after CoeffsToSlots the real slots hold t = m'/(K q0) with m' = m + q0 I; the
//     Chebyshev interpolant (degree 31 by default, at the Chebyshev points of the first kind) of
//     cos(2 pi K t / 2^r - pi / 2^(r+1)) followed by r double-angle steps c -> 2 c^2 - 1 gives
//     sin(2 pi m' / q0) = sin(2 pi m / q0);
//   * scales: level l has scale S_l with S_(l-1) = S_l^2 / q_(l-1) (FLEXIBLEAUTO's chain), so
//     products of two level-l operands land on the next level's scale; an operand moved down
//     several levels is multiplied by an integer constant that re-targets its scale first.
// The operation sequence, the order of every batched launch and every integer constant are the
// same as the Python driver's (fides_b200/bootstrap.py), so the two give the same residues on
// the same tables.  Intermediates are stream-ordered allocations on the bootstrap's stream, so
// a bootstrap can be captured in a CUDA graph like every other operation of the library.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <set>
#include <vector>

#include "../../include/fides_b200.h"
#include "capi_internal.hpp"
#include "encode.hpp"
#include "kernels.cuh"
#include "ntt.cuh"
#include "ops.hpp"

namespace fides {
namespace boot {

using cd = std::complex<double>;
using Diags = std::map<int, std::vector<cd>>;  // slot offset -> diagonal (n values)

// ---------------------------------------------------------------------- tables (host)
// out = roll(v, k): out[(i + k) mod n] = v[i]
std::vector<cd> roll(const std::vector<cd>& v, long k) {
  const long n = (long)v.size();
  std::vector<cd> out(n);
  k = ((k % n) + n) % n;
  for (long i = 0; i < n; ++i) out[(i + k) % n] = v[i];
  return out;
}

// Slot diagonals of S_h (forward) or S_h^-1 (inverse); unnorm doubles the inverse stage.
Diags stage(int n, int h, bool inverse, bool unnorm) {
  std::vector<cd> tw(h);
  const double M = 8.0 * h;
  uint64_t e = 1;
  for (int i = 0; i < h; ++i) {
    const double ang = M_PI * (double)e / (4.0 * h);
    tw[i] = cd(std::cos(ang), std::sin(ang));
    e = (e * 5) % (uint64_t)M;
  }
  std::vector<cd> d0(n, 0.0), dp(n, 0.0), dm(n, 0.0);
  for (int p = 0; p < n; ++p) {
    const int r = p % (2 * h);
    const bool lo = r < h;
    const cd t = tw[lo ? r : r - h];
    if (!inverse) {  // lo: a[p] + t a[p + h]; hi: a[p - h] - t a[p]
      if (lo) {
        d0[p] = 1.0;
        dp[p] = t;
      } else {
        d0[p] = -t;
        dm[p] = 1.0;
      }
    } else {  // lo: (a[p] + a[p + h]) / 2; hi: (a[p - h] - a[p]) / (2 t)
      if (lo) {
        d0[p] = 0.5;
        dp[p] = 0.5;
      } else {
        d0[p] = -0.5 / t;
        dm[p] = 0.5 / t;
      }
    }
  }
  Diags out;
  out[0] = d0;
  auto acc = [&](int k, const std::vector<cd>& v) {
    auto it = out.find(k);
    if (it == out.end())
      out[k] = v;
    else
      for (int i = 0; i < n; ++i) it->second[i] += v[i];
  };
  if (h < n) {
    acc(h % n, dp);
    acc(((-h) % n + n) % n, dm);
  }
  if (inverse && unnorm)
    for (auto& kv : out)
      for (auto& x : kv.second) x *= 2.0;
  return out;
}

// Diagonals of A B: (A B) v = sum_(r, s) (A_r * roll(B_s, -r)) * roll(v, -(r + s)).
Diags compose(const Diags& A, const Diags& B, int n) {
  Diags out;
  for (const auto& [r, Ar] : A)
    for (const auto& [s, Bs] : B) {
      const int k = (r + s) % n;
      const std::vector<cd> rb = roll(Bs, -r);
      auto it = out.find(k);
      if (it == out.end()) {
        std::vector<cd> v(n);
        for (int i = 0; i < n; ++i) v[i] = Ar[i] * rb[i];
        out[k] = std::move(v);
      } else {
        for (int i = 0; i < n; ++i) it->second[i] += Ar[i] * rb[i];
      }
    }
  for (auto it = out.begin(); it != out.end();) {
    double mx = 0;
    for (const auto& x : it->second) mx = std::max(mx, std::abs(x));
    it = mx > 0 ? std::next(it) : out.erase(it);
  }
  return out;
}

// F (or F^-1, unnormalised: n F^-1) as `levels` composed matrices in application order; the
// log2(n) stages are split into `levels` consecutive groups, the first (log2 n mod levels)
// groups one stage longer.
std::vector<Diags> fft_levels(int n, int levels, bool inverse, bool unnorm) {
  std::vector<int> hs;
  for (int h = 1; h < n; h <<= 1) hs.push_back(h);
  if (inverse) std::reverse(hs.begin(), hs.end());
  const int S = (int)hs.size(), base = S / levels, extra = S % levels;
  std::vector<Diags> mats;
  int at = 0;
  for (int g = 0; g < levels; ++g) {
    const int cnt = base + (g < extra ? 1 : 0);
    Diags M;
    bool first = true;
    for (int i = at; i < at + cnt; ++i) {
      Diags St = stage(n, hs[i], inverse, unnorm);
      M = first ? St : compose(St, M, n);
      first = false;
    }
    at += cnt;
    mats.push_back(std::move(M));
  }
  return mats;
}

// Chebyshev interpolant of degree d of f on [-1, 1] (values at the d + 1 Chebyshev points of
// the first kind): c_k = (2 / (d + 1)) sum_j f(x_j) T_k(x_j), c_0 halved.
template <typename Fn>
std::vector<double> cheb_interpolate(Fn f, int d) {
  const int m = d + 1;
  std::vector<double> fx(m), c(m, 0.0);
  for (int j = 0; j < m; ++j) fx[j] = f(std::cos(M_PI * (j + 0.5) / m));
  for (int k = 0; k < m; ++k) {
    double s = 0;
    for (int j = 0; j < m; ++j) s += fx[j] * std::cos(M_PI * k * (j + 0.5) / m);
    c[k] = 2.0 * s / m;
  }
  c[0] *= 0.5;
  return c;
}

long floordiv(long a, long b) {
  long q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return q;
}
long pymod(long a, long b) { return ((a % b) + b) % b; }

// Round half to even, as Python's round() on a float.  The result is an integer held exactly
// in a double: constants such as round(c_0 S_t q_t) reach ~2^100, so they are reduced modulo
// each prime from the double itself (residue_of), never through a 64-bit integer.
double rint_even(double v) { return std::nearbyint(v); }

// w mod q for an integer-valued double w (any magnitude), as a residue in [0, q).
uint64_t residue_of(double w, uint64_t q) {
  const bool neg = w < 0;
  const double a = std::fabs(w);
  uint64_t r;
  if (a < 9223372036854775808.0) {  // 2^63: exact in an unsigned 64-bit integer
    r = (uint64_t)a % q;
  } else {  // a = m 2^k with m < 2^53 an integer and k >= 11
    int e = 0;
    const double fr = std::frexp(a, &e);  // a = fr 2^e, 0.5 <= fr < 1
    const uint64_t m = (uint64_t)std::ldexp(fr, 53);
    r = h_mulmod(m % q, h_powmod(2, (uint64_t)(e - 53), q), q);
  }
  return neg && r ? q - r : r;
}

// ---------------------------------------------------------------------- device values
// A device polynomial buffer shared by the views (ciphertexts) that use it; freed on its stream
// when the last view goes away.
using Buf = std::shared_ptr<Scratch>;

struct Ct {
  Buf b0, b1;
  const uint64_t* c0 = nullptr;
  const uint64_t* c1 = nullptr;
  int level = 0;
  double scale = 0;
};

struct Plan {  // one BSGS matrix prepared at `level`
  int step = 0, level = 0;
  double pt_scale = 0;
  std::map<int, std::vector<int>> giant;  // i -> baby indices j (ascending)
  std::map<std::pair<int, int>, Buf> pts;  // (i, j) -> encoded diagonal (level limbs)
};

}  // namespace boot

struct Bootstrapper {
  Context* c;
  fides_boot_params prm;
  int n = 0;  // slots
  std::vector<double> S;  // canonical scale of each level
  std::vector<double> cheb;
  std::vector<boot::Diags> cts, stc;
  std::vector<int> rotations;
  const uint64_t *relin = nullptr, *conj = nullptr, *to_sparse = nullptr, *to_dense = nullptr;
  std::map<int, const uint64_t*> rot;
  // prepared state
  bool prepared = false;
  std::vector<boot::Plan> cts_pl, stc_pl;
  boot::Buf pt_i, pt_minus_i;
  int top = 0, cts_out_level = 0, stc_in_level = 0, out_level = 0;
  double in_scale = 0, msg_scale = 0;
  double corr = 0;  // correction_bits > 0: round(q_1 / 2^correction_bits)
  cudaStream_t own = nullptr;  // the prepared tables are allocated and freed on this stream

  ~Bootstrapper() {
    cts_pl.clear();
    stc_pl.clear();
    pt_i.reset();
    pt_minus_i.reset();
    if (own) {
      cudaStreamSynchronize(own);
      cudaStreamDestroy(own);
    }
  }

  // ---- BSGS plan of one composed matrix (the Python driver's _plan)
  void plan(const boot::Diags& M, int& step, std::map<int, std::vector<int>>& giant) const {
    const int g = prm.baby;
    long st = n;
    bool any = false;
    for (const auto& kv : M)
      if (kv.first) {
        st = any ? std::gcd(st, (long)kv.first) : std::gcd((long)kv.first, (long)n);
        any = true;
      }
    if (any) st = std::gcd(st, (long)n);
    step = (int)st;
    std::set<long> ts;
    for (const auto& kv : M) ts.insert(boot::floordiv(boot::pymod(kv.first + n / 2, n) - n / 2, step));
    giant.clear();
    for (long t : ts) {
      const long i = boot::floordiv(t, g), j = t - i * g;
      giant[(int)i].push_back((int)j);
    }
  }

  std::set<int> bsgs_rotations(const boot::Diags& M) const {
    int step;
    std::map<int, std::vector<int>> giant;
    plan(M, step, giant);
    std::set<int> rs;
    for (const auto& [i, js] : giant) {
      for (int j : js) rs.insert((int)boot::pymod((long)step * j, n));
      rs.insert((int)boot::pymod((long)step * prm.baby * i, n));
    }
    return rs;
  }

  void build_tables() {
    n = c->N / 2;
    const double K = prm.K, r = prm.r;
    cheb = boot::cheb_interpolate(
        [&](double t) { return std::cos(2 * M_PI * K * t / std::pow(2.0, r) - M_PI / std::pow(2.0, r + 1)); },
        prm.degree);
    cts = boot::fft_levels(n, prm.level_budget_cts, true, true);
    stc = boot::fft_levels(n, prm.level_budget_stc, false, false);
    std::set<int> rs;
    for (const auto* v : {&cts, &stc})
      for (const auto& M : *v)
        for (int x : bsgs_rotations(M)) rs.insert(x);
    rs.erase(0);
    rotations.assign(rs.begin(), rs.end());
    const int L = c->n_q;
    S.assign(L + 1, 0.0);
    S[L] = prm.top_scale;
    for (int l = L; l > 1; --l) S[l - 1] = S[l] * S[l] / (double)c->primes[l - 1];
  }

  // ---------------------------------------------------------------- device helpers
  boot::Buf alloc(int limbs, cudaStream_t s) const {
    return std::make_shared<Scratch>(c, sizeof(uint64_t) * (size_t)c->N * limbs, s);
  }
  boot::Ct fresh(int level, double scale, cudaStream_t s) const {
    boot::Ct a;
    a.b0 = alloc(level, s);
    a.b1 = alloc(level, s);
    a.c0 = a.b0->u64();
    a.c1 = a.b1->u64();
    a.level = level;
    a.scale = scale;
    return a;
  }
  // an extended-basis ciphertext: `level` Q limbs followed by the K special limbs (level stays
  // the Q level)
  boot::Ct fresh_ext(int level, double scale, cudaStream_t s) const {
    boot::Ct a;
    a.b0 = alloc(level + c->K, s);
    a.b1 = alloc(level + c->K, s);
    a.c0 = a.b0->u64();
    a.c1 = a.b1->u64();
    a.level = level;
    a.scale = scale;
    return a;
  }
  static uint64_t* mut(const uint64_t* p) { return const_cast<uint64_t*>(p); }
  uint64_t residue(double v, int i) const { return boot::residue_of(v, c->primes[i]); }

  boot::Ct drop(const boot::Ct& a, int level) const {
    boot::Ct b = a;
    b.level = level;
    return b;
  }

  // polynomial-wise add / sub / mul over `level` limbs (one launch per call, as the Python
  // driver's add_poly / sub_poly / mul_poly)
  void ew(int op, const uint64_t* a, const uint64_t* b, int level, uint64_t* out, cudaStream_t s) const {
    AddSubJob j{a, b, out, level, op};
    launch_addsub(c, &j, 1, s);
  }

  // polynomial-wise op of every ciphertext of a batch with its partner (bs) or with one
  // plaintext (pt), both polynomials of all of them in one launch
  std::vector<boot::Ct> ew_many(int op, const std::vector<boot::Ct>& as, const std::vector<boot::Ct>* bs,
                                const uint64_t* pt, cudaStream_t s) const {
    std::vector<boot::Ct> outs;
    std::vector<AddSubJob> jobs;
    for (size_t i = 0; i < as.size(); ++i) {
      const boot::Ct& a = as[i];
      outs.push_back(fresh(a.level, a.scale, s));
      const uint64_t* b0 = bs ? (*bs)[i].c0 : pt;
      const uint64_t* b1 = bs ? (*bs)[i].c1 : pt;
      jobs.push_back(AddSubJob{a.c0, b0, mut(outs.back().c0), a.level, op});
      jobs.push_back(AddSubJob{a.c1, b1, mut(outs.back().c1), a.level, op});
    }
    launch_addsub(c, jobs.data(), (int)jobs.size(), s);
    return outs;
  }
  std::vector<boot::Ct> add_raw_many(const std::vector<boot::Ct>& as, const std::vector<boot::Ct>& bs,
                                     cudaStream_t s) const {
    return ew_many(EW_ADD, as, &bs, nullptr, s);
  }
  std::vector<boot::Ct> sub_raw_many(const std::vector<boot::Ct>& as, const std::vector<boot::Ct>& bs,
                                     cudaStream_t s) const {
    return ew_many(EW_SUB, as, &bs, nullptr, s);
  }
  std::vector<boot::Ct> mul_plain_int_many(const std::vector<boot::Ct>& as, const boot::Buf& pt,
                                           cudaStream_t s) const {
    return ew_many(EW_MUL, as, nullptr, pt->u64(), s);
  }
  std::vector<boot::Ct> mul_int_many(const std::vector<boot::Ct>& as, double v, cudaStream_t s) const {
    std::vector<boot::Ct> outs;
    std::vector<ScalarJob> jobs;
    for (const auto& a : as) {
      if (a.level > MAX_SCALAR_LIMBS) throw Error(-1, "bootstrap: scalar product over more than 64 limbs");
      outs.push_back(fresh(a.level, a.scale, s));
      for (int k = 0; k < 2; ++k) {
        ScalarJob j{};
        j.a = k ? a.c1 : a.c0;
        j.out = mut(k ? outs.back().c1 : outs.back().c0);
        j.l = a.level;
        j.op = EW_MUL_SCALAR;
        for (int i = 0; i < a.level; ++i) j.s[i] = residue(v, i);
        jobs.push_back(j);
      }
    }
    launch_scalar(c, jobs.data(), (int)jobs.size(), s);
    return outs;
  }

  // the same integer combination of every lane (one launch): sum_t ints[t] lane[t] (+ add on c0)
  // ints / add: integers held exactly in doubles (see rint_even)
  // ext > 0: the operands are extended-basis polynomials (level Q limbs + ext special limbs)
  std::vector<boot::Ct> lincomb_lanes(const std::vector<std::vector<boot::Ct>>& lanes, const std::vector<double>& ints,
                                      const double* add, int level, double scale, cudaStream_t s, int ext = 0) const {
    if (lanes.empty() || ints.empty() || ints.size() > (size_t)MAX_LC_TERMS)
      throw Error(-1, "bootstrap: linear combination out of range");
    static thread_local LinCombJob j;
    const int limbs = level + ext;
    j.lq = ext ? level : 0;
    j.nq = c->n_q;
    for (size_t t = 0; t < ints.size(); ++t)
      for (int i = 0; i < limbs; ++i) j.s[t][i] = residue(ints[t], ext_prime(i, j.lq, j.nq));
    for (int i = 0; i < limbs; ++i) j.add0[i] = add ? residue(*add, ext_prime(i, j.lq, j.nq)) : 0;
    j.n = (int)ints.size();
    j.l = limbs;
    std::vector<boot::Ct> outs;
    for (size_t a0 = 0; a0 < lanes.size(); a0 += MAX_LC_LANES) {  // lanes in launches of up to 8
      const size_t m = std::min<size_t>(MAX_LC_LANES, lanes.size() - a0);
      for (size_t a = 0; a < m; ++a) {
        outs.push_back(ext ? fresh_ext(level, scale, s) : fresh(level, scale, s));
        j.out0[a] = mut(outs.back().c0);
        j.out1[a] = mut(outs.back().c1);
        for (size_t t = 0; t < ints.size(); ++t) {
          j.x0[a][t] = lanes[a0 + a][t].c0;
          j.x1[a][t] = lanes[a0 + a][t].c1;
        }
      }
      j.lanes = (int)m;
      launch_lincomb(c, j, s);
    }
    return outs;
  }

  std::vector<boot::Ct> lincomb_many(const std::vector<std::vector<boot::Ct>>& lanes, const std::vector<double>& ints,
                                     double cst, cudaStream_t s) const {
    const boot::Ct& a = lanes[0][0];
    int l = a.level;
    for (const auto& ln : lanes)
      for (const auto& b : ln) l = std::min(l, b.level);
    double add = 0;
    const bool has = cst != 0.0;
    if (has) add = boot::rint_even(cst * a.scale);
    return lincomb_lanes(lanes, ints, has ? &add : nullptr, l, a.scale, s);
  }

  std::vector<boot::Ct> add_many(const std::vector<boot::Ct>& xs, const std::vector<boot::Ct>& ys,
                                 cudaStream_t s) const {
    std::vector<std::vector<boot::Ct>> lanes;
    for (size_t i = 0; i < xs.size(); ++i) lanes.push_back({xs[i], ys[i]});
    return lincomb_many(lanes, {1, 1}, 0.0, s);
  }

  std::vector<boot::Ct> rescale_many_to(const std::vector<boot::Ct>& cts_, double new_scale, cudaStream_t s) const {
    std::vector<const uint64_t*> xs;
    std::vector<int> ls;
    std::vector<uint64_t*> outs;
    std::vector<boot::Ct> res;
    for (const auto& a : cts_) {
      res.push_back(fresh(a.level - 1, new_scale, s));
      xs.push_back(a.c0);
      xs.push_back(a.c1);
      ls.push_back(a.level);
      ls.push_back(a.level);
      outs.push_back(mut(res.back().c0));
      outs.push_back(mut(res.back().c1));
    }
    op_rescale_batch(c, xs.data(), ls.data(), outs.data(), (int)xs.size(), s);
    return res;
  }

  std::vector<boot::Ct> to_level_many(const std::vector<boot::Ct>& cts_, int level, cudaStream_t s) const {
    const boot::Ct& a = cts_[0];
    if (a.level == level && std::abs(a.scale / S[level] - 1) < 1e-15) return cts_;
    if (a.level <= level) throw Error(-4, "bootstrap: cannot raise a level");
    const double k = boot::rint_even(S[level] * (double)c->primes[level] / a.scale);
    std::vector<std::vector<boot::Ct>> lanes;
    for (const auto& b : cts_) lanes.push_back({drop(b, level + 1)});
    return rescale_many_to(lincomb_many(lanes, {k}, 0.0, s), S[level], s);
  }

  std::vector<boot::Ct> lincomb_to_many(const std::vector<std::vector<boot::Ct>>& lanes, const std::vector<double>& coefs,
                                        double cst, int target, cudaStream_t s) const {
    const double qt = (double)c->primes[target], St = S[target];
    std::vector<int> keep;
    std::vector<double> ints;
    for (size_t t = 0; t < coefs.size(); ++t) {
      const boot::Ct& a = lanes[0][t];
      if (a.level <= target) throw Error(-4, "bootstrap: operand below the combination's level");
      const double k = boot::rint_even(coefs[t] * St * qt / a.scale);
      if (k != 0) {
        keep.push_back((int)t);
        ints.push_back(k);
      }
    }
    if (keep.empty()) {
      keep = {0};
      ints = {0};
    }
    const double add = boot::rint_even(cst * St * qt);
    std::vector<std::vector<boot::Ct>> sel;
    for (const auto& ln : lanes) {
      std::vector<boot::Ct> v;
      for (int t : keep) v.push_back(ln[t]);
      sel.push_back(v);
    }
    auto outs = lincomb_lanes(sel, ints, add != 0 ? &add : nullptr, target + 1, 0.0, s);
    return rescale_many_to(outs, St, s);
  }

  // to_level of every operand, batched: operands sharing (level, scale, target) are brought
  // down together (lanes of a batch run the same computation, so they share all three)
  std::vector<boot::Ct> to_levels(const std::vector<boot::Ct>& xs, const std::vector<int>& targets,
                                  cudaStream_t s) const {
    std::vector<boot::Ct> out(xs.size());
    std::vector<bool> done(xs.size(), false);
    for (size_t i = 0; i < xs.size(); ++i) {
      if (done[i]) continue;
      std::vector<size_t> grp;
      for (size_t k = i; k < xs.size(); ++k)
        if (!done[k] && xs[k].level == xs[i].level && xs[k].scale == xs[i].scale && targets[k] == targets[i])
          grp.push_back(k);
      std::vector<boot::Ct> in;
      for (size_t k : grp) in.push_back(xs[k]);
      const std::vector<boot::Ct> r = to_level_many(in, targets[i], s);
      for (size_t m = 0; m < grp.size(); ++m) {
        out[grp[m]] = r[m];
        done[grp[m]] = true;
      }
    }
    return out;
  }

  std::vector<boot::Ct> mul_many(const std::vector<std::pair<boot::Ct, boot::Ct>>& pairs, cudaStream_t s) const {
    std::vector<boot::Ct> as, bs;
    std::vector<int> ls;
    for (const auto& [a, b] : pairs) {
      as.push_back(a);
      bs.push_back(b);
      ls.push_back(std::min(a.level, b.level));
    }
    as = to_levels(as, ls, s);
    bs = to_levels(bs, ls, s);
    std::vector<std::pair<boot::Ct, boot::Ct>> ab;
    for (size_t i = 0; i < pairs.size(); ++i) ab.push_back({as[i], bs[i]});
    std::vector<HMultItem> items;
    std::vector<boot::Ct> outs;
    for (const auto& [a, b] : ab) {
      outs.push_back(fresh(a.level - 1, S[a.level - 1], s));
      items.push_back(HMultItem{a.c0, a.c1, b.c0, b.c1, mut(outs.back().c0), mut(outs.back().c1), a.level});
    }
    op_hmult_batch(c, items.data(), (int)items.size(), relin, true, s);
    return outs;
  }

  std::vector<boot::Ct> conjugate_many(const std::vector<boot::Ct>& as, cudaStream_t s) const {
    std::vector<RotateItem> items;
    std::vector<boot::Ct> outs;
    for (const auto& a : as) {
      outs.push_back(fresh(a.level, a.scale, s));
      items.push_back(RotateItem{a.c0, a.c1, mut(outs.back().c0), mut(outs.back().c1), conj, a.level,
                                 (uint32_t)(2 * c->N - 1)});
    }
    op_rotate_batch(c, items.data(), (int)items.size(), s);
    return outs;
  }

  const uint64_t* rot_key(int r) const {
    auto it = rot.find((int)boot::pymod(r, n));
    if (it == rot.end()) throw Error(-5, "bootstrap: missing rotation key " + std::to_string(r));
    return it->second;
  }

  // hoisted rotations of every ciphertext of a batch by the same list rs (one ModUp each, the
  // key-switch inner products of all of them grouped by key): res[b][k] = rotate(as[b], rs[k])
  std::vector<std::vector<boot::Ct>> rotate_many(const std::vector<boot::Ct>& as, const std::vector<int>& rs,
                                                 cudaStream_t s) const {
    std::vector<HoistItem> items(as.size());
    std::vector<std::vector<boot::Ct>> res(as.size(), std::vector<boot::Ct>(rs.size()));
    for (size_t b = 0; b < as.size(); ++b) {
      const boot::Ct& a = as[b];
      HoistItem& it = items[b];
      it.c0 = a.c0;
      it.c1 = a.c1;
      it.l = a.level;
      for (size_t k = 0; k < rs.size(); ++k) {
        if (boot::pymod(rs[k], n) == 0) {
          res[b][k] = a;
          continue;
        }
        res[b][k] = fresh(a.level, a.scale, s);
        it.keys.push_back(rot_key(rs[k]));
        it.ks.push_back(h_auto_index(c->logN, rs[k]));
        it.out0.push_back(mut(res[b][k].c0));
        it.out1.push_back(mut(res[b][k].c1));
      }
    }
    if (!items.empty() && !items[0].keys.empty()) op_hoisted_batch(c, items.data(), (int)items.size(), s);
    return res;
  }

  std::vector<boot::Ct> rotate_batch(const std::vector<std::pair<boot::Ct, int>>& jobs, cudaStream_t s) const {
    std::vector<RotateItem> items;
    std::vector<boot::Ct> outs;
    for (const auto& [a, r] : jobs) {
      outs.push_back(fresh(a.level, a.scale, s));
      items.push_back(RotateItem{a.c0, a.c1, mut(outs.back().c0), mut(outs.back().c1), rot_key(r), a.level,
                                 h_auto_index(c->logN, r)});
    }
    if (!items.empty()) op_rotate_batch(c, items.data(), (int)items.size(), s);
    return outs;
  }

  // (c0, c1) -> (c0 + ks(c1)_0, ks(c1)_1) for every ciphertext of a batch, one key (the c0
  // addition is the ModDown epilogue's addend)
  std::vector<boot::Ct> keyswitch_add_many(const std::vector<boot::Ct>& as, const uint64_t* key,
                                           cudaStream_t s) const {
    std::vector<boot::Ct> outs;
    std::vector<KeySwitchItem> items;
    for (const auto& a : as) {
      outs.push_back(fresh(a.level, a.scale, s));
      items.push_back(KeySwitchItem{a.c1, a.level, key, mut(outs.back().c0), mut(outs.back().c1), a.c0, nullptr});
    }
    op_keyswitch_batch(c, items.data(), (int)items.size(), s);
    return outs;
  }

  // ---------------------------------------------------------------- preparation
  boot::Buf encode_pt(const std::vector<boot::cd>& z, int level, double scale, cudaStream_t s, int special = 0) const {
    Scratch slots(c, sizeof(double) * 2 * z.size(), s);
    FIDES_CUDA(cudaMemcpyAsync(slots.p, z.data(), sizeof(double) * 2 * z.size(), cudaMemcpyHostToDevice, s));
    boot::Buf out = alloc(level + special, s);
    op_encode_ext(c, static_cast<const double*>(slots.p), (int)z.size(), 1, scale, level, special, out->u64(), s);
    return out;
  }

  boot::Buf int_pt(const std::vector<double>& coeff, int level, cudaStream_t s) const {
    const size_t N = c->N;
    std::vector<uint64_t> h((size_t)level * N);
    for (int i = 0; i < level; ++i)
      for (size_t k = 0; k < N; ++k) h[i * N + k] = residue(coeff[k], i);
    boot::Buf out = alloc(level, s);
    FIDES_CUDA(cudaMemcpyAsync(out->u64(), h.data(), sizeof(uint64_t) * h.size(), cudaMemcpyHostToDevice, s));
    std::vector<int> ids(level);
    std::iota(ids.begin(), ids.end(), 0);
    ntt_polys(c, out->u64(), 1, level, ids.data(), false, s);
    return out;
  }

  boot::Plan prepare_matrix(const boot::Diags& M, double fac, int level, double scale, cudaStream_t s) const {
    boot::Plan P;
    plan(M, P.step, P.giant);
    P.level = level;
    const double target = S[level - 1];
    P.pt_scale = target * (double)c->primes[level - 1] / scale;
    for (const auto& [i, js] : P.giant)
      for (int j : js) {
        const int off = (int)boot::pymod((long)P.step * (prm.baby * (long)i + j), n);
        auto it = M.find(off);
        if (it == M.end()) continue;
        std::vector<boot::cd> d(it->second.size());
        for (size_t k = 0; k < d.size(); ++k) d[k] = it->second[k] * fac;
        P.pts[{i, j}] = encode_pt(boot::roll(d, (long)P.step * prm.baby * i), level, P.pt_scale, s,
                                  prm.double_hoist ? c->K : 0);
      }
    return P;
  }

  // Prepares on the bootstrapper's own stream (after the work already on `user`), so that the
  // tables outlive any stream of the caller; returns when they are ready.
  void prepare(cudaStream_t user) {
    if (!own) FIDES_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    cudaEvent_t ev;
    FIDES_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, user);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(own, ev, 0);
    cudaEventDestroy(ev);
    FIDES_CUDA(e);
    cts_pl.clear();
    stc_pl.clear();
    prepared = false;
    cudaStream_t s = own;
    const int top_level = prm.top_level;
    top = top_level;
    in_scale = S[top_level];
    msg_scale = prm.msg_scale * (double)(1ll << prm.prescale_bits);
    if (prm.correction_bits > 0) {  // the input is scaled by round(q_1 / 2^k) / q_1 first
      corr = boot::rint_even((double)c->primes[1] / std::ldexp(1.0, prm.correction_bits));
      msg_scale = msg_scale * corr / (double)c->primes[1];
    }
    // 2 K q0 is formed exactly and rounded once to a double (as an integer product would be)
    const double two_k_q0 = (double)((unsigned __int128)2 * (unsigned)prm.K * c->primes[0]);
    const double gfac = std::pow(in_scale / two_k_q0 / n, 1.0 / (double)cts.size());
    cts_pl.clear();
    stc_pl.clear();
    int level = top_level;
    double scale = in_scale;
    for (const auto& M : cts) {
      cts_pl.push_back(prepare_matrix(M, gfac, level, scale, s));
      level -= 1;
      scale = S[level];
    }
    cts_out_level = level;
    if (prm.double_hoist)  // the double-hoisted transform sums its giant steps in one combination
      for (const auto& P : cts_pl)
        if (P.giant.size() > (size_t)MAX_BSGS_GIANT || P.giant.size() > (size_t)MAX_LC_TERMS)
          throw Error(FIDES_ERR_ARG, "double hoisting supports at most 16 giant steps per transform");
    const int depth = (int)std::ceil(std::log2((double)prm.degree)) + 1 + prm.r;
    stc_in_level = cts_out_level - depth;
    if (stc_in_level - (int)stc.size() < 1) throw Error(-4, "bootstrap: not enough levels for the chosen budget");
    const double sfac = std::pow((double)c->primes[0] / (2.0 * M_PI * msg_scale), 1.0 / (double)stc.size());
    level = stc_in_level;
    for (const auto& M : stc) {
      stc_pl.push_back(prepare_matrix(M, sfac, level, S[level], s));
      level -= 1;
    }
    out_level = level;
    if (prm.double_hoist)
      for (const auto& P : stc_pl)
        if (P.giant.size() > (size_t)MAX_BSGS_GIANT || P.giant.size() > (size_t)MAX_LC_TERMS)
          throw Error(FIDES_ERR_ARG, "double hoisting supports at most 16 giant steps per transform");
    std::vector<double> mono(c->N, 0.0);
    mono[c->N / 2] = 1;  // X^(N/2): slots times i
    pt_i = int_pt(mono, top_level, s);
    mono[c->N / 2] = -1;
    pt_minus_i = int_pt(mono, top_level, s);
    FIDES_CUDA(cudaStreamSynchronize(s));
    uint32_t st = 0;
    FIDES_CUDA(cudaMemcpy(&st, c->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (st & 2u) throw Error(-1, "bootstrap: an encoded diagonal coefficient exceeded 2^62");
    prepared = true;
  }

  // ---------------------------------------------------------------- the linear transforms
  // One BSGS linear transform applied to every ciphertext of a batch: the baby-step rotations
  // of all of them in one hoisted batch, each giant step's plaintext inner products in one
  // launch (the diagonals shared by the lanes), all giant-step rotations in one batched key
  // switch, the sums and the rescale batched.
  std::vector<boot::Ct> apply_many(const std::vector<boot::Ct>& as, const boot::Plan& P, cudaStream_t s) const {
    const size_t B = as.size();
    for (const auto& a : as)
      if (a.level != P.level) throw Error(-4, "bootstrap: linear transform at the wrong level");
    const int g = prm.baby, level = as[0].level;
    const double scale = as[0].scale;
    std::set<int> jset;
    for (const auto& kv : P.giant)
      for (int j : kv.second) jset.insert(j);
    std::vector<int> js(jset.begin(), jset.end()), rs;
    for (int j : js) rs.push_back((int)boot::pymod((long)P.step * j, n));
    const std::vector<std::vector<boot::Ct>> bv = rotate_many(as, rs, s);  // [b][index in js]
    std::map<int, size_t> jpos;
    for (size_t k = 0; k < js.size(); ++k) jpos[js[k]] = k;
    // the giant steps that have terms, with their (baby index, diagonal) pairs
    std::vector<std::pair<int, std::vector<std::pair<int, boot::Buf>>>> gs;
    for (const auto& [i, jl] : P.giant) {
      std::vector<std::pair<int, boot::Buf>> terms;
      for (int j : jl) {
        auto it = P.pts.find({i, j});
        if (it != P.pts.end()) terms.push_back({j, it->second});
      }
      if (!terms.empty()) gs.push_back({i, terms});
    }
    std::vector<std::vector<boot::Ct>> inner(gs.size(), std::vector<boot::Ct>(B));  // [giant step][b]
    if (js.size() <= (size_t)MAX_BSGS_BABY && gs.size() <= (size_t)MAX_BSGS_GIANT) {
      // every giant step's inner product in one launch per 8 ciphertexts
      for (size_t b0 = 0; b0 < B; b0 += MAX_BSGS_LANES) {
        const size_t nl = std::min<size_t>(MAX_BSGS_LANES, B - b0);
        BsgsJob bj{};
        bj.nb = (int)js.size();
        bj.ng = (int)gs.size();
        bj.l = level;
        bj.lanes = (int)nl;
        for (size_t gi = 0; gi < gs.size(); ++gi)
          for (const auto& [j, pt] : gs[gi].second) bj.pt[gi][jpos.at(j)] = pt->u64();
        for (size_t ln = 0; ln < nl; ++ln) {
          const size_t b = b0 + ln;
          for (size_t k = 0; k < js.size(); ++k) {
            bj.x0[ln][k] = bv[b][k].c0;
            bj.x1[ln][k] = bv[b][k].c1;
          }
          for (size_t gi = 0; gi < gs.size(); ++gi) {
            inner[gi][b] = fresh(level, scale, s);
            bj.out0[ln][gi] = mut(inner[gi][b].c0);
            bj.out1[ln][gi] = mut(inner[gi][b].c1);
          }
        }
        launch_bsgs_dot(c, bj, s);
      }
    } else {
      for (size_t gi = 0; gi < gs.size(); ++gi) {
        const auto& terms = gs[gi].second;
        bool have = false;
        for (size_t k = 0; k < terms.size(); k += MAX_DOT_TERMS) {
          const size_t m = std::min<size_t>(MAX_DOT_TERMS, terms.size() - k);
          std::vector<boot::Ct> d(B);
          for (size_t b0 = 0; b0 < B; b0 += MAX_DOT_LANES) {
            const size_t nl = std::min<size_t>(MAX_DOT_LANES, B - b0);
            DotJob dj{};
            for (size_t t = 0; t < m; ++t) dj.pt[t] = terms[k + t].second->u64();
            for (size_t ln = 0; ln < nl; ++ln) {
              const size_t b = b0 + ln;
              d[b] = fresh(level, scale, s);
              for (size_t t = 0; t < m; ++t) {
                const boot::Ct& x = bv[b][jpos.at(terms[k + t].first)];
                dj.c0[ln][t] = x.c0;
                dj.c1[ln][t] = x.c1;
              }
              dj.out0[ln] = mut(d[b].c0);
              dj.out1[ln] = mut(d[b].c1);
            }
            dj.n = (int)m;
            dj.l = level;
            dj.lanes = (int)nl;
            launch_dot_plain(c, dj, s);
          }
          inner[gi] = have ? add_many(inner[gi], d, s) : d;
          have = true;
        }
      }
    }
    std::vector<std::vector<boot::Ct>> parts(B);
    std::vector<std::pair<boot::Ct, int>> turns;
    std::vector<size_t> owner;
    for (size_t gi = 0; gi < gs.size(); ++gi) {
      const int r = (int)boot::pymod((long)P.step * g * gs[gi].first, n);
      for (size_t b = 0; b < B; ++b) {
        if (r) {
          turns.push_back({inner[gi][b], r});
          owner.push_back(b);
        } else {
          parts[b].push_back(inner[gi][b]);
        }
      }
    }
    const std::vector<boot::Ct> turned = rotate_batch(turns, s);
    for (size_t k = 0; k < turned.size(); ++k) parts[owner[k]].push_back(turned[k]);
    while (parts[0].size() > 1) {  // every ciphertext has the same number of parts
      std::vector<std::vector<boot::Ct>> next(B);
      for (size_t k = 0; k < parts[0].size(); k += 16) {
        const size_t m = std::min<size_t>(16, parts[0].size() - k);
        if (m > 1) {
          std::vector<std::vector<boot::Ct>> lanes(B);
          for (size_t b = 0; b < B; ++b) lanes[b].assign(parts[b].begin() + k, parts[b].begin() + k + m);
          const auto sums = lincomb_many(lanes, std::vector<double>(m, 1.0), 0.0, s);
          for (size_t b = 0; b < B; ++b) next[b].push_back(sums[b]);
        } else {
          for (size_t b = 0; b < B; ++b) next[b].push_back(parts[b][k]);
        }
      }
      parts = next;
    }
    std::vector<boot::Ct> sums;
    for (size_t b = 0; b < B; ++b) sums.push_back(parts[b][0]);
    return rescale_many_to(sums, S[level - 1], s);
  }

  // P mod q_i for the Q limbs (the extended-basis form of an unrotated baby step is P a)
  std::vector<uint64_t> p_mod_q() const {
    std::vector<uint64_t> v(c->n_q);
    for (int i = 0; i < c->n_q; ++i) {
      const uint64_t q = c->primes[i];
      uint64_t x = 1 % q;
      for (int k = 0; k < c->K; ++k) x = h_mulmod(x, c->primes[c->n_q + k] % q, q);
      v[i] = x;
    }
    return v;
  }

  // The linear transform double-hoisted: the baby-step rotations of every ciphertext are left
  // in the extended basis (the KSK outputs with P c0 added and the automorphism applied, no
  // ModDown), each giant step's inner product is taken there against diagonals encoded with
  // the special limbs too, a rotated giant step's c1 alone is brought down (one ModDown) and
  // key-switched with its extended-basis c0 added to the output as it is, and the giant steps
  // are summed in the extended basis and brought down once, fused with the rescale.  Every
  // term carries the factor P, so the final ModDown divides it out; the rounding differs from
  // the single-hoisted form's by one ModDown rounding per giant step and transform (each term
  // below K / 2 per coefficient before the secret's multiplication).
  std::vector<boot::Ct> apply_many_dh(const std::vector<boot::Ct>& as, const boot::Plan& P, cudaStream_t s) const {
    const size_t B = as.size();
    for (const auto& a : as)
      if (a.level != P.level) throw Error(-4, "bootstrap: linear transform at the wrong level");
    const int g = prm.baby, l = as[0].level, K = c->K;
    const size_t N = c->N;
    const double scale = as[0].scale;
    std::set<int> jset;
    for (const auto& kv : P.giant)
      for (int j : kv.second) jset.insert(j);
    std::vector<int> js(jset.begin(), jset.end()), rs;
    for (int j : js) rs.push_back((int)boot::pymod((long)P.step * j, n));
    std::map<int, size_t> jpos;
    for (size_t k = 0; k < js.size(); ++k) jpos[js[k]] = k;
    // baby steps: X[b][k] = P rotate(a_b, rs[k]) in the extended basis
    std::vector<std::vector<boot::Ct>> X(B, std::vector<boot::Ct>(js.size()));
    std::vector<HoistItem> items(B);
    std::vector<ScalarJob> pj;
    const std::vector<uint64_t> pq = p_mod_q();
    for (size_t b = 0; b < B; ++b) {
      const boot::Ct& a = as[b];
      HoistItem& it = items[b];
      it.c0 = a.c0;
      it.c1 = a.c1;
      it.l = l;
      for (size_t k = 0; k < js.size(); ++k) {
        X[b][k] = fresh_ext(l, scale, s);
        if (boot::pymod(rs[k], n) == 0) {
          for (int poly = 0; poly < 2; ++poly) {
            ScalarJob j{};
            j.a = poly ? a.c1 : a.c0;
            j.out = mut(poly ? X[b][k].c1 : X[b][k].c0);
            j.l = l;
            j.op = EW_MUL_SCALAR;
            for (int i = 0; i < l; ++i) j.s[i] = pq[i];
            pj.push_back(j);
            FIDES_CUDA(cudaMemsetAsync(j.out + (size_t)l * N, 0, sizeof(uint64_t) * N * K, s));
          }
        } else {
          it.keys.push_back(rot_key(rs[k]));
          it.ks.push_back(h_auto_index(c->logN, rs[k]));
          it.out0.push_back(mut(X[b][k].c0));
          it.out1.push_back(mut(X[b][k].c1));
        }
      }
    }
    if (!pj.empty()) launch_scalar(c, pj.data(), (int)pj.size(), s);
    if (!items.empty() && !items[0].keys.empty()) op_hoisted_ext_batch(c, items.data(), (int)items.size(), s);
    // the giant steps that have terms
    std::vector<std::pair<int, std::vector<std::pair<int, boot::Buf>>>> gs;
    for (const auto& [i, jl] : P.giant) {
      std::vector<std::pair<int, boot::Buf>> terms;
      for (int j : jl) {
        auto it = P.pts.find({i, j});
        if (it != P.pts.end()) terms.push_back({j, it->second});
      }
      if (!terms.empty()) gs.push_back({i, terms});
    }
    if (js.size() > (size_t)MAX_BSGS_BABY || gs.size() > (size_t)MAX_BSGS_GIANT || gs.size() > (size_t)MAX_LC_TERMS)
      throw Error(-1, "bootstrap: double hoisting needs at most 16 baby and 16 giant steps");
    std::vector<std::vector<boot::Ct>> Y(gs.size(), std::vector<boot::Ct>(B));  // [giant step][b], extended
    for (size_t b0 = 0; b0 < B; b0 += MAX_BSGS_LANES) {
      const size_t nl = std::min<size_t>(MAX_BSGS_LANES, B - b0);
      BsgsJob bj{};
      bj.nb = (int)js.size();
      bj.ng = (int)gs.size();
      bj.l = l + K;
      bj.lq = l;
      bj.nq = c->n_q;
      bj.lanes = (int)nl;
      for (size_t gi = 0; gi < gs.size(); ++gi)
        for (const auto& [j, pt] : gs[gi].second) bj.pt[gi][jpos.at(j)] = pt->u64();
      for (size_t ln = 0; ln < nl; ++ln) {
        const size_t b = b0 + ln;
        for (size_t k = 0; k < js.size(); ++k) {
          bj.x0[ln][k] = X[b][k].c0;
          bj.x1[ln][k] = X[b][k].c1;
        }
        for (size_t gi = 0; gi < gs.size(); ++gi) {
          Y[gi][b] = fresh_ext(l, scale, s);
          bj.out0[ln][gi] = mut(Y[gi][b].c0);
          bj.out1[ln][gi] = mut(Y[gi][b].c1);
        }
      }
      launch_bsgs_dot(c, bj, s);
    }
    X.clear();
    // rotated giant steps: c1 down to the Q basis, then key-switched in the extended basis
    std::vector<uint64_t*> md_in, md_out;
    std::vector<int> md_l;
    std::vector<boot::Buf> c1q;
    std::vector<HoistItem> gitems;
    std::vector<std::vector<boot::Ct>> Z(gs.size(), std::vector<boot::Ct>(B));
    for (size_t gi = 0; gi < gs.size(); ++gi) {
      const int r = (int)boot::pymod((long)P.step * g * gs[gi].first, n);
      if (!r) continue;
      for (size_t b = 0; b < B; ++b) {
        c1q.push_back(alloc(l, s));
        md_in.push_back(mut(Y[gi][b].c1));
        md_out.push_back(c1q.back()->u64());
        md_l.push_back(l);
        Z[gi][b] = fresh_ext(l, scale, s);
        HoistItem it;
        it.c0 = nullptr;
        it.c1 = c1q.back()->u64();
        it.l = l;
        it.keys.push_back(rot_key(r));
        it.ks.push_back(h_auto_index(c->logN, r));
        it.out0.push_back(mut(Z[gi][b].c0));
        it.out1.push_back(mut(Z[gi][b].c1));
        it.c0x = Y[gi][b].c0;
        gitems.push_back(it);
      }
    }
    op_moddown_batch(c, md_in.data(), md_l.data(), md_out.data(), (int)md_in.size(), s);
    if (!gitems.empty()) op_hoisted_ext_batch(c, gitems.data(), (int)gitems.size(), s);
    // the sum of every ciphertext's giant steps, in the extended basis
    std::vector<std::vector<boot::Ct>> lanes(B);
    for (size_t gi = 0; gi < gs.size(); ++gi) {
      const bool rot = boot::pymod((long)P.step * g * gs[gi].first, n) != 0;
      for (size_t b = 0; b < B; ++b) lanes[b].push_back(rot ? Z[gi][b] : Y[gi][b]);
    }
    std::vector<boot::Ct> acc;
    if (lanes[0].size() == 1) {
      for (size_t b = 0; b < B; ++b) acc.push_back(lanes[b][0]);
    } else {
      acc = lincomb_lanes(lanes, std::vector<double>(lanes[0].size(), 1.0), nullptr, l, scale, s, K);
    }
    lanes.clear();
    Y.clear();
    Z.clear();
    // one ModDown per polynomial, fused with the rescale by q_(l-1)
    std::vector<boot::Ct> outs;
    std::vector<uint64_t*> ex, o;
    std::vector<int> ls2;
    for (size_t b = 0; b < B; ++b) {
      outs.push_back(fresh(l - 1, S[l - 1], s));
      ex.push_back(mut(acc[b].c0));
      ex.push_back(mut(acc[b].c1));
      o.push_back(mut(outs.back().c0));
      o.push_back(mut(outs.back().c1));
      ls2.push_back(l);
      ls2.push_back(l);
    }
    op_moddown_rescale_batch(c, ex.data(), ls2.data(), o.data(), (int)ex.size(), s);
    return outs;
  }

  // ---------------------------------------------------------------- EvalMod
  static constexpr int PS_BABY = 16;

  struct Powers {
    std::map<int, std::vector<boot::Ct>> T;
    std::map<std::pair<int, int>, std::vector<boot::Ct>> at;
  };

  const std::vector<boot::Ct>& t_at(Powers& P, int k, int level, cudaStream_t s) const {
    auto key = std::make_pair(k, level);
    auto it = P.at.find(key);
    if (it == P.at.end()) it = P.at.emplace(key, to_level_many(P.T.at(k), level, s)).first;
    return it->second;
  }

  // T_1 .. T_min(PS_BABY, degree) and the doublings T_32, T_64, ... up to `degree`
  Powers cheb_powers(const std::vector<boot::Ct>& ts, int degree, cudaStream_t s) const {
    Powers P;
    P.T[1] = ts;
    auto make = [&](int k) {
      std::vector<std::pair<boot::Ct, boot::Ct>> pr;
      if (k % 2 == 0) {
        for (const auto& a : P.T.at(k / 2)) pr.push_back({a, a});
        auto x = mul_many(pr, s);
        std::vector<std::vector<boot::Ct>> lanes;
        for (const auto& p : x) lanes.push_back({p});
        P.T[k] = lincomb_many(lanes, {2}, -1.0, s);
      } else {
        const auto &A = P.T.at(k / 2), &B = P.T.at(k / 2 + 1);
        for (size_t i = 0; i < A.size(); ++i) pr.push_back({A[i], B[i]});
        auto x = mul_many(pr, s);
        const auto& one = t_at(P, 1, x[0].level, s);
        std::vector<std::vector<boot::Ct>> lanes;
        for (size_t i = 0; i < x.size(); ++i) lanes.push_back({x[i], one[i]});
        P.T[k] = lincomb_many(lanes, {2, -1}, 0.0, s);
      }
    };
    for (int k = 2; k <= std::min(PS_BABY, degree); ++k) make(k);
    for (int m = 2 * PS_BABY; m <= degree; m *= 2) make(m);
    return P;
  }

  std::vector<boot::Ct> ps(const std::vector<double>& coeffs, int level_out, Powers& P, int nl, cudaStream_t s) const {
    const int nc = (int)coeffs.size();
    if (nc <= PS_BABY) {
      std::vector<int> ks;
      for (int k = 1; k < nc; ++k) ks.push_back(k);
      if (ks.empty()) ks.push_back(1);
      std::vector<double> cf;
      for (int k : ks) cf.push_back(k < nc ? coeffs[k] : 0.0);
      std::vector<std::vector<boot::Ct>> lanes(nl);
      for (int i = 0; i < nl; ++i)
        for (int k : ks) lanes[i].push_back(P.T.at(k)[i]);
      return lincomb_to_many(lanes, cf, coeffs[0], level_out, s);
    }
    int m = 1;
    while (m * 2 <= nc - 1) m *= 2;  // 1 << ((nc - 1).bit_length() - 1)
    std::vector<double> q(nc - m, 0.0), r(coeffs.begin(), coeffs.begin() + m);
    q[0] = coeffs[m];
    for (int j = 1; j < nc - m; ++j) {
      q[j] = 2 * coeffs[m + j];
      r[m - j] -= coeffs[m + j];
    }
    auto qc = ps(q, level_out + 1, P, nl, s);
    const auto& tm = t_at(P, m, level_out + 1, s);
    std::vector<std::pair<boot::Ct, boot::Ct>> pr;
    for (int i = 0; i < nl; ++i) pr.push_back({qc[i], tm[i]});
    auto prod = mul_many(pr, s);
    auto rc = ps(r, level_out, P, nl, s);
    return add_many(prod, rc, s);
  }

  std::vector<boot::Ct> eval_mod_many(const std::vector<boot::Ct>& ts, cudaStream_t s) const {
    Powers P = cheb_powers(ts, prm.degree, s);
    const int depth = (int)std::ceil(std::log2((double)prm.degree)) + 1;
    auto cs = ps(cheb, ts[0].level - depth, P, (int)ts.size(), s);
    for (int k = 0; k < prm.r; ++k) {
      std::vector<std::pair<boot::Ct, boot::Ct>> pr;
      for (const auto& x : cs) pr.push_back({x, x});
      auto sq = mul_many(pr, s);
      std::vector<std::vector<boot::Ct>> lanes;
      for (const auto& x : sq) lanes.push_back({x});
      cs = lincomb_many(lanes, {2}, -1.0, s);
    }
    return cs;
  }

  // Chebyshev series in OpenFHE's convention, p(x) = c_0 / 2 + sum_(k >= 1) c_k T_k(t) with
  // t = (2 x - (lo + hi)) / (hi - lo) (reference evalChebyshevSeries, src/CKKS/ApproxModEval.cu:
  // 527; CryptoContext::EvalChebyshevSeries), by the Paterson-Stockmeyer evaluation above.
  // Inputs at their level's canonical scale (else brought there one level down).  Levels
  // consumed: ceil(log2 d) + 1 for degree d, one more when [lo, hi] is not [-1, 1].
  std::vector<boot::Ct> eval_chebyshev_many(std::vector<boot::Ct> xs, std::vector<double> coeffs, double lo, double hi,
                                            cudaStream_t s) const {
    while (coeffs.size() > 1 && coeffs.back() == 0.0) coeffs.pop_back();
    if (coeffs.empty()) throw Error(-1, "chebyshev: no coefficients");
    coeffs[0] /= 2;
    if (!(hi > lo)) throw Error(-1, "chebyshev: empty interval");
    const int d = (int)coeffs.size() - 1;
    const int depth = d <= 1 ? 1 : (int)std::ceil(std::log2((double)d)) + 1;
    const bool affine = std::abs(lo + 1.0) > 1e-12 || std::abs(hi - 1.0) > 1e-12;
    int l = xs[0].level;
    if (std::abs(xs[0].scale / S[l] - 1) > 1e-12) xs = to_level_many(xs, --l, s);
    if (l - depth - (affine ? 1 : 0) < 1) throw Error(-4, "chebyshev: not enough levels for this degree");
    if (affine) {
      std::vector<std::vector<boot::Ct>> lanes;
      for (const auto& x : xs) lanes.push_back({x});
      xs = lincomb_to_many(lanes, {2.0 / (hi - lo)}, -(hi + lo) / (hi - lo), l - 1, s);
      --l;
    }
    Powers P = cheb_powers(xs, std::max(d, 1), s);
    return ps(coeffs, l - depth, P, (int)xs.size(), s);
  }

  // ---------------------------------------------------------------- the bootstrap
  // Bootstraps a batch of level-1 ciphertexts (c0s[b], c1s[b]) together: every step is one
  // launch sequence over the whole batch (EvalMod runs 2 x batch lanes: the real and imaginary
  // halves of each ciphertext).  Each ciphertext's arithmetic is the same as alone.
  std::vector<boot::Ct> run_many(const std::vector<const uint64_t*>& c0s, const std::vector<const uint64_t*>& c1s,
                                 cudaStream_t s) const {
    if (!prepared) throw Error(-7, "bootstrap: fides_boot_prepare has not run");
    if (!relin || !conj) throw Error(-5, "bootstrap: relinearization / conjugation key not set");
    const size_t B = c0s.size();
    std::vector<boot::Ct> x(B);
    for (size_t b = 0; b < B; ++b) {
      x[b].c0 = c0s[b];
      x[b].c1 = c1s[b];
      x[b].level = 1;
      x[b].scale = prm.msg_scale;
    }
    if (prm.correction_bits > 0) {  // scale down by ~2^k: times round(q_1 / 2^k) at level 2, rescale by q_1
      for (auto& v : x) v.level = 2;
      x = rescale_many_to(mul_int_many(x, corr, s), x[0].scale * corr / (double)c->primes[1], s);
    }
    if (prm.sparse_encapsulation) {
      if (!to_sparse || !to_dense) throw Error(-5, "bootstrap: encapsulation keys not set");
      x = keyswitch_add_many(x, to_sparse, s);  // dense -> sparse secret, at level 1
    }
    if (prm.prescale_bits) x = mul_int_many(x, (double)(1ll << prm.prescale_bits), s);
    std::vector<boot::Ct> a;
    std::vector<const uint64_t*> rin;
    std::vector<uint64_t*> rout;
    for (size_t b = 0; b < B; ++b) {  // ModRaise: m -> m + q0 I on every limb of the top level
      a.push_back(fresh(top, in_scale, s));
      rin.push_back(x[b].c0);
      rin.push_back(x[b].c1);
      rout.push_back(mut(a.back().c0));
      rout.push_back(mut(a.back().c1));
    }
    op_mod_raise_batch(c, rin.data(), (int)rin.size(), top, rout.data(), s);
    if (prm.sparse_encapsulation) a = keyswitch_add_many(a, to_dense, s);  // back to the dense secret
    for (const auto& P : cts_pl) a = prm.double_hoist ? apply_many_dh(a, P, s) : apply_many(a, P, s);
    const std::vector<boot::Ct> cj = conjugate_many(a, s);
    const std::vector<boot::Ct> t_re = add_raw_many(a, cj, s);
    const std::vector<boot::Ct> t_im = mul_plain_int_many(sub_raw_many(a, cj, s), pt_minus_i, s);
    std::vector<boot::Ct> ts;
    for (size_t b = 0; b < B; ++b) {
      ts.push_back(t_re[b]);
      ts.push_back(t_im[b]);
    }
    const std::vector<boot::Ct> sm = eval_mod_many(ts, s);
    std::vector<boot::Ct> sre, sim;
    for (size_t b = 0; b < B; ++b) {
      sre.push_back(sm[2 * b]);
      sim.push_back(sm[2 * b + 1]);
    }
    sre = to_level_many(sre, stc_in_level, s);
    sim = to_level_many(sim, stc_in_level, s);
    std::vector<boot::Ct> u = add_raw_many(sre, mul_plain_int_many(sim, pt_i, s), s);
    for (const auto& P : stc_pl) u = prm.double_hoist ? apply_many_dh(u, P, s) : apply_many(u, P, s);
    return u;
  }

  void run_into(const std::vector<const uint64_t*>& c0s, const std::vector<const uint64_t*>& c1s,
                const std::vector<uint64_t*>& o0s, const std::vector<uint64_t*>& o1s, cudaStream_t s) const {
    const std::vector<boot::Ct> us = run_many(c0s, c1s, s);
    for (size_t b = 0; b < us.size(); ++b) {
      const size_t bytes = sizeof(uint64_t) * (size_t)c->N * us[b].level;
      FIDES_CUDA(cudaMemcpyAsync(o0s[b], us[b].c0, bytes, cudaMemcpyDeviceToDevice, s));
      FIDES_CUDA(cudaMemcpyAsync(o1s[b], us[b].c1, bytes, cudaMemcpyDeviceToDevice, s));
    }
  }
};

}  // namespace fides

struct fides_boot {
  fides_ctx* ctx;
  std::unique_ptr<fides::Bootstrapper> b;
};

namespace {
template <typename F>
int bguard(const char* name, F&& f) {
  (void)name;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  int rc = FIDES_OK;
  try {
    f();
  } catch (const fides::Error& e) {
    fides::set_last_error(e.what());
    rc = e.code;
  } catch (const std::bad_alloc&) {
    fides::set_last_error("host allocation failed");
    rc = FIDES_ERR_OOM;
  } catch (const std::exception& e) {
    fides::set_last_error(e.what());
    rc = FIDES_ERR_STATE;
  }
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}

fides::Bootstrapper* B(fides_boot* b) {
  if (!b || !b->b) throw fides::Error(FIDES_ERR_ARG, "null bootstrapper");
  FIDES_CUDA(cudaSetDevice(b->b->c->device));
  return b->b.get();
}
}  // namespace

extern "C" {

int fides_eval_chebyshev(fides_ctx* ctx, const uint64_t* relin_key, double top_scale, const uint64_t* c0,
                         const uint64_t* c1, int level, double scale, const double* coeffs, int n_coeffs, double lo,
                         double hi, uint64_t* out0, uint64_t* out1, int* out_level, double* out_scale,
                         void* stream) {
  return bguard(__func__, [&] {
    if (!ctx || !ctx->c || !relin_key || !c0 || !c1 || !coeffs || !out0 || !out1)
      throw fides::Error(FIDES_ERR_ARG, "null argument");
    fides::Context* c = ctx->c;
    FIDES_CUDA(cudaSetDevice(c->device));
    if (c->K < 1) throw fides::Error(FIDES_ERR_ARG, "relinearisation needs special primes");
    if (level < 2 || level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "level out of range");
    if (n_coeffs < 1 || n_coeffs > 1025) throw fides::Error(FIDES_ERR_ARG, "1..1025 coefficients");
    if (!(top_scale > 0) || !(scale > 0)) throw fides::Error(FIDES_ERR_ARG, "scales must be positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an evaluator over the context: the canonical scale chain of top_scale and the relinearisation
    // key (no bootstrapping tables)
    fides::Bootstrapper ev{};
    ev.c = c;
    ev.relin = relin_key;
    ev.S.assign(c->n_q + 1, 0.0);
    ev.S[c->n_q] = top_scale;
    for (int l = c->n_q; l > 1; --l) ev.S[l - 1] = ev.S[l] * ev.S[l] / (double)c->primes[l - 1];
    fides::boot::Ct x;
    x.c0 = c0;
    x.c1 = c1;
    x.level = level;
    x.scale = scale;
    auto r = ev.eval_chebyshev_many({x}, std::vector<double>(coeffs, coeffs + n_coeffs), lo, hi, s);
    const size_t bytes = sizeof(uint64_t) * (size_t)c->N * r[0].level;
    FIDES_CUDA(cudaMemcpyAsync(out0, r[0].c0, bytes, cudaMemcpyDeviceToDevice, s));
    FIDES_CUDA(cudaMemcpyAsync(out1, r[0].c1, bytes, cudaMemcpyDeviceToDevice, s));
    if (out_level) *out_level = r[0].level;
    if (out_scale) *out_scale = r[0].scale;
  });
}

int fides_boot_create(fides_ctx* ctx, const fides_boot_params* p, fides_boot** out) {
  return bguard(__func__, [&] {
    if (!ctx || !ctx->c || !p || !out) throw fides::Error(FIDES_ERR_ARG, "null argument");
    fides::Context* c = ctx->c;
    FIDES_CUDA(cudaSetDevice(c->device));
    if (p->level_budget_cts < 1 || p->level_budget_stc < 1 || p->level_budget_cts > c->logN - 1 ||
        p->level_budget_stc > c->logN - 1)
      throw fides::Error(FIDES_ERR_ARG, "level budget out of range");
    if (p->top_level < 2 || p->top_level > c->n_q) throw fides::Error(FIDES_ERR_LEVEL, "top level out of range");
    if (!(p->top_scale > 0) || !(p->msg_scale > 0)) throw fides::Error(FIDES_ERR_ARG, "scales must be positive");
    if (p->degree < 2 || p->K < 1 || p->r < 0 || p->baby < 1 || p->prescale_bits < 0 || p->prescale_bits > 30)
      throw fides::Error(FIDES_ERR_ARG, "EvalMod / BSGS parameters out of range");
    if (p->correction_bits < 0 || p->correction_bits > 40 || (p->correction_bits > 0 && c->n_q < 3))
      throw fides::Error(FIDES_ERR_ARG, "correction_bits out of range (and needs q_1)");
    if (p->double_hoist && p->baby > fides::MAX_BSGS_BABY)
      throw fides::Error(FIDES_ERR_ARG, "double hoisting supports at most 16 baby steps");
    if (c->K < 1) throw fides::Error(FIDES_ERR_ARG, "bootstrapping needs special primes");
    auto* bs = new fides::Bootstrapper{};
    bs->c = c;
    bs->prm = *p;
    try {
      bs->build_tables();
    } catch (...) {
      delete bs;
      throw;
    }
    *out = new fides_boot{ctx, std::unique_ptr<fides::Bootstrapper>(bs)};
  });
}

int fides_boot_destroy(fides_boot* b) {
  return bguard(__func__, [&] {
    if (!b) return;
    if (b->b) {
      cudaSetDevice(b->b->c->device);
      cudaDeviceSynchronize();
    }
    delete b;
  });
}

int fides_boot_rotations(const fides_boot* b, int* out, int cap) {
  if (!b || !b->b) return FIDES_ERR_ARG;
  const auto& r = b->b->rotations;
  for (int i = 0; out && i < cap && i < (int)r.size(); ++i) out[i] = r[i];
  return (int)r.size();
}

int fides_boot_set_keys(fides_boot* b, const uint64_t* relin_key, const uint64_t* conj_key, const uint64_t* to_sparse,
                        const uint64_t* to_dense) {
  return bguard(__func__, [&] {
    auto* bs = B(b);
    if (!relin_key || !conj_key) throw fides::Error(FIDES_ERR_KEY, "relinearization and conjugation keys needed");
    if (bs->prm.sparse_encapsulation && (!to_sparse || !to_dense))
      throw fides::Error(FIDES_ERR_KEY, "sparse encapsulation needs both switching keys");
    bs->relin = relin_key;
    bs->conj = conj_key;
    bs->to_sparse = to_sparse;
    bs->to_dense = to_dense;
  });
}

int fides_boot_set_rotation_key(fides_boot* b, int rotation, const uint64_t* key) {
  return bguard(__func__, [&] {
    auto* bs = B(b);
    if (!key) throw fides::Error(FIDES_ERR_KEY, "null rotation key");
    bs->rot[(int)fides::boot::pymod(rotation, bs->n)] = key;
  });
}

int fides_boot_prepare(fides_boot* b, void* stream) {
  return bguard(__func__, [&] {
    auto* bs = B(b);
    for (int r : bs->rotations)
      if (!bs->rot.count(r)) throw fides::Error(FIDES_ERR_KEY, "missing rotation key " + std::to_string(r));
    bs->prepare(static_cast<cudaStream_t>(stream));
  });
}

int fides_boot_levels(const fides_boot* b, int* out_level, double* out_scale) {
  if (!b || !b->b || !b->b->prepared) return FIDES_ERR_STATE;
  if (out_level) *out_level = b->b->out_level;
  if (out_scale) *out_scale = b->b->S[b->b->out_level];
  return FIDES_OK;
}

int fides_bootstrap(fides_boot* b, const uint64_t* c0, const uint64_t* c1, uint64_t* out0, uint64_t* out1,
                    void* stream) {
  return bguard(__func__, [&] {
    auto* bs = B(b);
    if (!c0 || !c1 || !out0 || !out1) throw fides::Error(FIDES_ERR_ARG, "null polynomial pointer");
    bs->run_into({c0}, {c1}, {out0}, {out1}, static_cast<cudaStream_t>(stream));
  });
}

int fides_bootstrap_batch(fides_boot* b, int n, const uint64_t* const* c0s, const uint64_t* const* c1s,
                          uint64_t* const* out0s, uint64_t* const* out1s, void* stream) {
  return bguard(__func__, [&] {
    auto* bs = B(b);
    if (n < 0) throw fides::Error(FIDES_ERR_ARG, "negative count");
    if (n == 0) return;
    if (!c0s || !c1s || !out0s || !out1s) throw fides::Error(FIDES_ERR_ARG, "null pointer array");
    // batches of up to 16 ciphertexts through one launch sequence each (bounds the memory of
    // the hoisted rotations' extended-basis intermediates)
    constexpr int kChunk = 16;
    for (int i0 = 0; i0 < n; i0 += kChunk) {
      const int m = std::min(kChunk, n - i0);
      std::vector<const uint64_t*> a0, a1;
      std::vector<uint64_t*> o0, o1;
      for (int i = i0; i < i0 + m; ++i) {
        if (!c0s[i] || !c1s[i] || !out0s[i] || !out1s[i]) throw fides::Error(FIDES_ERR_ARG, "null polynomial pointer");
        a0.push_back(c0s[i]);
        a1.push_back(c1s[i]);
        o0.push_back(out0s[i]);
        o1.push_back(out1s[i]);
      }
      bs->run_into(a0, a1, o0, o1, static_cast<cudaStream_t>(stream));
    }
  });
}

int fides_boot_chebyshev(const fides_boot* b, double* coeffs, int cap) {
  if (!b || !b->b) return FIDES_ERR_ARG;
  const auto& v = b->b->cheb;
  for (int i = 0; coeffs && i < cap && i < (int)v.size(); ++i) coeffs[i] = v[i];
  return (int)v.size();
}

int fides_boot_table(const fides_boot* b, int which, int m, int* offsets, int cap, double* diags) {
  if (!b || !b->b || (which != 0 && which != 1)) return FIDES_ERR_ARG;
  const auto& mats = which == 0 ? b->b->cts : b->b->stc;
  if (m < 0 || m >= (int)mats.size()) return FIDES_ERR_ARG;
  const auto& M = mats[m];
  int k = 0;
  for (const auto& [off, d] : M) {
    if (k < cap) {
      if (offsets) offsets[k] = off;
      if (diags) std::memcpy(diags + (size_t)k * 2 * d.size(), d.data(), sizeof(double) * 2 * d.size());
    }
    ++k;
  }
  return k;
}

int fides_boot_plaintext(const fides_boot* b, int which, int m, int i, int j, uint64_t* out, void* stream) {
  return bguard(__func__, [&] {
    if (!b || !b->b || !b->b->prepared || !out) throw fides::Error(FIDES_ERR_STATE, "bootstrapper not prepared");
    const auto& pl = which == 0 ? b->b->cts_pl : b->b->stc_pl;
    if (m < 0 || m >= (int)pl.size()) throw fides::Error(FIDES_ERR_ARG, "matrix index out of range");
    auto it = pl[m].pts.find({i, j});
    if (it == pl[m].pts.end()) throw fides::Error(FIDES_ERR_ARG, "no diagonal at (i, j)");
    FIDES_CUDA(cudaSetDevice(b->b->c->device));
    FIDES_CUDA(cudaMemcpyAsync(out, it->second->u64(), sizeof(uint64_t) * (size_t)b->b->c->N * pl[m].level,
                               cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  });
}

int fides_boot_matrices(const fides_boot* b, int which) {
  if (!b || !b->b || (which != 0 && which != 1)) return FIDES_ERR_ARG;
  return (int)(which == 0 ? b->b->cts : b->b->stc).size();
}

}  // extern "C"
