// Ciphertext operations: hybrid key switching, HMult + relinearize + rescale, rotations.
//
// Stage order follows the reference's live key-switch path
// (src/CKKS/LimbPartitionMGPU.cu:669-1980, modup_ksk_moddown_mgpu):
//   INTT(d) -> ModUp conversion per digit -> NTT(new limbs) -> KSK inner product
//   -> INTT(special limbs) -> ModDown conversion -> NTT -> (x - conv) P^-1
// and, for rotations, the fused hoisted form (LimbPartitionMGPU.cu:517-667): ModUp(c1),
// then one KSK pass that adds P c0 and applies the automorphism as a scatter, then ModDown.
// Each stage is ONE launch over all items of a batch, whatever their levels, and the
// elementwise steps around the transforms are fused into them:
//   * the INTT before ModUp reads its input directly (out of place), or computes the tensor
//     term a1 b1 on the fly (HMult), so d2 is never written;
//   * the ModDown finish (x - conv) P^-1 (+ the tensor terms d0 / d1) is the epilogue of the
//     forward NTT of the converted limbs;
//   * rescale is INTT(top limb) followed by one forward NTT whose prologue applies
//     SwitchModulus to the top limb and whose epilogue forms q_l^-1 x + QlQlInv t.
#include <algorithm>
#include <cstring>

#include "kernels.cuh"
#include "ntt.cuh"
#include "ops.hpp"

namespace fides {

namespace {

struct Bump {
  uint64_t* base;
  size_t N, off = 0;
  uint64_t* take(size_t limbs) {
    uint64_t* p = base + off * N;
    off += limbs;
    return p;
  }
};

void check_level(Context* c, int l, int min_l = 1) {
  if (l < min_l || l > c->n_q) throw Error(-4, "level " + std::to_string(l) + " out of range");
}

// ModUp, first phase: INTT of xs[i] (times ys[i] when given) into tmps[i].
void modup_intt(Context* c, const uint64_t* const* xs, const uint64_t* const* ys, const int* ls,
                uint64_t* const* tmps, int n, cudaStream_t s) {
  const size_t N = c->N;
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < ls[i]; ++j) {
      LimbRef r = lref(tmps[i] + j * N, j);
      r.src = xs[i] + j * N;
      if (ys) r.pro = ys[i] + j * N;
      refs.push_back(r);
    }
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s, ys ? IN_MUL : IN_PLAIN);
}

// ModUp, second phase: conversion of each digit of tmps[i] into digits[i], NTT of the new
// limbs (one conversion launch and one NTT launch sequence for all n inputs).  Own-digit
// limbs of digits[i] are not written.
void modup_convert(Context* c, const int* ls, uint64_t* const* tmps, uint64_t* const* digits, int n,
                   cudaStream_t s) {
  const size_t N = c->N;
  std::vector<ConvJob> jobs;
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i], ext = l + c->K, b = c->beta(l);
    for (int d = 0; d < b; ++d) {
      uint64_t* D = digits[i] + (size_t)d * ext * N;
      jobs.push_back(ConvJob{c->modup_table(l, d), tmps[i], D});
      const int s0 = d * c->alpha, s1 = std::min(l, (d + 1) * c->alpha);
      for (int j = 0; j < l; ++j)
        if (j < s0 || j >= s1) refs.push_back(lref(D + j * N, j));
      for (int k = 0; k < c->K; ++k) refs.push_back(lref(D + (l + k) * N, c->n_q + k));
    }
  }
  launch_conv(c, jobs.data(), (int)jobs.size(), s);
  ntt_limbs(c, refs.data(), (int)refs.size(), false, s);
}

// ModUp of n inputs: INTT of xs[i] (times ys[i] when given) into tmps[i], conversion of each
// digit into digits[i], NTT of the new limbs.  Own-digit limbs of digits[i] are not written.
void modup_stage(Context* c, const uint64_t* const* xs, const uint64_t* const* ys, const int* ls,
                 uint64_t* const* tmps, uint64_t* const* digits, int n, cudaStream_t s) {
  modup_intt(c, xs, ys, ls, tmps, n, s);
  modup_convert(c, ls, tmps, digits, n, s);
}

// ModDown, first phase: INTT of the special limbs of the extended polys exts[i] (in place)
// and their conversion to the Q basis into convs[i] (coefficient form).
void moddown_prep(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs, int n,
                  cudaStream_t s) {
  const size_t N = c->N;
  const int K = c->K;
  if (K == 0) throw Error(-1, "ModDown needs special primes");
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < K; ++k) refs.push_back(lref(exts[i] + (ls[i] + k) * N, c->n_q + k));
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  std::vector<ConvJob> jobs;
  for (int i = 0; i < n; ++i) jobs.push_back(ConvJob{c->moddown_table(ls[i]), exts[i] + ls[i] * N, convs[i]});
  launch_conv(c, jobs.data(), (int)jobs.size(), s);
}

// ModDown, second phase: out = (x - NTT(conv)) P^-1 (+ adds[i]) in one NTT launch sequence.
void moddown_finish(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs,
                    uint64_t* const* outs, const uint64_t* const* adds, int n, cudaStream_t s) {
  const size_t N = c->N;
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i];
    for (int j = 0; j < l; ++j) {
      LimbRef r = lref(outs[i] + j * N, j);
      r.src = convs[i] + j * N;
      r.ep0 = exts[i] + j * N;
      r.ep1 = (adds && adds[i]) ? adds[i] + j * N : nullptr;
      refs.push_back(r);
    }
  }
  ntt_limbs(c, refs.data(), (int)refs.size(), false, s, IN_PLAIN, OUT_MODDOWN);
}

// ModDown of extended polys exts[i] (special limbs are transformed in place) into outs[i],
// adding adds[i] when given.
void moddown_stage(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs, uint64_t* const* outs,
                   const uint64_t* const* adds, int n, cudaStream_t s) {
  moddown_prep(c, exts, ls, convs, n, s);
  moddown_finish(c, exts, ls, convs, outs, adds, n, s);
}

// ModDown fused with the rescale that follows it.  With u = ModDown(x) + add the value
// being rescaled from level l (top prime q_t = q_(l-1)), linearity of the transforms over
// Z_q gives, residue for residue:
//   top   = INTT(u_t) = (INTT(x_t + P add_t) - conv_t) P^-1                (coefficients)
//   out_j = (x_j - NTT(conv_j + P SwitchModulus(top))) (P q_t)^-1 + q_t^-1 add_j,  j < l - 1
// so the result equals ModDown followed by Rescale (reference: NTT<NTT_MODDOWN> then
// rescale, src/CKKS/LimbPartitionMGPU.cu:89-232) bit for bit, with one INTT and l - 1 NTTs
// in place of l NTTs, one INTT and l - 1 NTTs.
// Second phase of a ModDown fused with the rescale (after moddown_prep): the top limb's INTT
// and the forward transforms of the other limbs with the conv + P SwitchModulus(top) prologue.
void moddown_rescale_finish(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs,
                            uint64_t* const* tops, uint64_t* const* outs, const uint64_t* const* adds, int n,
                            cudaStream_t s) {
  const size_t N = c->N;
  std::vector<LimbRef> top_add, top_plain, fwd;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i];
    const uint64_t* add = adds ? adds[i] : nullptr;
    LimbRef t = lref(tops[i], l - 1);
    t.src = exts[i] + (size_t)(l - 1) * N;
    t.pro = add ? add + (size_t)(l - 1) * N : nullptr;
    t.ep0 = convs[i] + (size_t)(l - 1) * N;
    (add ? top_add : top_plain).push_back(t);
    for (int j = 0; j < l - 1; ++j) {
      LimbRef r = lref(outs[i] + j * N, j);
      r.src = convs[i] + j * N;
      r.pro = tops[i];
      r.ep0 = exts[i] + j * N;
      r.ep1 = add ? add + j * N : nullptr;
      r.aux = l;
      fwd.push_back(r);
    }
  }
  ntt_limbs(c, top_add.data(), (int)top_add.size(), true, s, IN_ADD_PMUL, OUT_SUB_PINV);
  ntt_limbs(c, top_plain.data(), (int)top_plain.size(), true, s, IN_PLAIN, OUT_SUB_PINV);
  ntt_limbs(c, fwd.data(), (int)fwd.size(), false, s, IN_CONV_SW, OUT_MDRS);
}

void moddown_rescale_stage(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs,
                           uint64_t* const* tops, uint64_t* const* outs, const uint64_t* const* adds, int n,
                           cudaStream_t s) {
  moddown_prep(c, exts, ls, convs, n, s);
  moddown_rescale_finish(c, exts, ls, convs, tops, outs, adds, n, s);
}

// Scratch limbs of one key switch at level l: INTT copy, digits, A, B, two conversions,
// two rescale tops.
size_t ks_limbs(Context* c, int l) {
  const int ext = l + c->K;
  return (size_t)l + (size_t)c->beta(l) * ext + 2 * (size_t)ext + 2 * (size_t)l + 2;
}

// Key switch of n items whose inputs are xs[i] (or xs[i] * ys[i]); with `rescale` the
// outputs f0/f1 (+ add0/add1) are rescaled to level l - 1 in the same ModDown.
void keyswitch_stage(Context* c, const uint64_t* const* xs, const uint64_t* const* ys, const int* ls,
                     const uint64_t* const* keys, uint64_t* const* f0, uint64_t* const* f1,
                     const uint64_t* const* add0, const uint64_t* const* add1, int n, cudaStream_t s,
                     bool rescale = false, const uint64_t* const* a0s = nullptr,
                     const uint64_t* const* b0s = nullptr) {
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < n; ++i) total += ks_limbs(c, ls[i]);
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<int> ls2(2 * n);
  std::vector<uint64_t*> tmp(n), dig(n), ex(2 * n), conv(2 * n), outs(2 * n), tops(2 * n);
  std::vector<const uint64_t*> adds(2 * n);
  std::vector<KskJob> kj;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i], ext = l + c->K;
    tmp[i] = bp.take(l);
    dig[i] = bp.take((size_t)c->beta(l) * ext);
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    KskJob kjob{xs[i], ys ? ys[i] : nullptr, dig[i], keys[i], nullptr, A, B, l, 0};
    if (a0s) {
      kjob.a0 = a0s[i];
      kjob.b0 = b0s[i];
    }
    kj.push_back(kjob);
    ex[2 * i] = B;
    ex[2 * i + 1] = A;
    conv[2 * i] = bp.take(l);
    conv[2 * i + 1] = bp.take(l);
    tops[2 * i] = bp.take(1);
    tops[2 * i + 1] = bp.take(1);
    outs[2 * i] = f0[i];
    outs[2 * i + 1] = f1[i];
    adds[2 * i] = add0 ? add0[i] : nullptr;
    adds[2 * i + 1] = add1 ? add1[i] : nullptr;
    ls2[2 * i] = ls2[2 * i + 1] = l;
  }
  modup_stage(c, xs, ys, ls, tmp.data(), dig.data(), n, s);
  launch_ksk(c, kj.data(), n, s);
  if (rescale)
    moddown_rescale_stage(c, ex.data(), ls2.data(), conv.data(), tops.data(), outs.data(), adds.data(), 2 * n, s);
  else
    moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), adds.data(), 2 * n, s);
}

}  // namespace

void op_modup(Context* c, const uint64_t* x, int l, uint64_t* digits, cudaStream_t s) {
  check_level(c, l);
  const size_t N = c->N;
  Scratch sc(c, sizeof(uint64_t) * N * l, s);
  uint64_t* tmp = sc.u64();
  modup_stage(c, &x, nullptr, &l, &tmp, &digits, 1, s);
  const int ext = l + c->K;
  for (int d = 0; d < c->beta(l); ++d) {
    const int s0 = d * c->alpha, s1 = std::min(l, (d + 1) * c->alpha);
    FIDES_CUDA(cudaMemcpyAsync(digits + ((size_t)d * ext + s0) * N, x + (size_t)s0 * N,
                               sizeof(uint64_t) * N * (s1 - s0), cudaMemcpyDeviceToDevice, s));
  }
}

void op_ksk_ip(Context* c, const uint64_t* x, const uint64_t* digits, int l, const uint64_t* key, uint64_t* out_a,
               uint64_t* out_b, cudaStream_t s) {
  check_level(c, l);
  if (!key) throw Error(-5, "null key");
  KskJob j{x, nullptr, digits, key, nullptr, out_a, out_b, l, 0};
  launch_ksk(c, &j, 1, s);
}

void op_moddown(Context* c, const uint64_t* x_ext, int l, uint64_t* out, cudaStream_t s) {
  check_level(c, l);
  const size_t N = c->N;
  const int ext = l + c->K;
  Scratch sc(c, sizeof(uint64_t) * N * (ext + l), s);
  uint64_t* e = sc.u64();
  uint64_t* conv = e + (size_t)ext * N;
  FIDES_CUDA(cudaMemcpyAsync(e, x_ext, sizeof(uint64_t) * N * ext, cudaMemcpyDeviceToDevice, s));
  moddown_stage(c, &e, &l, &conv, &out, nullptr, 1, s);
}

void op_tensor(Context* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
               uint64_t* d0, uint64_t* d1, uint64_t* d2, cudaStream_t s) {
  check_level(c, l);
  TensorJob j{a0, a1, b0, b1, d0, d1, d2, l, 0};
  launch_tensor(c, &j, 1, s);
}

void op_keyswitch_batch(Context* c, const KeySwitchItem* items, int n, cudaStream_t s) {
  if (n <= 0) return;
  std::vector<const uint64_t*> xs(n), keys(n), a0(n), a1(n);
  std::vector<uint64_t*> f0(n), f1(n);
  std::vector<int> ls(n);
  for (int i = 0; i < n; ++i) {
    check_level(c, items[i].l);
    if (!items[i].key) throw Error(-5, "null key");
    xs[i] = items[i].d;
    ls[i] = items[i].l;
    keys[i] = items[i].key;
    f0[i] = items[i].f0;
    f1[i] = items[i].f1;
    a0[i] = items[i].add0;
    a1[i] = items[i].add1;
  }
  keyswitch_stage(c, xs.data(), nullptr, ls.data(), keys.data(), f0.data(), f1.data(), a0.data(), a1.data(), n, s);
}

LimbRef rescale_top_ref(Context* c, const uint64_t* x, int l, uint64_t* top) {
  LimbRef r = lref(top, l - 1);
  r.src = x + (size_t)(l - 1) * c->N;
  return r;
}

LimbRef rescale_limb_ref(Context* c, const uint64_t* x, int l, const uint64_t* top, uint64_t* dst, int j) {
  LimbRef t = lref(dst, j);
  t.pro = top;
  t.ep0 = x + (size_t)j * c->N;
  t.aux = l;
  return t;
}

void op_rescale_batch(Context* c, const uint64_t* const* xs, const int* ls, uint64_t* const* outs, int n,
                      cudaStream_t s) {
  if (n <= 0) return;
  const size_t N = c->N;
  // The fused NTT writes its output before its epilogue reads x, so an output that
  // overlaps its input is produced in scratch and copied.
  std::vector<bool> alias(n);
  size_t extra = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, ls[i], 2);
    const uint64_t *x0 = xs[i], *x1 = xs[i] + (size_t)ls[i] * N;
    const uint64_t *o0 = outs[i], *o1 = outs[i] + (size_t)(ls[i] - 1) * N;
    alias[i] = o0 < x1 && x0 < o1;
    if (alias[i]) extra += ls[i] - 1;
  }
  Scratch sc(c, sizeof(uint64_t) * N * (n + extra), s);
  Bump bp{sc.u64(), N};
  std::vector<LimbRef> refs, refs2;
  std::vector<std::pair<uint64_t*, int>> copies;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i];
    uint64_t* dst = outs[i];
    if (alias[i]) {
      dst = bp.take(l - 1);
      copies.push_back({dst, i});
    }
    uint64_t* top = bp.take(1);
    refs.push_back(rescale_top_ref(c, xs[i], l, top));
    for (int j = 0; j < l - 1; ++j) refs2.push_back(rescale_limb_ref(c, xs[i], l, top, dst + j * N, j));
  }
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  ntt_limbs(c, refs2.data(), (int)refs2.size(), false, s, IN_SWITCH, OUT_RESCALE);
  for (auto& cp : copies)
    FIDES_CUDA(cudaMemcpyAsync(outs[cp.second], cp.first, sizeof(uint64_t) * N * (ls[cp.second] - 1),
                               cudaMemcpyDeviceToDevice, s));
}

void op_hmult_batch(Context* c, const HMultItem* items, int n, const uint64_t* relin_key, bool rescale,
                    cudaStream_t s) {
  if (n <= 0) return;
  if (!relin_key) throw Error(-5, "null relinearization key");
  std::vector<const uint64_t*> xs(n), ys(n), a0s(n), b0s(n), keys(n, relin_key);
  std::vector<uint64_t*> f0(n), f1(n);
  std::vector<int> ls(n);
  for (int i = 0; i < n; ++i) {
    const HMultItem& it = items[i];
    check_level(c, it.l, rescale ? 2 : 1);
    xs[i] = it.a1;
    ys[i] = it.b1;
    a0s[i] = it.a0;
    b0s[i] = it.b0;
    ls[i] = it.l;
    f0[i] = it.out0;
    f1[i] = it.out1;
  }
  // The tensor terms d0 = a0 b0 and d1 = a0 b1 + a1 b0 enter the KSK inner product as
  // P d0 / P d1 on the Q limbs (ModDown(x + P d) = ModDown(x) + d exactly), and d2 = a1 b1
  // is formed inside the ModUp INTT and the KSK's own-digit term, so no tensor product is
  // ever written.  The inputs are consumed before the outputs are first written by the
  // final transforms, so outputs may alias inputs.
  keyswitch_stage(c, xs.data(), ys.data(), ls.data(), keys.data(), f0.data(), f1.data(), nullptr, nullptr, n, s,
                  rescale, a0s.data(), b0s.data());
}

void op_rotate_batch(Context* c, const RotateItem* items, int n, cudaStream_t s) {
  if (n <= 0) return;
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, items[i].l);
    if (!items[i].key) throw Error(-5, "null rotation key");
    total += ks_limbs(c, items[i].l);
  }
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<const uint64_t*> xs(n);
  std::vector<int> ls(n), ls2(2 * n);
  std::vector<uint64_t*> tmp(n), dig(n), ex(2 * n), conv(2 * n), outs(2 * n);
  std::vector<KskJob> kj;
  for (int i = 0; i < n; ++i) {
    const RotateItem& it = items[i];
    const int l = it.l, ext = l + c->K;
    xs[i] = it.c1;
    ls[i] = l;
    tmp[i] = bp.take(l);
    dig[i] = bp.take((size_t)c->beta(l) * ext);
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    kj.push_back(KskJob{it.c1, nullptr, dig[i], it.key, it.c0, A, B, l, it.k});
    ex[2 * i] = B;
    ex[2 * i + 1] = A;
    conv[2 * i] = bp.take(l);
    conv[2 * i + 1] = bp.take(l);
    outs[2 * i] = it.out0;
    outs[2 * i + 1] = it.out1;
    ls2[2 * i] = ls2[2 * i + 1] = l;
  }
  modup_stage(c, xs.data(), nullptr, ls.data(), tmp.data(), dig.data(), n, s);
  launch_ksk(c, kj.data(), n, s);
  moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, 2 * n, s);
}

void op_mixed_batch(Context* c, const HMultItem* hm, int nh, const uint64_t* relin_key, bool rescale,
                    const RotateItem* ro, int nr, cudaStream_t s) {
  // HMults and rotations share the stages that do not depend on the kind: one conversion and
  // one NTT launch sequence for every ModUp, one KSK launch (groups by key), one special-limb
  // INTT and one conversion for every ModDown.  The kind-specific transforms (the INTT with
  // the a1 b1 prologue, the final ModDown / ModDown + rescale transforms) stay separate
  // launches.  Each item's arithmetic is that of op_hmult_batch / op_rotate_batch.
  if (nh <= 0 && nr <= 0) return;
  if (nh > 0 && !relin_key) throw Error(-5, "null relinearization key");
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < nh; ++i) {
    check_level(c, hm[i].l, rescale ? 2 : 1);
    total += ks_limbs(c, hm[i].l);
  }
  for (int i = 0; i < nr; ++i) {
    check_level(c, ro[i].l);
    if (!ro[i].key) throw Error(-5, "null rotation key");
    total += ks_limbs(c, ro[i].l);
  }
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  const int n = nh + nr;
  std::vector<const uint64_t*> hx(nh), hy(nh), rx(nr);
  std::vector<int> ls(n), ls2(2 * n);
  std::vector<uint64_t*> tmp(n), dig(n), ex(2 * n), conv(2 * n), tops(2 * n), outs(2 * n);
  std::vector<KskJob> kj;
  for (int i = 0; i < n; ++i) {
    const bool mult = i < nh;
    const int l = mult ? hm[i].l : ro[i - nh].l, ext = l + c->K;
    ls[i] = l;
    tmp[i] = bp.take(l);
    dig[i] = bp.take((size_t)c->beta(l) * ext);
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    if (mult) {
      const HMultItem& it = hm[i];
      hx[i] = it.a1;
      hy[i] = it.b1;
      KskJob job{it.a1, it.b1, dig[i], relin_key, nullptr, A, B, l, 0};
      job.a0 = it.a0;
      job.b0 = it.b0;
      kj.push_back(job);
      outs[2 * i] = it.out0;
      outs[2 * i + 1] = it.out1;
    } else {
      const RotateItem& it = ro[i - nh];
      rx[i - nh] = it.c1;
      kj.push_back(KskJob{it.c1, nullptr, dig[i], it.key, it.c0, A, B, l, it.k});
      outs[2 * i] = it.out0;
      outs[2 * i + 1] = it.out1;
    }
    ex[2 * i] = B;
    ex[2 * i + 1] = A;
    conv[2 * i] = bp.take(l);
    conv[2 * i + 1] = bp.take(l);
    tops[2 * i] = bp.take(1);
    tops[2 * i + 1] = bp.take(1);
    ls2[2 * i] = ls2[2 * i + 1] = l;
  }
  if (nh) modup_intt(c, hx.data(), hy.data(), ls.data(), tmp.data(), nh, s);
  if (nr) modup_intt(c, rx.data(), nullptr, ls.data() + nh, tmp.data() + nh, nr, s);
  modup_convert(c, ls.data(), tmp.data(), dig.data(), n, s);
  launch_ksk(c, kj.data(), n, s);
  moddown_prep(c, ex.data(), ls2.data(), conv.data(), 2 * n, s);
  if (nh) {
    if (rescale)
      moddown_rescale_finish(c, ex.data(), ls2.data(), conv.data(), tops.data(), outs.data(), nullptr, 2 * nh, s);
    else
      moddown_finish(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, 2 * nh, s);
  }
  if (nr)
    moddown_finish(c, ex.data() + 2 * nh, ls2.data() + 2 * nh, conv.data() + 2 * nh, outs.data() + 2 * nh, nullptr,
                   2 * nr, s);
}

namespace {
// Hoisted rotations of several ciphertexts: with `ext_out` the key-switch outputs are left in
// the extended basis in the items' out buffers (l + K limbs each), otherwise one ModDown
// covers every output.
void hoisted_batch(Context* c, const HoistItem* items, int n_items, bool ext_out, cudaStream_t s) {
  // Every ciphertext's c1 is raised once (one ModUp launch sequence over all of them), the KSK
  // pass covers every (ciphertext, rotation) pair -- adding P c0 (or an extended-basis c0)
  // and scattering by the automorphism -- and one ModDown covers every output
  // (hoistedRotateDotKSK_2_ and fusedHoistedRotateBatch, ElemenwiseBatchKernels.cu:277-377,
  // LimbPartitionBatch.cu:526+).
  if (n_items <= 0) return;
  const size_t N = c->N;
  size_t total = 0;
  int n_out = 0;
  for (int i = 0; i < n_items; ++i) {
    const HoistItem& it = items[i];
    check_level(c, it.l);
    for (auto* k : it.keys)
      if (!k) throw Error(-5, "null rotation key");
    if (it.c0 && it.c0x) throw Error(-1, "hoisted rotation: c0 and an extended-basis c0 both given");
    const int l = it.l, ext = l + c->K, r = (int)it.keys.size();
    total += (size_t)l + (size_t)c->beta(l) * ext + (ext_out ? 0 : (size_t)r * (2 * ext + 2 * l));
    n_out += r;
  }
  if (n_out == 0) return;
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<const uint64_t*> xs(n_items);
  std::vector<int> ls(n_items);
  std::vector<uint64_t*> tmp(n_items), dig(n_items);
  for (int i = 0; i < n_items; ++i) {
    const int l = items[i].l, ext = l + c->K;
    xs[i] = items[i].c1;
    ls[i] = l;
    tmp[i] = bp.take(l);
    dig[i] = bp.take((size_t)c->beta(l) * ext);
  }
  modup_stage(c, xs.data(), nullptr, ls.data(), tmp.data(), dig.data(), n_items, s);
  // Job order of the KSK pass.  One ciphertext: its rotations are consecutive, so groups share
  // the digit tile.  Several: the jobs are ordered by (key, level), so the ciphertexts that use
  // one rotation key at one level are consecutive and their groups read each key tile once --
  // the key is the larger stream (2 beta (l + K) limbs against beta (l + K) of digits).
  std::vector<std::pair<int, int>> order;  // (item, rotation)
  for (int i = 0; i < n_items; ++i)
    for (int j = 0; j < (int)items[i].keys.size(); ++j) order.push_back({i, j});
  if (n_items > 1)
    std::stable_sort(order.begin(), order.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
      const uint64_t *ka = items[a.first].keys[a.second], *kb = items[b.first].keys[b.second];
      if (ka != kb) return std::less<const uint64_t*>()(ka, kb);
      return items[a.first].l < items[b.first].l;
    });
  std::vector<KskJob> kj;
  std::vector<uint64_t*> ex, conv, outs;
  std::vector<int> ls2;
  for (const auto& ij : order) {
    const HoistItem& it = items[ij.first];
    const int i = ij.first, l = it.l, ext = l + c->K, j = ij.second;
    uint64_t* A = ext_out ? it.out1[j] : bp.take(ext);
    uint64_t* B = ext_out ? it.out0[j] : bp.take(ext);
    KskJob job{it.c1, nullptr, dig[i], it.keys[j], it.c0, A, B, l, it.ks[j]};
    job.c0x = it.c0x;
    kj.push_back(job);
    if (!ext_out) {
      ex.push_back(B);
      ex.push_back(A);
      conv.push_back(bp.take(l));
      conv.push_back(bp.take(l));
      outs.push_back(it.out0[j]);
      outs.push_back(it.out1[j]);
      ls2.push_back(l);
      ls2.push_back(l);
    }
  }
  launch_ksk(c, kj.data(), (int)kj.size(), s);
  if (!ext_out) moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, (int)outs.size(), s);
}
}  // namespace

void op_hoisted_batch(Context* c, const HoistItem* items, int n_items, cudaStream_t s) {
  hoisted_batch(c, items, n_items, false, s);
}

void op_hoisted_ext_batch(Context* c, const HoistItem* items, int n_items, cudaStream_t s) {
  hoisted_batch(c, items, n_items, true, s);
}

void op_moddown_batch(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* outs, int n, cudaStream_t s) {
  if (n <= 0) return;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, ls[i]);
    total += ls[i];
  }
  Scratch sc(c, sizeof(uint64_t) * c->N * total, s);
  Bump bp{sc.u64(), (size_t)c->N};
  std::vector<uint64_t*> conv(n);
  for (int i = 0; i < n; ++i) conv[i] = bp.take(ls[i]);
  moddown_stage(c, exts, ls, conv.data(), outs, nullptr, n, s);
}

// Rotation sum (reference Accumulate, src/CKKS/AccumulateBroadcast.cu:122-160, behind
// CryptoContext::AccumulateSum): rounds t = 1, radix, radix^2, ... < size; round t rotates the
// running value by stride t k (k = 1 .. radix - 1, while below stride size) as hoisted rotations
// left in the extended basis and adds them.  As in the reference, c0 stays in the extended basis
// (P c0 plus the rotations' extended c0 parts, each rotation adding the running extended c0
// instead of P c0) until one ModDown at the end, while c1 (P c1 + the rotations' c1 parts) is
// brought back by a ModDown every round, because the next round's ModUp reads it.
void op_accumulate(Context* c, const uint64_t* c0, const uint64_t* c1, int l, int radix, int stride, int size,
                   const std::vector<std::pair<int, const uint64_t*>>& keys, uint64_t* out0, uint64_t* out1,
                   cudaStream_t s) {
  check_level(c, l);
  if (radix < 2 || (radix & (radix - 1))) throw Error(-1, "accumulate: radix must be a power of two >= 2");
  if (stride < 1 || size < 1 || (long)stride * size > c->N / 2) throw Error(-1, "accumulate: stride / size out of range");
  const int K = c->K, ext = l + K;
  if (K < 1) throw Error(-1, "accumulate: needs special primes");
  if (ext > MAX_LC_LIMBS || radix > MAX_LC_TERMS) throw Error(-1, "accumulate: too many limbs or terms");
  const size_t N = c->N, lb = sizeof(uint64_t) * N;
  if (out0 != c0) FIDES_CUDA(cudaMemcpyAsync(out0, c0, lb * l, cudaMemcpyDeviceToDevice, s));
  if (out1 != c1) FIDES_CUDA(cudaMemcpyAsync(out1, c1, lb * l, cudaMemcpyDeviceToDevice, s));
  if (size <= 1) return;
  auto key_of = [&](int r) {
    for (const auto& kv : keys)
      if (kv.first == r) return kv.second;
    throw Error(-5, "accumulate: no key for rotation " + std::to_string(r));
  };
  // P mod each limb's prime (0 on the special limbs)
  std::vector<uint64_t> pm(ext, 0);
  for (int j = 0; j < l; ++j) {
    uint64_t v = 1;
    for (int k = 0; k < K; ++k) v = h_mulmod(v, c->primes[c->n_q + k] % c->primes[j], c->primes[j]);
    pm[j] = v;
  }
  // extended buffers: x0e (running c0), x1e (P c1 operand), a1 (c1 sum), radix - 1 rotation pairs
  Scratch sc(c, lb * ext * (3 + 2 * (size_t)(radix - 1)), s);
  Bump bp{sc.u64(), N};
  uint64_t *x0e = bp.take(ext), *x1e = bp.take(ext), *a1 = bp.take(ext);
  std::vector<uint64_t*> r0(radix - 1), r1(radix - 1);
  for (int k = 0; k < radix - 1; ++k) r0[k] = bp.take(ext), r1[k] = bp.take(ext);
  static thread_local LinCombJob j;
  auto combine = [&](const uint64_t* first, const uint64_t* first_scale, int m, uint64_t* const* parts,
                     uint64_t* out) {  // out = first (times first_scale per limb, or 1) + sum parts
    j.n = m + 1;
    j.l = ext;
    j.lanes = 1;
    j.lq = l;
    j.nq = c->n_q;
    for (int i = 0; i < ext; ++i) {
      j.s[0][i] = first_scale ? first_scale[i] : 1;
      j.add0[i] = 0;
    }
    j.x0[0][0] = j.x1[0][0] = first;
    for (int t = 0; t < m; ++t) {
      for (int i = 0; i < ext; ++i) j.s[t + 1][i] = 1;
      j.x0[0][t + 1] = j.x1[0][t + 1] = parts[t];
    }
    j.out0[0] = j.out1[0] = out;  // one polynomial per lane: both halves name the same buffers
    launch_lincomb(c, j, s);
  };
  // x0e = P c0 (its special limbs are zero)
  FIDES_CUDA(cudaMemcpyAsync(x1e, c0, lb * l, cudaMemcpyDeviceToDevice, s));
  FIDES_CUDA(cudaMemsetAsync(x1e + (size_t)l * N, 0, lb * K, s));
  combine(x1e, pm.data(), 0, nullptr, x0e);
  for (long t = 1; t < size; t *= radix) {
    HoistItem it;
    it.c0 = nullptr;
    it.c1 = out1;
    it.l = l;
    it.c0x = x0e;
    for (int k = 1; k < radix && (long)stride * t * k < (long)stride * size; ++k) {
      const int r = (int)(stride * t * k);
      it.keys.push_back(key_of(r));
      it.ks.push_back(h_auto_index(c->logN, r));
      it.out0.push_back(r0[k - 1]);
      it.out1.push_back(r1[k - 1]);
    }
    const int m = (int)it.ks.size();
    op_hoisted_ext_batch(c, &it, 1, s);
    combine(x0e, nullptr, m, r0.data(), a1);  // the extended c0 sum, then back into x0e
    FIDES_CUDA(cudaMemcpyAsync(x0e, a1, lb * ext, cudaMemcpyDeviceToDevice, s));
    FIDES_CUDA(cudaMemcpyAsync(x1e, out1, lb * l, cudaMemcpyDeviceToDevice, s));
    FIDES_CUDA(cudaMemsetAsync(x1e + (size_t)l * N, 0, lb * K, s));
    combine(x1e, pm.data(), m, r1.data(), a1);  // P c1 + the rotations' c1 parts
    int lv = l;
    op_moddown_batch(c, &a1, &lv, &out1, 1, s);
  }
  int lv = l;
  op_moddown_batch(c, &x0e, &lv, &out0, 1, s);
}

void op_moddown_rescale_batch(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* outs, int n,
                              cudaStream_t s) {
  if (n <= 0) return;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, ls[i], 2);
    total += ls[i] + 1;
  }
  Scratch sc(c, sizeof(uint64_t) * c->N * total, s);
  Bump bp{sc.u64(), (size_t)c->N};
  std::vector<uint64_t*> conv(n), tops(n);
  for (int i = 0; i < n; ++i) {
    conv[i] = bp.take(ls[i]);
    tops[i] = bp.take(1);
  }
  moddown_rescale_stage(c, exts, ls, conv.data(), tops.data(), outs, nullptr, n, s);
}

void op_hoisted(Context* c, const HoistItem& it, cudaStream_t s) { op_hoisted_batch(c, &it, 1, s); }

void op_hoisted_digits(Context* c, const uint64_t* c0, const uint64_t* digits, int l, const uint64_t* const* keys,
                       const uint32_t* ks, int n, uint64_t* const* out0, uint64_t* const* out1, cudaStream_t s) {
  // The second half of op_hoisted_batch for digits raised earlier (EvalFastRotationPrecompute):
  // one KSK pass over the n rotations (they share the digit tile), adding P c0 and scattering by
  // each automorphism, then one ModDown over the 2n outputs.  The own-digit limbs are read from
  // the digits (op_modup writes them).
  check_level(c, l);
  if (n <= 0) return;
  const size_t N = c->N;
  const int ext = l + c->K;
  Scratch sc(c, sizeof(uint64_t) * N * (size_t)n * (2 * ext + 2 * l), s);
  Bump bp{sc.u64(), N};
  std::vector<KskJob> kj;
  std::vector<uint64_t*> ex, conv, outs;
  std::vector<int> ls2;
  for (int j = 0; j < n; ++j) {
    if (!keys[j]) throw Error(-5, "null rotation key");
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    kj.push_back(KskJob{nullptr, nullptr, digits, keys[j], c0, A, B, l, ks[j]});
    ex.push_back(B);
    ex.push_back(A);
    conv.push_back(bp.take(l));
    conv.push_back(bp.take(l));
    outs.push_back(out0[j]);
    outs.push_back(out1[j]);
    ls2.push_back(l);
    ls2.push_back(l);
  }
  launch_ksk(c, kj.data(), (int)kj.size(), s);
  moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, (int)outs.size(), s);
}

void op_mod_raise_batch(Context* c, const uint64_t* const* xs, int n, int out_level, uint64_t* const* outs,
                        cudaStream_t s) {
  check_level(c, out_level);
  if (n <= 0) return;
  const size_t N = c->N;
  Scratch sc(c, sizeof(uint64_t) * N * n, s);
  std::vector<LimbRef> in(n);
  for (int i = 0; i < n; ++i) {
    in[i] = lref(sc.u64() + i * N, 0);
    in[i].src = xs[i];
  }
  ntt_limbs(c, in.data(), n, true, s);
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < out_level; ++j) {
      LimbRef t = lref(outs[i] + j * N, j);
      t.pro = sc.u64() + i * N;
      t.aux = 1;  // source prime = aux - 1 = q_0
      refs.push_back(t);
    }
  ntt_limbs(c, refs.data(), (int)refs.size(), false, s, IN_SWITCH, OUT_PLAIN);
}

void op_mod_raise(Context* c, const uint64_t* x, int out_level, uint64_t* out, cudaStream_t s) {
  op_mod_raise_batch(c, &x, 1, out_level, &out, s);
}

}  // namespace fides
