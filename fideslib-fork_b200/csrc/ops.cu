// Ciphertext operations: hybrid key switching, HMult + relinearize + rescale, rotations.
//
// Stage order follows the reference's live key-switch path
// (src/CKKS/LimbPartitionMGPU.cu:669-1980, modup_ksk_moddown_mgpu):
//   INTT(d) -> ModUp conversion per digit -> NTT(new limbs) -> KSK inner product
//   -> INTT(special limbs) -> ModDown conversion -> NTT -> (x - conv) P^-1
// and, for rotations, the fused hoisted form (LimbPartitionMGPU.cu:517-667): ModUp(c1),
// then one KSK pass that adds P c0 and applies the automorphism as a scatter, then ModDown.
// Each stage is ONE launch over all items of a batch, whatever their levels.
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

// INTT copies of xs into tmps, ModUp conversions into digits, NTT of the new limbs.
void modup_stage(Context* c, const uint64_t* const* xs, const int* ls, uint64_t* const* tmps,
                 uint64_t* const* digits, int n, cudaStream_t s) {
  const size_t N = c->N;
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i) {
    FIDES_CUDA(cudaMemcpyAsync(tmps[i], xs[i], sizeof(uint64_t) * N * ls[i], cudaMemcpyDeviceToDevice, s));
    for (int j = 0; j < ls[i]; ++j) refs.push_back(LimbRef{tmps[i] + j * N, j, 0});
  }
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  std::vector<ConvJob> jobs;
  refs.clear();
  for (int i = 0; i < n; ++i) {
    const int l = ls[i], ext = l + c->K, b = c->beta(l);
    for (int d = 0; d < b; ++d) {
      uint64_t* D = digits[i] + (size_t)d * ext * N;
      jobs.push_back(ConvJob{c->modup_tab[l][d], tmps[i], D});
      const int s0 = d * c->alpha, s1 = std::min(l, (d + 1) * c->alpha);
      for (int j = 0; j < l; ++j)
        if (j < s0 || j >= s1) refs.push_back(LimbRef{D + j * N, j, 0});
      for (int k = 0; k < c->K; ++k) refs.push_back(LimbRef{D + (l + k) * N, c->n_q + k, 0});
    }
  }
  launch_conv(c, jobs.data(), (int)jobs.size(), s);
  ntt_limbs(c, refs.data(), (int)refs.size(), false, s);
}

// ModDown of extended polys exts[i] (special limbs are transformed in place) into outs[i].
void moddown_stage(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* convs, uint64_t* const* outs,
                   const uint64_t* const* adds, int n, cudaStream_t s) {
  const size_t N = c->N;
  const int K = c->K;
  std::vector<LimbRef> refs;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < K; ++k) refs.push_back(LimbRef{exts[i] + (ls[i] + k) * N, c->n_q + k, 0});
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  std::vector<ConvJob> jobs;
  refs.clear();
  std::vector<FinJob> fin;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i];
    jobs.push_back(ConvJob{c->moddown_tab[l], exts[i] + l * N, convs[i]});
    for (int j = 0; j < l; ++j) refs.push_back(LimbRef{convs[i] + j * N, j, 0});
    fin.push_back(FinJob{exts[i], convs[i], adds ? adds[i] : nullptr, outs[i], l, 0});
  }
  if (K > 0) {
    launch_conv(c, jobs.data(), (int)jobs.size(), s);
    ntt_limbs(c, refs.data(), (int)refs.size(), false, s);
  } else {
    for (int i = 0; i < n; ++i) FIDES_CUDA(cudaMemsetAsync(convs[i], 0, sizeof(uint64_t) * N * ls[i], s));
  }
  launch_moddown_finish(c, fin.data(), (int)fin.size(), s);
}

size_t ks_limbs(Context* c, int l) {
  const int ext = l + c->K;
  return (size_t)l + (size_t)c->beta(l) * ext + 2 * (size_t)ext + 2 * (size_t)l;
}

}  // namespace

void op_modup(Context* c, const uint64_t* x, int l, uint64_t* digits, cudaStream_t s) {
  check_level(c, l);
  const size_t N = c->N;
  Scratch sc(c, sizeof(uint64_t) * N * l, s);
  uint64_t* tmp = sc.u64();
  modup_stage(c, &x, &l, &tmp, &digits, 1, s);
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
  KskJob j{x, digits, key, nullptr, out_a, out_b, l, 0};
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
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, items[i].l);
    if (!items[i].key) throw Error(-5, "null key");
    total += ks_limbs(c, items[i].l);
  }
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<const uint64_t*> xs(n);
  std::vector<int> ls(n), ls2(2 * n);
  std::vector<uint64_t*> tmp(n), dig(n), ex(2 * n), conv(2 * n), outs(2 * n);
  std::vector<const uint64_t*> adds(2 * n);
  std::vector<KskJob> kj;
  for (int i = 0; i < n; ++i) {
    const KeySwitchItem& it = items[i];
    const int l = it.l, ext = l + c->K;
    xs[i] = it.d;
    ls[i] = l;
    tmp[i] = bp.take(l);
    dig[i] = bp.take((size_t)c->beta(l) * ext);
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    kj.push_back(KskJob{it.d, dig[i], it.key, nullptr, A, B, l, 0});
    ex[2 * i] = B;
    ex[2 * i + 1] = A;
    conv[2 * i] = bp.take(l);
    conv[2 * i + 1] = bp.take(l);
    outs[2 * i] = it.f0;
    outs[2 * i + 1] = it.f1;
    adds[2 * i] = it.add0;
    adds[2 * i + 1] = it.add1;
    ls2[2 * i] = ls2[2 * i + 1] = l;
  }
  modup_stage(c, xs.data(), ls.data(), tmp.data(), dig.data(), n, s);
  launch_ksk(c, kj.data(), n, s);
  moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), adds.data(), 2 * n, s);
}

void op_rescale_batch(Context* c, const uint64_t* const* xs, const int* ls, uint64_t* const* outs, int n,
                      cudaStream_t s) {
  if (n <= 0) return;
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, ls[i], 2);
    total += 1 + (size_t)(ls[i] - 1);
  }
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<LimbRef> refs, refs2;
  std::vector<SwitchJob> sw;
  std::vector<RescaleJob> fin;
  for (int i = 0; i < n; ++i) {
    const int l = ls[i];
    uint64_t* top = bp.take(1);
    uint64_t* t = bp.take(l - 1);
    FIDES_CUDA(cudaMemcpyAsync(top, xs[i] + (size_t)(l - 1) * N, sizeof(uint64_t) * N, cudaMemcpyDeviceToDevice, s));
    refs.push_back(LimbRef{top, l - 1, 0});
    sw.push_back(SwitchJob{top, t, l, 0});
    for (int j = 0; j < l - 1; ++j) refs2.push_back(LimbRef{t + j * N, j, 0});
    fin.push_back(RescaleJob{xs[i], t, outs[i], l, 0});
  }
  ntt_limbs(c, refs.data(), (int)refs.size(), true, s);
  launch_switch_modulus(c, sw.data(), n, s);
  ntt_limbs(c, refs2.data(), (int)refs2.size(), false, s);
  launch_rescale_finish(c, fin.data(), n, s);
}

void op_hmult_batch(Context* c, const HMultItem* items, int n, const uint64_t* relin_key, bool rescale,
                    cudaStream_t s) {
  if (n <= 0) return;
  if (!relin_key) throw Error(-5, "null relinearization key");
  const size_t N = c->N;
  size_t total = 0;
  for (int i = 0; i < n; ++i) {
    check_level(c, items[i].l, rescale ? 2 : 1);
    total += (size_t)items[i].l * (rescale ? 5 : 3);
  }
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  std::vector<TensorJob> tj;
  std::vector<KeySwitchItem> ks;
  std::vector<const uint64_t*> rx;
  std::vector<uint64_t*> ro;
  std::vector<int> rl;
  for (int i = 0; i < n; ++i) {
    const HMultItem& it = items[i];
    const int l = it.l;
    uint64_t* d0 = bp.take(l);
    uint64_t* d1 = bp.take(l);
    uint64_t* d2 = bp.take(l);
    tj.push_back(TensorJob{it.a0, it.a1, it.b0, it.b1, d0, d1, d2, l, 0});
    uint64_t* o0 = it.out0;
    uint64_t* o1 = it.out1;
    if (rescale) {
      o0 = bp.take(l);
      o1 = bp.take(l);
      rx.push_back(o0);
      rx.push_back(o1);
      ro.push_back(it.out0);
      ro.push_back(it.out1);
      rl.push_back(l);
      rl.push_back(l);
    }
    ks.push_back(KeySwitchItem{d2, l, relin_key, o0, o1, d0, d1});
  }
  launch_tensor(c, tj.data(), n, s);
  op_keyswitch_batch(c, ks.data(), n, s);
  if (rescale) op_rescale_batch(c, rx.data(), rl.data(), ro.data(), (int)rx.size(), s);
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
    kj.push_back(KskJob{it.c1, dig[i], it.key, it.c0, A, B, l, it.k});
    ex[2 * i] = B;
    ex[2 * i + 1] = A;
    conv[2 * i] = bp.take(l);
    conv[2 * i + 1] = bp.take(l);
    outs[2 * i] = it.out0;
    outs[2 * i + 1] = it.out1;
    ls2[2 * i] = ls2[2 * i + 1] = l;
  }
  modup_stage(c, xs.data(), ls.data(), tmp.data(), dig.data(), n, s);
  launch_ksk(c, kj.data(), n, s);
  moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, 2 * n, s);
}

void op_hoisted(Context* c, const HoistItem& it, cudaStream_t s) {
  const int n = (int)it.keys.size();
  if (n <= 0) return;
  check_level(c, it.l);
  const size_t N = c->N;
  const int l = it.l, ext = l + c->K;
  for (int j = 0; j < n; ++j)
    if (!it.keys[j]) throw Error(-5, "null rotation key");
  size_t total = (size_t)l + (size_t)c->beta(l) * ext + (size_t)n * (2 * ext + 2 * l);
  Scratch sc(c, sizeof(uint64_t) * N * total, s);
  Bump bp{sc.u64(), N};
  uint64_t* tmp = bp.take(l);
  uint64_t* dig = bp.take((size_t)c->beta(l) * ext);
  modup_stage(c, &it.c1, &l, &tmp, &dig, 1, s);
  std::vector<KskJob> kj;
  std::vector<uint64_t*> ex(2 * n), conv(2 * n), outs(2 * n);
  std::vector<int> ls2(2 * n, l);
  for (int j = 0; j < n; ++j) {
    uint64_t* A = bp.take(ext);
    uint64_t* B = bp.take(ext);
    kj.push_back(KskJob{it.c1, dig, it.keys[j], it.c0, A, B, l, it.ks[j]});
    ex[2 * j] = B;
    ex[2 * j + 1] = A;
    conv[2 * j] = bp.take(l);
    conv[2 * j + 1] = bp.take(l);
    outs[2 * j] = it.out0[j];
    outs[2 * j + 1] = it.out1[j];
  }
  launch_ksk(c, kj.data(), n, s);
  moddown_stage(c, ex.data(), ls2.data(), conv.data(), outs.data(), nullptr, 2 * n, s);
}

}  // namespace fides
