// Ciphertext-level operations composed from the kernels.  Every operation is written for
// a batch of items at arbitrary (uneven) levels; each stage is one launch over all items.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "context.hpp"
#include "ntt.cuh"

namespace fides {

struct KeySwitchItem {
  const uint64_t* d;  // EVAL, level l
  int l;
  const uint64_t* key;
  uint64_t* f0;  // ModDown(sum d b) (+ add0)
  uint64_t* f1;  // ModDown(sum d a) (+ add1)
  const uint64_t* add0 = nullptr;
  const uint64_t* add1 = nullptr;
};

struct HMultItem {
  const uint64_t *a0, *a1, *b0, *b1;
  uint64_t *out0, *out1;
  int l;
};

struct RotateItem {
  const uint64_t *c0, *c1;
  uint64_t *out0, *out1;
  const uint64_t* key;
  int l;
  uint32_t k;  // automorphism index
};

// Hoisted rotations of one ciphertext.
struct HoistItem {
  const uint64_t *c0, *c1;
  int l;
  std::vector<const uint64_t*> keys;
  std::vector<uint32_t> ks;
  std::vector<uint64_t*> out0, out1;
  // instead of P c0 (c0 in the Q basis): an extended-basis c0 (l + K limbs) added as it is
  const uint64_t* c0x = nullptr;
};

void op_modup(Context* c, const uint64_t* x, int l, uint64_t* digits, cudaStream_t s);
void op_ksk_ip(Context* c, const uint64_t* x, const uint64_t* digits, int l, const uint64_t* key, uint64_t* out_a,
               uint64_t* out_b, cudaStream_t s);
void op_moddown(Context* c, const uint64_t* x_ext, int l, uint64_t* out, cudaStream_t s);
void op_tensor(Context* c, const uint64_t* a0, const uint64_t* a1, const uint64_t* b0, const uint64_t* b1, int l,
               uint64_t* d0, uint64_t* d1, uint64_t* d2, cudaStream_t s);

// The NTT limb descriptors of a rescale of one polynomial x at level l (FIXEDMANUAL
// DropLastElementAndScale, Ciphertext::rescale, src/CKKS/Ciphertext.cpp:569-607):
//   * rescale_top_ref: the inverse transform of the top limb x_(l-1) into `top` (one limb);
//   * rescale_limb_ref: output limb j < l - 1 = the forward transform of SwitchModulus(top)
//     (prologue IN_SWITCH) finished by q_(l-1)^-1 x_j + QlQlInvModqlDivqlModq_j t_j (epilogue
//     OUT_RESCALE), written to dst.
// Both rescale paths (op_rescale_batch and the allocation-free entry point) build their
// launches from these, so they run the same transforms.
LimbRef rescale_top_ref(Context* c, const uint64_t* x, int l, uint64_t* top);
LimbRef rescale_limb_ref(Context* c, const uint64_t* x, int l, const uint64_t* top, uint64_t* dst, int j);

void op_keyswitch_batch(Context* c, const KeySwitchItem* items, int n, cudaStream_t s);
void op_rescale_batch(Context* c, const uint64_t* const* xs, const int* ls, uint64_t* const* outs, int n,
                      cudaStream_t s);
void op_hmult_batch(Context* c, const HMultItem* items, int n, const uint64_t* relin_key, bool rescale,
                    cudaStream_t s);
void op_rotate_batch(Context* c, const RotateItem* items, int n, cudaStream_t s);
// HMults (relinearised with relin_key, rescaled when `rescale`) and rotations in one launch
// sequence: the stages common to both kinds (the ModUp conversion and NTT, the KSK inner
// product, the ModDown's special-limb INTT and conversion) run once over all items.  Results
// equal op_hmult_batch / op_rotate_batch item for item.
void op_mixed_batch(Context* c, const HMultItem* hm, int nh, const uint64_t* relin_key, bool rescale,
                    const RotateItem* ro, int nr, cudaStream_t s);
void op_hoisted(Context* c, const HoistItem& item, cudaStream_t s);
// Hoisted rotations of several ciphertexts (any levels, own rotation lists) in one launch
// sequence per stage.
void op_hoisted_batch(Context* c, const HoistItem* items, int n, cudaStream_t s);
// op_hoisted_batch without the ModDown: out0 / out1 of every rotation are extended-basis
// buffers (l + K limbs) that receive the automorphism-scattered key-switch outputs (+ P c0, or
// + c0x), i.e. P times the rotated ciphertext up to the ModDown rounding.
void op_hoisted_ext_batch(Context* c, const HoistItem* items, int n_items, cudaStream_t s);
// ModDown of n extended-basis polynomials exts[i] (l_i + K limbs; their special limbs are
// transformed in place) into outs[i] (l_i limbs), EVAL in and out.
void op_moddown_batch(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* outs, int n, cudaStream_t s);
// Rotation sum x + sum of its rotations by stride t k over rounds t = 1, radix, radix^2, ... <
// size (reference Accumulate); keys = (rotation index, device key) pairs.
void op_accumulate(Context* c, const uint64_t* c0, const uint64_t* c1, int l, int radix, int stride, int size,
                   const std::vector<std::pair<int, const uint64_t*>>& keys, uint64_t* out0, uint64_t* out1,
                   cudaStream_t s);
// ModDown followed by the rescale by q_(l_i - 1), fused (outs[i]: l_i - 1 limbs).
void op_moddown_rescale_batch(Context* c, uint64_t* const* exts, const int* ls, uint64_t* const* outs, int n,
                              cudaStream_t s);
// Hoisted rotations from ModUp digits computed earlier (op_modup of c1, own-digit limbs included):
// rotation j = automorphism ks[j] with key keys[j]; outputs [l][N] each.
void op_hoisted_digits(Context* c, const uint64_t* c0, const uint64_t* digits, int l, const uint64_t* const* keys,
                       const uint32_t* ks, int n, uint64_t* const* out0, uint64_t* const* out1, cudaStream_t s);
// ModRaise (reference Bootstrap.cu ModRaise): a level-1 polynomial (limb q_0, EVAL) raised to
// `out_level` limbs: INTT, SwitchModulus(q_0 -> q_j) of the centred residues, NTT.
void op_mod_raise(Context* c, const uint64_t* x, int out_level, uint64_t* out, cudaStream_t s);
// op_mod_raise of n polynomials in one launch pair each for the INTT and the NTT.
void op_mod_raise_batch(Context* c, const uint64_t* const* xs, int n, int out_level, uint64_t* const* outs,
                        cudaStream_t s);

}  // namespace fides
