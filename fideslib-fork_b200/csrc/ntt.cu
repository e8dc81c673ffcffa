// Negacyclic NTT / INTT: launch planning (see ntt.cuh for the design, ntt_impl.cuh for
// the kernels).
#include <algorithm>
#include <vector>

#include "ntt_impl.cuh"

namespace fides {

void ntt_limbs(Context* c, const LimbRef* limbs, int n, bool inverse, cudaStream_t s, NttIn in, NttOut out) {
  if (n <= 0) return;
  if (c->logN < 10) throw Error(-1, "GPU NTT needs logN >= 10");
  const bool ok = inverse ? ((in == IN_PLAIN || in == IN_MUL || in == IN_ADD_PMUL) &&
                             (out == OUT_PLAIN || out == OUT_SUB_PINV))
                          : ((in == IN_PLAIN || in == IN_SWITCH || in == IN_CONV_SW || in == IN_SIGNED) &&
                             (out == OUT_PLAIN || out == OUT_MODDOWN || out == OUT_RESCALE || out == OUT_MDRS));
  if (!ok) throw Error(-1, "NTT prologue/epilogue not available in this direction");
  nttk::PassArgs a;
  a.primes = c->d_prime;
  a.tw = inverse ? c->d_tw_inv : c->d_tw_fwd;
  a.twf = inverse ? c->d_twf_inv : c->d_twf_fwd;
  a.tww = inverse ? c->d_tww_inv : c->d_tww_fwd;
  a.f64 = c->d_f64;
  a.inv_last = c->d_inv_last;
  a.pinv = c->d_pinv;
  a.rescale = c->d_rescale;
  a.pmod = c->d_pmod;
  a.pqinv = c->d_pqinv;
  a.logN = c->logN;
  a.log1 = (c->logN + 1) / 2;
  a.n_q = c->n_q;
  {
    uint64_t nf = 0;
    for (int i = 0; i < n; ++i) nf += c->primes[limbs[i].prime] < (1ull << 50);
    c->ntt_limbs_by_form[0] += nf;
    c->ntt_limbs_by_form[1] += (uint64_t)n - nf;
  }
  static thread_local NttLimbList L;  // ~25 KB: keep off the stack
  // balanced chunks of at most the context's chunk size, both passes of a chunk back to back
  const int cap = c->ntt_chunk > 0 ? std::min(c->ntt_chunk, MAX_NTT_LIMBS) : MAX_NTT_LIMBS;
  const int nchunks = (n + cap - 1) / cap, per = (n + nchunks - 1) / nchunks;
  for (int off = 0; off < n; off += per) {
    L.n = std::min(per, n - off);
    std::copy(limbs + off, limbs + off + L.n, L.limbs);
    switch (c->logN) {
      case 10: ntt_transform_10(c, a, L, inverse, in, out, s); break;
      case 11: ntt_transform_11(c, a, L, inverse, in, out, s); break;
      case 12: ntt_transform_12(c, a, L, inverse, in, out, s); break;
      case 13: ntt_transform_13(c, a, L, inverse, in, out, s); break;
      case 14: ntt_transform_14(c, a, L, inverse, in, out, s); break;
      case 15: ntt_transform_15(c, a, L, inverse, in, out, s); break;
      case 16: ntt_transform_16(c, a, L, inverse, in, out, s); break;
      case 17: ntt_transform_17(c, a, L, inverse, in, out, s); break;
      default: throw Error(-1, "GPU NTT supports logN 10..17");
    }
  }
}

void ntt_polys(Context* c, uint64_t* data, int n_polys, int n_limbs, const int* prime_ids, bool inverse,
               cudaStream_t s) {
  std::vector<LimbRef> v((size_t)n_polys * n_limbs);
  for (int p = 0; p < n_polys; ++p)
    for (int i = 0; i < n_limbs; ++i)
      v[(size_t)p * n_limbs + i] = lref(data + ((size_t)p * n_limbs + i) * c->N, prime_ids[i]);
  ntt_limbs(c, v.data(), (int)v.size(), inverse, s);
}

}  // namespace fides
