// Basis conversion on the tensor cores: an exact INT8-split product on tcgen05.
//
// The conversion out_j = [sum_i y_i T_ij]_{p_j} (ApproxSwitchCRTBasis, reference
// src/Conv.cu:27-423) is written as a byte-level integer matrix product.  With
// y_i = sum_a y_i[a] 2^(8a) (bytes of the pre-scaled residue) and
// T'_ija = T_ij 2^(8a) mod p_j = sum_c t_ija[c] 2^(8c):
//     sum_i y_i T_ij  ==  sum_c 2^(8c) D_c   (mod p_j),   D_c = sum_(i,a) y_i[a] t_ija[c],
// so D = A B with A[m][(i,a)] = y_i[a] (m = coefficient) and B[(i,a)][(j,c)] = t_ija[c]: a
// u8 x u8 -> s32 MMA with K = 8 n_src.  Every D_c is below K 255^2 < 2^23, so the s32
// accumulation is exact; the epilogue recombines the eight planes and reduces modulo p_j,
// giving the same fully reduced residue as the 64-bit SIMT conversion.
#pragma once
#include <cstdint>
#include <vector>

#include "context.hpp"

namespace fides {

// CONV_AUTO runs tables that have a tensor-core form on the tensor cores: at N = 2^16,
// level 30, dnum 3 the conversions of a batched HMult + HRotate step take 0.66 ms there
// against 1.19 ms on the 64-bit SIMT kernel, with identical results.
constexpr bool kConvAutoTensor = true;

constexpr int TC_MAX_SRC = 16;          // K = 8 n_src <= 128 bytes
constexpr int TC_MAX_B_BYTES = 24576;   // B image kept whole in shared memory

inline int tc_kpad(int ns) { return (8 * ns + 31) / 32 * 32; }
inline int tc_nd_pad(int nd) { return (nd + 1) & ~1; }

// Whether a conversion of ns -> nd limbs at ring degree 2^logN has a tensor-core form
// (destination primes must lie in (2^48, 2^62) for the epilogue's reduction).
inline bool conv_tc_fits(int logN, int ns, int nd, const uint64_t* primes, const std::vector<int>& dst_prime) {
  if (logN < 7 || ns < 1 || ns > TC_MAX_SRC || nd < 1 || tc_kpad(ns) * 8 * tc_nd_pad(nd) > TC_MAX_B_BYTES)
    return false;
  for (int id : dst_prime)
    if (primes[id] <= (1ull << 48) || primes[id] >= (1ull << 62)) return false;
  return true;
}

// Builds the B operand image and the per-destination epilogue constants of one table.
void build_tc_image(const uint64_t* mat, int ns, int nd, const std::vector<int>& dst_prime,
                    const uint64_t* primes, std::vector<uint8_t>& b, std::vector<TcDest>& dst,
                    int& kpad, int& nd_pad);

struct ConvJob;
// Launches the tensor-core conversion for jobs whose tables have a tensor-core form.
void launch_conv_tc(Context* c, const ConvJob* jobs, int n, cudaStream_t s);

}  // namespace fides
