// Exercise of the C++ host API (FIDESlibB200.hpp) for the GPU test suite
// (tests/test_cpp_host.py).  Reads parameters, keys and two ciphertexts from a binary
// file, runs the reference-shaped calls and writes every result for the oracle check.
//
// input : u64 logN, n_q, K, dnum, level, rot; primes[n_q+K]; relin key; rotation key;
//         a.c0, a.c1, b.c0, b.c1 (level limbs each)
// output: mult(rescale) c0,c1 | add c0,c1 | rotate c0,c1 | hoisted c0,c1 | keySwitch c0,c1 |
//         rescale c0,c1, each prefixed by its limb count
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "FIDESlibB200.hpp"

using namespace FIDESlib::B200;

static std::vector<uint64_t> rd(FILE* f, size_t n) {
  std::vector<uint64_t> v(n);
  if (fread(v.data(), 8, n, f) != n) {
    fprintf(stderr, "short read\n");
    exit(2);
  }
  return v;
}

static RawCipherText raw_of(const std::vector<uint64_t>& c0, const std::vector<uint64_t>& c1, int l, int N) {
  RawCipherText r;
  r.N = N;
  r.numRes = l;
  for (int i = 0; i < l; ++i) {
    r.sub_0.emplace_back(c0.begin() + (size_t)i * N, c0.begin() + (size_t)(i + 1) * N);
    r.sub_1.emplace_back(c1.begin() + (size_t)i * N, c1.begin() + (size_t)(i + 1) * N);
  }
  return r;
}

static void emit(FILE* f, const Ciphertext& ct) {
  RawCipherText r;
  ct.store(r);
  uint64_t l = (uint64_t)r.numRes;
  fwrite(&l, 8, 1, f);
  for (auto& v : r.sub_0) fwrite(v.data(), 8, v.size(), f);
  for (auto& v : r.sub_1) fwrite(v.data(), 8, v.size(), f);
}

int main(int argc, char** argv) {
  if (argc != 3 && argc != 4) {
    fprintf(stderr, "usage: %s input.bin output.bin [reduced-noise]\n", argv[0]);
    return 2;
  }
  FILE* in = fopen(argv[1], "rb");
  if (!in) return 2;
  auto hdr = rd(in, 6);
  const int logN = (int)hdr[0], nq = (int)hdr[1], K = (int)hdr[2], dnum = (int)hdr[3], l = (int)hdr[4];
  const int rot = (int)(int64_t)hdr[5];
  const int N = 1 << logN;
  auto primes = rd(in, nq + K);
  const size_t ksz = 2 * (size_t)dnum * (nq + K) * N;
  auto rk = rd(in, ksz), kr = rd(in, ksz);
  auto a0 = rd(in, (size_t)l * N), a1 = rd(in, (size_t)l * N), b0 = rd(in, (size_t)l * N), b1 = rd(in, (size_t)l * N);
  fclose(in);
  try {
    Parameters p;
    p.logN = logN;
    p.dnum = dnum;
    p.primes.assign(primes.begin(), primes.begin() + nq);
    p.Sprimes.assign(primes.begin() + nq, primes.end());
    p.reducedNoise = argc == 4;
    Context cc(p);
    {
      KeySwitchingKey k(cc);
      k.InitializeFlat(rk.data());
      cc.AddEvalKey(std::move(k));
    }
    {
      // exercise the RawKeySwitchKey path for the rotation key
      RawKeySwitchKey raw;
      raw.r_key.resize(2);
      for (int ab = 0; ab < 2; ++ab) {
        raw.r_key[ab].resize(dnum);
        for (int d = 0; d < dnum; ++d)
          for (int i = 0; i < nq + K; ++i) {
            auto it = kr.begin() + (((size_t)ab * dnum + d) * (nq + K) + i) * N;
            raw.r_key[ab][d].emplace_back(it, it + N);
          }
      }
      KeySwitchingKey k(cc);
      k.Initialize(raw);
      cc.AddRotationKey(rot, std::move(k));
    }
    FILE* out = fopen(argv[2], "wb");
    Ciphertext A(cc, raw_of(a0, a1, l, N)), B(cc, raw_of(b0, b1, l, N));
    Ciphertext M(cc, raw_of(a0, a1, l, N));
    M.mult(B, /*rescale=*/true);
    emit(out, M);
    Ciphertext S(cc, raw_of(a0, a1, l, N));
    S.add(B);
    emit(out, S);
    Ciphertext R(cc, raw_of(a0, a1, l, N));
    R.rotate(rot);
    emit(out, R);
    Ciphertext H(cc);
    A.rotate_hoisted({rot}, {&H});
    emit(out, H);
    Ciphertext KS(cc, raw_of(a0, a1, l, N));
    KS.keySwitch(cc.GetEvalKey());
    emit(out, KS);
    Ciphertext RS(cc, raw_of(a0, a1, l, N));
    RS.rescale();
    emit(out, RS);
    fclose(out);
    // error path: a missing key surfaces as an exception with the library's status
    try {
      Ciphertext X(cc, raw_of(a0, a1, l, N));
      X.rotate(rot + 1);
      fprintf(stderr, "missing key not reported\n");
      return 1;
    } catch (const Error& e) {
      if (e.code != FIDES_ERR_KEY) return 1;
    }
  } catch (const std::exception& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  printf("host api ok\n");
  return 0;
}
