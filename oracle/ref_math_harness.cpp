// Harness that runs the REFERENCE's own host math (src/Math.cu, compiled from the
// reference tree by oracle/Makefile's `ref` target) on a prime set given on stdin and
// prints its CRT tables as JSON.  Test infrastructure: it generates golden fixtures that
// pin the oracle's basis-conversion tables (tests/golden/make_golden.py).
//
// stdin: nq np q_0 .. q_{nq-1} p_0 .. p_{np-1}
// stdout: {"q_hat_inv_Q": [[...]], "q_hat_inv_P": [[...]], "p_hat_PQ": [[...]],
//          "P_inv_mod_q": [...], "modinv": [...]}
#include <cstdio>
#include <vector>

#include "Math.cuh"

using FIDESlib::PrimeRecord;

static void print_mat(const char* name, const std::vector<std::vector<uint64_t>>& m, bool comma) {
  printf("\"%s\": [", name);
  for (size_t i = 0; i < m.size(); ++i) {
    printf("%s[", i ? "," : "");
    for (size_t j = 0; j < m[i].size(); ++j) printf("%s%llu", j ? "," : "", (unsigned long long)m[i][j]);
    printf("]");
  }
  printf("]%s\n", comma ? "," : "");
}

int main() {
  int nq = 0, np = 0;
  if (scanf("%d %d", &nq, &np) != 2) return 1;
  std::vector<PrimeRecord> q(nq), p(np);
  for (auto& r : q) {
    unsigned long long v;
    if (scanf("%llu", &v) != 1) return 1;
    r.p = v;
  }
  for (auto& r : p) {
    unsigned long long v;
    if (scanf("%llu", &v) != 1) return 1;
    r.p = v;
  }
  printf("{\n");
  print_mat("q_hat_inv_Q", FIDESlib::q_hat_inv(q), true);
  print_mat("q_hat_inv_P", FIDESlib::q_hat_inv(p), true);
  print_mat("p_hat_PQ", FIDESlib::p_hat(q, p), true);
  auto pinv = FIDESlib::big_P_inv_mod_q(q, p);
  printf("\"P_inv_mod_q\": [");
  for (size_t i = 0; i < pinv.size(); ++i) printf("%s%llu", i ? "," : "", (unsigned long long)pinv[i]);
  printf("],\n\"modinv\": [");
  for (int i = 0; i < nq; ++i)
    printf("%s%llu", i ? "," : "", (unsigned long long)FIDESlib::modinv(12345 + i, q[i].p));
  printf("]\n}\n");
  return 0;
}
