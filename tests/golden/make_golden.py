"""Generate the golden fixtures that pin the CPU oracle to the reference.

Run where the reference tree is checked out, with FIDES_REFERENCE=<its directory>; the
outputs are committed, so nothing at test time reads the reference.

  * ref_params.json      -- the reference's own test moduli (test/ParametrizedTest.cuh:
                            p64 / sp64 lists) and the q=17, N=8 negacyclic known-answer
                            vectors of test/NegacyclicNTTtests.cu:25-124, with the
                            schoolbook negacyclic product computed here in Python ints.
  * ref_math_tables.json -- CRT tables produced by RUNNING the reference's src/Math.cu
                            (q_hat_inv, p_hat, big_P_inv_mod_q, modinv) through
                            oracle/_ref/ref_math (built by `make -C oracle ref`) on the
                            params64_13 moduli (logN 13, L+1 = 6, dnum = 2 -> alpha = 3,
                            3 special primes): ModDown tables and per-digit ModUp tables.
"""
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("FIDES_REFERENCE", "")
if not REF or not os.path.isdir(os.path.join(REF, "src")):
    sys.exit("make_golden.py: set FIDES_REFERENCE to the reference source tree")


def prime_list(text, name):
    m = re.search(r"PrimeRecord>\s+%s\{(.*?)\};" % name, text, re.S)
    return [int(x) for x in re.findall(r"\.p\s*=\s*(\d+)", m.group(1))]


def kat_vectors(text):
    v1 = re.search(r"std::vector<uint64_t> v1\{([^}]*)\}", text).group(1)
    v2 = re.search(r"std::vector<uint64_t> v2\{([^}]*)\}", text).group(1)
    return [int(x) for x in v1.split(",")], [int(x) for x in v2.split(",")]


def run_ref_math(q, p):
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_math")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    inp = f"{len(q)} {len(p)} " + " ".join(str(x) for x in q + p)
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout
    return json.loads(out)


def main():
    hdr = open(os.path.join(REF, "test", "ParametrizedTest.cuh")).read()
    p64, sp64 = prime_list(hdr, "p64"), prime_list(hdr, "sp64")
    kat = open(os.path.join(REF, "test", "NegacyclicNTTtests.cu")).read()
    v1, v2 = kat_vectors(kat)
    q, N = 17, 8
    prod = [0] * N
    for i in range(N):
        for j in range(N):
            k = i + j
            if k >= N:
                prod[k - N] = (prod[k - N] - v1[i] * v2[j]) % q
            else:
                prod[k] = (prod[k] + v1[i] * v2[j]) % q
    params = {
        "source": "reference test/ParametrizedTest.cuh (p64, sp64); test/NegacyclicNTTtests.cu:25-124",
        "p64": p64, "sp64": sp64,
        "kat_negacyclic": {"q": q, "N": N, "v1": v1, "v2": v2, "product": prod},
        "params64_13": {"logN": 13, "L": 5, "dnum": 2},
    }
    json.dump(params, open(os.path.join(HERE, "ref_params.json"), "w"), indent=1)

    # params64_13: Q = p64[0:6], P = sp64[0:3], alpha = 3 (dnum 2)
    Q, P, alpha = p64[:6], sp64[:3], 3
    tables = {"Q": Q, "P": P, "alpha": alpha,
              "moddown": run_ref_math(Q, P), "modup": []}
    for l in (6, 4):
        for d in range((l + alpha - 1) // alpha):
            digit = Q[d * alpha:min(l, (d + 1) * alpha)]
            targets = [x for i, x in enumerate(Q[:l]) if not d * alpha <= i < (d + 1) * alpha] + P
            t = run_ref_math(targets, digit)
            tables["modup"].append({"level": l, "digit": d, "src": digit, "dst": targets,
                                    "pre": t["q_hat_inv_P"][-1], "mat": t["p_hat_PQ"]})
    json.dump(tables, open(os.path.join(HERE, "ref_math_tables.json"), "w"), indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    sys.exit(main())
