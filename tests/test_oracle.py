"""CPU tests of the oracle: pinned against the reference's golden vectors and tables,
plus the algebraic properties the reference's own tests check."""
import json
import os

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, decode, encode, xrng
from conftest import GOLDEN


def ref_params():
    return json.load(open(os.path.join(GOLDEN, "ref_params.json")))


def negacyclic_schoolbook(a, b, q):
    N = len(a)
    out = [0] * N
    for i in range(N):
        for j in range(N):
            k = i + j
            v = int(a[i]) * int(b[j])
            if k >= N:
                out[k - N] = (out[k - N] - v) % q
            else:
                out[k] = (out[k] + v) % q
    return out


def test_kat_negacyclic_q17():
    """test/NegacyclicNTTtests.cu:25-124: q = 17, N = 8, NTT round trip and NTT product."""
    k = ref_params()["kat_negacyclic"]
    o = O.Oracle(3, [k["q"]], [], 1)
    assert o.psi[0] == 3  # smallest generator of Z_17^* raised to (q-1)/2N
    v1 = np.array([k["v1"]], dtype=np.uint64)
    v2 = np.array([k["v2"]], dtype=np.uint64)
    f1, f2 = o.ntt(v1, [0]), o.ntt(v2, [0])
    assert np.array_equal(o.ntt(f2, [0], inverse=True), v2)
    prod = o.ntt(o.mul(f1, f2, [0]), [0], inverse=True)
    assert [int(x) for x in prod[0]] == k["product"]


@pytest.mark.parametrize("logN", [4, 6, 8])
def test_ntt_product_matches_schoolbook_on_reference_primes(logN):
    rp = ref_params()
    primes = rp["p64"][:2] + rp["sp64"][:1]
    o = O.Oracle(logN, primes, [], 1)
    rng = xrng(100 + logN)
    ids = list(range(3))
    a = np.stack([rng.integers(0, q, o.N, dtype=np.uint64) for q in primes])
    b = np.stack([rng.integers(0, q, o.N, dtype=np.uint64) for q in primes])
    fa, fb = o.ntt(a, ids), o.ntt(b, ids)
    assert np.array_equal(o.ntt(fa, ids, inverse=True), a)
    c = o.ntt(o.mul(fa, fb, ids), ids, inverse=True)
    for i, q in enumerate(primes):
        assert [int(x) for x in c[i]] == negacyclic_schoolbook(a[i], b[i], q)


def test_ntt_is_bit_reversed_evaluation():
    """EVALUATION order: slot j holds x(psi^(2 brev(j) + 1)) (test/NTTtests.cu:447-467)."""
    logN, N = 5, 32
    q = O.gen_primes(logN, 50, 1)[0]
    o = O.Oracle(logN, [q], [], 1)
    psi = o.psi[0]
    rng = xrng(5)
    x = rng.integers(0, q, N, dtype=np.uint64)
    got = o.ntt(x[None, :], [0])[0]
    for j in range(N):
        e = 2 * int(format(j, f"0{logN}b")[::-1], 2) + 1
        want = sum(int(x[i]) * pow(psi, e * i, q) for i in range(N)) % q
        assert int(got[j]) == want


def test_root_rule():
    for logN, bits in ((13, 50), (16, 60)):
        q = O.gen_primes(logN, bits, 1)[0]
        psi = O.root_2n(q, logN)
        N = 1 << logN
        assert pow(psi, N, q) == q - 1 and pow(psi, 2 * N, q) == 1


def test_conversion_tables_match_reference_math():
    """Pin the oracle's ModUp/ModDown tables to the reference's src/Math.cu (run through
    oracle/_ref/ref_math by tests/golden/make_golden.py)."""
    t = json.load(open(os.path.join(GOLDEN, "ref_math_tables.json")))
    Q, P = t["Q"], t["P"]

    def table_probe(src, dst):
        o = O.Oracle(4, src + dst, [], 1)
        ns, nd = len(src), len(dst)
        sid, did = list(range(ns)), list(range(ns, ns + nd))
        pre, mat = [], []
        for i in range(ns):
            x = np.zeros((ns, o.N), dtype=np.uint64)
            x[i, 0] = 1  # y_i = pre_i
            pre_out = o.switch_basis(x, sid, did)[:, 0]
            qi = src[i]
            hat = 1
            for k, s in enumerate(src):
                if k != i:
                    hat = hat * s % qi
            x[i, 0] = hat  # y_i = 1 -> out_j = mat[i][j]
            mat.append([int(v) for v in o.switch_basis(x, sid, did)[:, 0]])
            pre.append(pre_out)
        return pre, mat

    _, mat = table_probe(P, Q)
    md = t["moddown"]
    assert mat == md["p_hat_PQ"]  # PHatModq
    for e in t["modup"]:
        pre, mat = table_probe(e["src"], e["dst"])
        assert mat == e["mat"]  # PartQlHatModp
        # pre-scale pinned through the product pre_i * mat_ij
        for i, qi in enumerate(e["src"]):
            for j, pj in enumerate(e["dst"]):
                assert int(pre[i][j]) == e["pre"][i] * e["mat"][i][j] % pj
    # P^-1 mod q_j (PInvModq) and PHatInvModp through ModDown of P*x = x
    o = O.Oracle(4, Q, P, 2)
    rng = xrng(9)
    l = len(Q)
    x = np.stack([rng.integers(0, q, o.N, dtype=np.uint64) for q in Q])
    Pm = [1] * l
    for j, q in enumerate(Q):
        for p in P:
            Pm[j] = Pm[j] * p % q
    ext = np.zeros((l + len(P), o.N), dtype=np.uint64)
    ext[:l] = o.mul(x, np.array([[v] * o.N for v in Pm], dtype=np.uint64), list(range(l)))
    assert np.array_equal(o.moddown(ext), x)
    assert md["P_inv_mod_q"] == [pow(Pm[j], q - 2, q) for j, q in enumerate(Q)]


def test_rescale_is_rounded_division():
    """DropLastElementAndScale: out = (x - [x]_{q_top}) / q_top with SwitchModulus' centred lift."""
    logN = 4
    q = O.gen_primes(logN, 50, 4)
    o = O.Oracle(logN, q, [], 1)
    rng = xrng(11)
    l = 4
    coeff = [int(v) for v in rng.integers(-(1 << 62), 1 << 62, o.N)]
    coeff = [c * (1 << 100) + 12345 for c in coeff]
    limbs = np.stack([np.array([c % qi for c in coeff], dtype=np.uint64) for qi in q])
    ev = o.ntt(limbs, list(range(l)))
    out = o.ntt(o.rescale(ev), list(range(l - 1)), inverse=True)
    qt = q[-1]
    for n, c in enumerate(coeff):
        r = c % qt
        if r > qt // 2:
            r -= qt
        want = (c - r) // qt
        for j in range(l - 1):
            assert int(out[j, n]) == want % q[j]


@pytest.fixture(scope="module")
def small_ctx():
    logN = 12
    q = O.gen_primes(logN, 60, 1)
    q += O.gen_primes(logN, 50, 5, exclude=q)
    p = O.gen_primes(logN, 61, 3, exclude=q)
    o = O.Oracle(logN, q, p, 2)
    return o, KeyGen(o)


def test_hmult_and_rotation_decrypt(small_ctx):
    o, kg = small_ctx
    N, D = o.N, 2.0 ** 50
    rng = xrng(7)
    z1 = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    z2 = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    c = kg.encrypt(encode(z1, N, D).astype(np.int64), 6)
    d = kg.encrypt(encode(z2, N, D).astype(np.int64), 6)
    o0, o1 = o.hmult(c[0], c[1], d[0], d[1], kg.relin_key(), rescale=True)
    got = decode(kg.decrypt_limb0(o0, o1), N, D * D / o.q[5])
    assert np.abs(got - z1 * z2).max() < 1e-6
    for r in (1, -3):
        r0, r1 = o.rotate(c[0], c[1], kg.rotation_key(r), r)
        assert np.abs(decode(kg.decrypt_limb0(r0, r1), N, D) - np.roll(z1, -r)).max() < 1e-6
    # conjugation (automorphism index 2N - 1)
    k = 2 * N - 1
    r0, r1 = o.rotate_auto(c[0], c[1], kg.auto_key(k), k)
    assert np.abs(decode(kg.decrypt_limb0(r0, r1), N, D) - np.conj(z1)).max() < 1e-6


def test_hoisted_equals_individual_rotations(small_ctx):
    o, kg = small_ctx
    rng = xrng(8)
    c0 = np.stack([rng.integers(0, q, o.N, dtype=np.uint64) for q in o.q[:4]])
    c1 = np.stack([rng.integers(0, q, o.N, dtype=np.uint64) for q in o.q[:4]])
    rs = [1, -2, 4]
    keys = [kg.rotation_key(r) for r in rs]
    h0, h1 = o.rotate_hoisted(c0, c1, keys, rs)
    for j, r in enumerate(rs):
        s0, s1 = o.rotate(c0, c1, keys[j], r)
        assert np.array_equal(h0[j], s0) and np.array_equal(h1[j], s1)


def test_keyswitch_is_linear(small_ctx):
    """KeySwitch(d) is Z-linear up to the approximate-conversion error: exact on the digit
    inner product, so KSK_IP(digits(a)) + KSK_IP(digits(b)) == KSK_IP of the sums when no
    digit wraps -- checked on the inner product stage, which is exactly linear."""
    o, kg = small_ctx
    key = kg.relin_key()
    rng = xrng(12)
    l = 5
    ids = o.ext_ids(l)
    dA = np.stack([np.stack([rng.integers(0, o.primes[i], o.N, dtype=np.uint64) for i in ids])
                   for _ in range(o.beta(l))])
    dB = np.stack([np.stack([rng.integers(0, o.primes[i], o.N, dtype=np.uint64) for i in ids])
                   for _ in range(o.beta(l))])
    dS = np.stack([o.add(dA[k], dB[k], ids) for k in range(o.beta(l))])
    aA, bA = o.ksk_ip(dA, l, key)
    aB, bB = o.ksk_ip(dB, l, key)
    aS, bS = o.ksk_ip(dS, l, key)
    assert np.array_equal(o.add(aA, aB, ids), aS) and np.array_equal(o.add(bA, bB, ids), bS)


def test_rotation_auto_index():
    logN = 16
    N = 1 << logN
    assert O.rotation_auto_index(logN, 2 * N - 1) == 2 * N - 1
    for r in (1, 2, 5, -1, N // 2 + 3):
        k = O.rotation_auto_index(logN, r)
        rr = r % (N // 2)
        assert k == pow(5, 2 * N - rr, 2 * N)
        assert k * pow(5, rr, 2 * N) % (2 * N) == 1
