"""Exactness of the floating-point modular arithmetic inside the kernels, checked on the CPU.

The kernels compute integer results with FP64 operations whose exactness rests on rounding
bounds; these tests replay the same operation sequences in Python (IEEE doubles, and an exact
fused multiply-add through rational arithmetic) on random and extreme operands, and compare
with exact integer arithmetic:

* the NTT butterfly product for primes below 2^50 (`f_mulmod`, `f_reduce`,
  fideslib-fork_b200/csrc/ntt_impl.cuh), the row passes' twiddle w recovered from its stored
  w / q, and the first stage of a transform on uncentred inputs in [0, q);
* the key-switch inner product's data x data product and final reduction (`ksk_mul_f64`,
  `ksk_canon_f64`, csrc/kernels.cu);
* the tensor-core conversion's fold of eight s32 byte planes with a one-sided quotient
  correction (`tc_fold`, csrc/conv_tc.cu).
"""
import math
import random
from fractions import Fraction

import pytest

RND = 6755399441055744.0  # 1.5 * 2^52
TWO52 = 4503599627370496.0


def fma(a: float, b: float, c: float) -> float:
    """a * b + c with one rounding (float(Fraction) rounds to nearest, ties to even)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def rint(x: float) -> float:
    return (x + RND) - RND


def primes50():
    from fides_b200 import params
    return [q for q in params.config_c(4).q if q < (1 << 50)]


def f_mulmod(y, w, wq, q):
    p = y * w
    e = fma(y, w, -p)
    k = fma(y, wq, RND) - RND
    return fma(-k, q, p) + e


def f_reduce(x, q, qinv):
    return fma(-(fma(x, qinv, RND) - RND), q, x)


def test_ntt_fp64_butterfly_product_is_exact():
    rng = random.Random(11)
    qs = primes50()
    for q in qs[:6] + qs[-3:]:
        qd, qinv = float(q), 1.0 / q
        for it in range(400):
            w = rng.randrange(1, q)
            wq = float(Fraction(w, q))
            bound = int(1.9 * q) if it % 4 else q
            y = rng.randrange(-bound, bound + 1)
            if it % 50 == 0:
                y = bound
            r = f_mulmod(float(y), float(w), wq, qd)
            assert r == int(r)
            r = int(r)
            assert (r - y * w) % q == 0
            assert abs(r) <= q * (0.5 + abs(y) * 2.0 ** -53) + 1
            # alternate-stage reduction of the other operand
            x = rng.randrange(-2 * q + 1, 2 * q)
            xr = f_reduce(float(x), qd, qinv)
            assert (int(xr) - x) % q == 0 and abs(xr) <= q / 2 + 1


def test_row_twiddle_recovered_from_quotient():
    """Row passes store the correctly rounded w / q and recover w = fma(w / q, q, RND) - RND."""
    rng = random.Random(12)
    for q in primes50() + [(1 << 50) - 27, 12289]:
        qd = float(q)
        ws = [rng.randrange(1, q) for _ in range(300)] + [1, 2, q - 1, q - 2, q // 2]
        for w in ws:
            wq = w / q  # correctly rounded, as the host builds the table
            assert wq == float(Fraction(w, q))
            assert fma(wq, qd, RND) - RND == float(w)


def test_first_stage_on_uncentred_inputs():
    """The first pass converts canonical residues in [0, q) without centring them: the
    forward first stage reduces its x operand and multiplies y < q; the inverse first stage
    reduces the sum (< 2q) and multiplies the difference (|d| < q).  Both stay exact and leave
    the bounds the later stages assume (forward: |x +- r| <= 1.125 q + 1; inverse: q / 2 + 1)."""
    rng = random.Random(13)
    for q in primes50()[:4] + [(1 << 50) - 27]:
        qd, qinv = float(q), 1.0 / q
        for it in range(300):
            w = rng.randrange(1, q)
            wq = w / q
            x, y = rng.randrange(0, q), rng.randrange(0, q)
            if it % 50 == 0:
                x, y = q - 1, q - 1
            # forward butterfly
            a = f_reduce(float(x), qd, qinv)
            r = f_mulmod(float(y), float(w), wq, qd)
            for v, ref in ((a + r, x + y * w), (a - r, x - y * w)):
                assert v == int(v) and (int(v) - ref) % q == 0 and abs(v) <= 1.125 * q + 1
            # inverse butterfly
            s0 = f_reduce(float(x) + float(y), qd, qinv)
            s1 = f_mulmod(float(x) - float(y), float(w), wq, qd)
            assert (int(s0) - (x + y)) % q == 0 and abs(s0) <= q / 2 + 1
            assert (int(s1) - (x - y) * w) % q == 0 and abs(s1) <= q * (0.5 + q * 2.0 ** -53) + 1


def ksk_mul_f64(a, b, q, qinv):
    x, y = float(a), float(b)
    p = x * y
    e = fma(x, y, -p)
    k = fma(p, qinv, RND) - RND
    return fma(-k, q, p) + e


def ksk_canon_f64(s, q, qinv):
    k = fma(s, qinv, RND) - RND
    r = fma(-k, q, s)
    if r < 0:
        r = r + q
    bits = Fraction(r + TWO52) - Fraction(TWO52)  # the low 52 bits of r + 2^52
    return int(bits)


def test_ksk_fp64_products_and_reduction():
    rng = random.Random(13)
    for q in primes50():
        qd, qinv = float(q), 1.0 / q
        for it in range(200):
            terms = []
            s = 0.0
            for _ in range(6):  # four digits and two tensor terms at most
                a = rng.randrange(q) if it % 7 else q - 1
                b = rng.randrange(q) if it % 5 else q - 1
                r = ksk_mul_f64(a, b, qd, qinv)
                assert r == int(r) and abs(r) <= q and (int(r) - a * b) % q == 0
                terms.append(a * b)
                s = s + r
            assert s == int(s)
            assert ksk_canon_f64(s, qd, qinv) == sum(terms) % q


def tc_fold(d, q, qinv):
    a0, a1 = d[0] + (d[1] << 8), d[2] + (d[3] << 8)
    a2, a3 = d[4] + (d[5] << 8), d[6] + (d[7] << 8)
    assert max(a0, a1, a2, a3) < 1 << 32
    x, y = a0 + (a1 << 16), a2 + (a3 << 16)
    vd = fma(float(y), 4294967296.0, float(x))
    t = fma(vd, qinv, 2.0 ** -17)
    qh = math.floor(t)
    assert 0 <= qh < 1 << 32
    m = (1 << 64) - 1
    r = (x + (y << 32) - qh * q) & m
    if r >> 63:
        r = (r + q) & m
    return r


@pytest.mark.parametrize("bits", [49, 50, 55, 60, 61])
def test_conversion_fold_one_sided_correction(bits):
    rng = random.Random(bits)
    dmax = 128 * 255 * 255  # K = 128 bytes of u8 x u8 products
    for _ in range(40):
        q = rng.randrange(1 << (bits - 1), 1 << bits) | 1
        if q <= 1 << 48:
            continue
        qinv = 1.0 / q
        for it in range(60):
            if it % 3 == 0:  # next to a multiple of q
                k = rng.randrange((dmax << 56) // q)
                v = k * q + rng.randrange(-32, 33)
                v = max(v, 0)
                d = [(v >> (8 * c)) & 255 for c in range(7)] + [v >> 56]
            else:
                d = [rng.randrange(dmax + 1) for _ in range(8)]
                if it % 11 == 1:
                    d = [dmax] * 8
            v = sum(dc << (8 * c) for c, dc in enumerate(d))
            assert tc_fold(d, q, qinv) == v % q
