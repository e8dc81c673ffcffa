"""Chebyshev series evaluation (fides_eval_chebyshev; CryptoContext::EvalChebyshevSeries of the
reference, src/CKKS/ApproxModEval.cu:527, OpenFHE's convention p(x) = c_0 / 2 + sum c_k T_k(t)
on [lo, hi]): decrypted results match the FP64 evaluation of the series at the encrypted slots,
the output level and scale follow the documented depth, the C++ facade's EvalChebyshevSeries
gives the same residues, and a series too deep for the input level is refused."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, decode, encode, xrng

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.chain(13, 60, 50, 14, 3, name="chebyshev")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=83)
    rk = kg.relin_key()
    top = 2.0 ** 50
    S = [0.0] * (prm.n_q + 1)
    S[prm.n_q] = top
    for k in range(prm.n_q, 1, -1):
        S[k - 1] = S[k] * S[k] / prm.q[k - 1]
    return fides, prm, ctx, kg, rk, fides.to_device(rk), top, S


def series(coeffs, x, lo, hi):
    """FP64 value of c_0 / 2 + sum c_k T_k(t), t = (2x - lo - hi) / (hi - lo)."""
    t = (2 * x - lo - hi) / (hi - lo)
    c = np.array(coeffs, dtype=np.float64).copy()
    c[0] /= 2
    return np.polynomial.chebyshev.chebval(t, c)


def openfhe_coeffs(f, lo, hi, degree):
    """Interpolation coefficients of f on [lo, hi] in OpenFHE's convention (c_0 doubled)."""
    c = np.polynomial.chebyshev.chebinterpolate(lambda t: f((hi - lo) / 2 * t + (hi + lo) / 2), degree)
    c[0] *= 2
    return list(c)


@pytest.mark.parametrize("case", ["tanh31", "cubic", "poly7_unit"])
def test_chebyshev_series_decrypts(env, case):
    F, prm, ctx, kg, rk, rk_d, top, S = env
    N, l = prm.N, prm.n_q
    if case == "tanh31":
        lo, hi, coeffs = -4.0, 4.0, openfhe_coeffs(np.tanh, -4.0, 4.0, 31)
    elif case == "cubic":
        lo, hi, coeffs = -2.0, 3.0, [0.5, -0.25, 0.75, 0.125]
    else:
        lo, hi, coeffs = -1.0, 1.0, [0.3, 0.1, -0.2, 0.05, 0.4, -0.1, 0.2, 0.15]
    rng = xrng(400 + len(coeffs))
    x = rng.uniform(lo, hi, N // 2)
    c0, c1 = kg.encrypt(encode(x.astype(np.complex128), N, S[l]).astype(np.int64), l)
    ct = F.Ciphertext(F.to_device(c0), F.to_device(c1))
    out, sc = ctx.eval_chebyshev(ct, rk_d, top, S[l], coeffs, lo, hi)
    d = len(coeffs) - 1
    depth = 1 if d <= 1 else math.ceil(math.log2(d)) + 1
    affine = not (lo == -1.0 and hi == 1.0)
    lvl = out.c0.shape[0]
    assert lvl == l - depth - (1 if affine else 0)
    assert abs(sc / S[lvl] - 1) < 1e-12
    got = decode(kg.decrypt_limb0(F.to_host(out.c0), F.to_host(out.c1)), N, sc).real
    err = np.abs(got - series(coeffs, x, lo, hi)).max()
    assert err < 2.0 ** -20, err
    if case == "tanh31":
        assert np.abs(got - np.tanh(x)).max() < 1e-3  # the interpolant itself is that close


def test_facade_chebyshev_equals_abi(env):
    F, prm, ctx, kg, rk, rk_d, top, S = env
    from test_bootstrap import _facade_lib
    lib = _facade_lib()
    u64p, dp = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
    lib.facade_chebyshev.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, C.c_void_p, C.c_int,
                                     u64p, u64p, dp, C.c_int, C.c_double, C.c_double, u64p, C.POINTER(C.c_int),
                                     dp, C.c_char_p, C.c_int]
    N, l = prm.N, prm.n_q
    lo, hi = -4.0, 4.0
    coeffs = np.array(openfhe_coeffs(np.tanh, lo, hi, 15), dtype=np.float64)
    rng = xrng(450)
    x = rng.uniform(lo, hi, N // 2)
    c0, c1 = kg.encrypt(encode(x.astype(np.complex128), N, S[l]).astype(np.int64), l)
    ref, sc = ctx.eval_chebyshev(F.Ciphertext(F.to_device(c0), F.to_device(c1)), rk_d, top, S[l], coeffs, lo, hi)
    lvl = ref.c0.shape[0]
    out = np.zeros(2 * l * N, dtype=np.uint64)
    ol, osc = C.c_int(0), C.c_double(0)
    err = C.create_string_buffer(512)
    u64 = lambda a: np.ascontiguousarray(a, dtype=np.uint64).ctypes.data_as(u64p)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    rc = lib.facade_chebyshev(prm.logN, l, prm.K, prm.dnum, u64(primes), top, rk_d.data_ptr(), l, u64(c0), u64(c1),
                              coeffs.ctypes.data_as(dp), len(coeffs), lo, hi, u64(out), C.byref(ol), C.byref(osc),
                              err, 512)
    assert rc == 0, err.value.decode()
    assert ol.value == lvl and abs(osc.value / sc - 1) < 1e-15
    assert np.array_equal(out[:lvl * N].reshape(lvl, N), F.to_host(ref.c0))
    assert np.array_equal(out[lvl * N:2 * lvl * N].reshape(lvl, N), F.to_host(ref.c1))


def test_chebyshev_too_deep_refused(env):
    F, prm, ctx, kg, rk, rk_d, top, S = env
    N, l = prm.N, 4
    rng = xrng(460)
    x = rng.uniform(-1, 1, N // 2)
    c0, c1 = kg.encrypt(encode(x.astype(np.complex128), N, S[l]).astype(np.int64), l)
    ct = F.Ciphertext(F.to_device(c0), F.to_device(c1))
    with pytest.raises(F.FidesError) as e:
        ctx.eval_chebyshev(ct, rk_d, top, S[l], [0.1] * 32, -1.0, 1.0)  # degree 31 needs 6 levels
    assert e.value.code == -4
