"""Reduced-noise basis conversion: the reference's Parameters::reducedNoise option
(src/CKKS/Parameters.cuh:31), read by its ModUp and ModDown conversions (DecompAndModUpConv and
ModDown2, src/CKKS/Conv.cu:356-381 and :76-87; ReducedNoise.cuh:14-16): a pre-scaled source
residue y_i above q_i / 2 is taken as y_i - q_i, so the converted value gains
cnt * [-Q_src]_{p_j}, cnt the number of such residues of the coefficient.

CPU: the oracle's lifted conversion equals an exact big-integer restatement, its ModUp and
ModDown use it only with the flag, and the flag shrinks the key-switching error as intended.
GPU: ModUp / ModDown / key switching / HMult / rotations / hoisted rotations with the flag equal
the oracle with the flag on both conversion engines, and the reference's own conversion kernels
with the flag equal the oracle (tests/test_ref_kernels.py)."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng


def small_params():
    from fides_b200 import params as P
    return P.chain(10, 60, 50, 6, 2, K=2)


def lifted_switch(x, src, dst, primes, lift):
    """Exact restatement with Python integers: out_j = [sum_i y'_i Qhat_i]_{p_j}."""
    Q = 1
    for s in src:
        Q *= primes[s]
    N = x.shape[1]
    out = np.zeros((len(dst), N), dtype=np.uint64)
    qh = [Q // primes[s] for s in src]
    pre = [pow(qh[i] % primes[s], -1, primes[s]) for i, s in enumerate(src)]
    for n in range(N):
        v = 0
        for i, s in enumerate(src):
            q = primes[s]
            y = int(x[i, n]) * pre[i] % q
            if lift and y > q >> 1:
                y -= q
            v += y * qh[i]
        for j, t in enumerate(dst):
            out[j, n] = v % primes[t]
    return out


def test_oracle_lifted_conversion_equals_bigint_restatement():
    prm = small_params()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    primes = prm.q + prm.p
    src, dst = [0, 1, 2], [3, 4, 5, 6, 7]  # a ModUp digit: 3 Q primes -> the rest and P
    x = uniform_limbs(xrng(3100), [primes[s] for s in src], o.N)
    plain = o.switch_basis(x, src, dst)
    lifted = o.switch_basis(x, src, dst, lift=True)
    assert np.array_equal(plain, lifted_switch(x, src, dst, primes, False))
    assert np.array_equal(lifted, lifted_switch(x, src, dst, primes, True))
    assert not np.array_equal(plain, lifted)
    # ModDown direction: the special primes -> Q primes
    sp = uniform_limbs(xrng(3101), prm.p, o.N)
    src, dst = [prm.n_q, prm.n_q + 1], list(range(prm.n_q))
    assert np.array_equal(o.switch_basis(sp, src, dst, lift=True), lifted_switch(sp, src, dst, primes, True))


def test_oracle_modup_moddown_follow_the_flag():
    """With the flag, the oracle's ModUp and ModDown are INTT -> lifted conversion -> NTT."""
    prm = small_params()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=True)
    plain = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    l = prm.n_q
    x = uniform_limbs(xrng(3200), prm.q, o.N)
    dig = o.modup(x)
    assert not np.array_equal(dig, plain.modup(x))
    ext = l + prm.K
    for d in range(o.beta(l)):
        lo, hi = d * o.alpha, min(l, (d + 1) * o.alpha)
        src = list(range(lo, hi))
        dst = [i for i in range(l) if i < lo or i >= hi] + list(range(prm.n_q, prm.n_q + prm.K))
        pos = [i for i in range(l) if i < lo or i >= hi] + list(range(l, ext))
        conv = o.switch_basis(o.ntt(x[lo:hi], src, inverse=True), src, dst, lift=True)
        assert np.array_equal(dig[d][pos], o.ntt(conv, dst))
        assert np.array_equal(dig[d][lo:hi], x[lo:hi])
    y = uniform_limbs(xrng(3201), prm.q + prm.p, o.N)
    sp_ids = list(range(prm.n_q, prm.n_q + prm.K))
    conv = o.ntt(o.switch_basis(o.ntt(y[l:], sp_ids, inverse=True), sp_ids, list(range(l)), lift=True),
                 list(range(l)))
    Pinv = []
    for q in prm.q:
        P = 1
        for p in prm.p:
            P = P * p % q
        Pinv.append(pow(P, -1, q))
    want = o.mul(o.sub(y[:l], conv, list(range(l))), np.array([[v] * o.N for v in Pinv], dtype=np.uint64),
                 list(range(l)))
    assert np.array_equal(o.moddown(y), want)
    assert not np.array_equal(o.moddown(y), plain.moddown(y))


def _keyswitch_error_rms(prm, reduced_noise):
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=reduced_noise)
    kg = KeyGen(o, seed_stream=41)  # the same keys for both settings
    rk = kg.relin_key()
    d = uniform_limbs(xrng(3300), prm.q, o.N)
    f0, f1 = o.keyswitch(d, rk)
    s = kg.s_eval[:1]
    err = o.sub(o.add(f0[:1], o.mul(f1[:1], s, [0]), [0]), o.mul(d[:1], o.mul(s, s, [0]), [0]), [0])
    e = o.ntt(err, [0], inverse=True)[0].astype(object)
    q0 = prm.q[0]
    c = np.array([int(v) - q0 if int(v) > q0 // 2 else int(v) for v in e], dtype=np.float64)
    return float(np.sqrt(np.mean(c * c)))


def test_reduced_noise_shrinks_key_switch_error():
    """With P well below the first digit's modulus Q_0 the key-switch error is dominated by
    rep(d_0) e_0 / P, rep = the integer ModUp lifts the digit to: sum_i y_i Qhat_i lies in
    [0, alpha Q_0) (RMS about 2.1 Q_0 for alpha = 4), its centred form in (-alpha Q_0 / 2,
    alpha Q_0 / 2] (RMS about 0.58 Q_0).  The error shrinks by about that ratio."""
    from fides_b200 import params as P
    prm = P.chain(12, 60, 50, 7, 2, K=3)  # Q_0 about 2^210, P about 2^183
    plain, lifted = _keyswitch_error_rms(prm, False), _keyswitch_error_rms(prm, True)
    assert plain > 2.5 * lifted, (plain, lifted)
    assert lifted < 2.0 ** 45 < plain * 2 ** 10  # both well inside q_0 / 2


# ---------------------------------------------------------------- GPU parity
@pytest.fixture(scope="module")
def RN(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=True)
    o_plain = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=True)
    kg = KeyGen(o)
    rk = kg.relin_key()
    rot = {r: kg.rotation_key(r) for r in (1, -2, 128)}
    return dict(F=fides, prm=prm, o=o, o_plain=o_plain, ctx=ctx, rk=rk, rk_d=fides.to_device(rk), rot=rot,
                rot_d={r: fides.to_device(k) for r, k in rot.items()})


def _ct(prm, l, stream):
    rng = xrng(stream)
    return uniform_limbs(rng, prm.q[:l], prm.N), uniform_limbs(rng, prm.q[:l], prm.N)


def _eq(F, t, h):
    return np.array_equal(F.to_host(t), h)


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["tensor", "simt"])
@pytest.mark.parametrize("level", [30, 16, 6])
def test_reduced_noise_key_switching_equals_oracle(RN, engine, level):
    F, prm, o, ctx = RN["F"], RN["prm"], RN["o"], RN["ctx"]
    ctx.set_conv_engine(engine)
    try:
        x = _ct(prm, level, 3400 + level)[0]
        xd = F.to_device(x)
        dig = ctx.modup(xd)
        dig_ref = o.modup(x)
        assert _eq(F, dig, dig_ref)
        assert not _eq(F, dig, RN["o_plain"].modup(x))  # the lift fired
        a, b = ctx.ksk_inner_product(dig, level, RN["rk_d"])
        a_ref, b_ref = o.ksk_ip(dig_ref, level, RN["rk"])
        assert _eq(F, ctx.moddown(a), o.moddown(a_ref))
        a_c, b_c = _ct(prm, level, 3500 + level), _ct(prm, level, 3600 + level)
        out = ctx.mult(F.Ciphertext(F.to_device(a_c[0]), F.to_device(a_c[1])),
                       F.Ciphertext(F.to_device(b_c[0]), F.to_device(b_c[1])), RN["rk_d"], rescale=True)
        r0, r1 = o.hmult(*a_c, *b_c, RN["rk"], rescale=True)
        assert _eq(F, out.c0, r0) and _eq(F, out.c1, r1)
        ct = F.Ciphertext(F.to_device(a_c[0]), F.to_device(a_c[1]))
        rot = ctx.rotate(ct, RN["rot_d"][-2], -2)
        r0, r1 = o.rotate(*a_c, RN["rot"][-2], -2)
        assert _eq(F, rot.c0, r0) and _eq(F, rot.c1, r1)
        rs = [1, -2, 128]
        outs = ctx.rotate_hoisted(ct, [RN["rot_d"][r] for r in rs], rs)
        h0, h1 = o.rotate_hoisted(*a_c, [RN["rot"][r] for r in rs], rs)
        for k in range(len(rs)):
            assert _eq(F, outs[k].c0, h0[k]) and _eq(F, outs[k].c1, h1[k]), f"rotation {rs[k]}"
    finally:
        ctx.set_conv_engine("auto")


@pytest.mark.gpu
def test_reduced_noise_flag_switches_back(RN):
    """Turning the flag off restores the plain conversions on the same context."""
    F, prm, ctx = RN["F"], RN["prm"], RN["ctx"]
    x = _ct(prm, 20, 3700)[0]
    ctx.set_reduced_noise(False)
    try:
        assert _eq(F, ctx.modup(F.to_device(x)), RN["o_plain"].modup(x))
    finally:
        ctx.set_reduced_noise(True)
    assert _eq(F, ctx.modup(F.to_device(x)), RN["o"].modup(x))
    noK = F.Context(prm.logN, prm.q[:4], [], 1)
    with pytest.raises(F.FidesError):
        noK.set_reduced_noise(True)
