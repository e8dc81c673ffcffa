"""GPU tests of the NTT tile shapes and their autotuner (fides_ctx_autotune).

Every shape (4, 8 or 16 sub-transforms per CTA) only regroups the same butterflies, so the
transforms and the fused key-switch / rescale paths built on them must stay bit-exact
against the oracle whatever the shape table holds -- forced shapes, and the autotuned one."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def eq(gpu_t, host):
    import fides_b200 as F
    return np.array_equal(F.to_host(gpu_t), host)


def force(ctx, g):
    for inv in (0, 1):
        for p in (0, 1):
            for cls in range(4):
                ctx.set_ntt_shape(inv, p, cls, g)


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o)
    rk = kg.relin_key()
    return fides, prm, o, ctx, rk, fides.to_device(rk)


@pytest.mark.parametrize("g", [4, 8, 16])
@pytest.mark.parametrize("limbs", [3, 20, 40])
def test_forced_shapes_ntt(env, g, limbs):
    F, prm, o, ctx, _, _ = env
    force(ctx, g)
    allq = prm.q + prm.p
    ids = [i % len(allq) for i in range(limbs)]
    x = uniform_limbs(xrng(1000 + limbs), [allq[i] for i in ids], prm.N)
    d = F.to_device(x)
    ctx.ntt_limbs([d[i] for i in range(limbs)], ids)
    assert eq(d, o.ntt(x, ids))
    ctx.ntt_limbs([d[i] for i in range(limbs)], ids, inverse=True)
    assert eq(d, x)


@pytest.mark.parametrize("g", [4, 8])
def test_forced_shapes_hmult(env, g):
    F, prm, o, ctx, rk, rk_d = env
    force(ctx, g)
    l = 12
    rng = xrng(1200 + g)
    a = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    b = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    out = ctx.mult(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])),
                   F.Ciphertext(F.to_device(b[0]), F.to_device(b[1])), rk_d, rescale=True)
    r0, r1 = o.hmult(*a, *b, rk, rescale=True)
    assert eq(out.c0, r0) and eq(out.c1, r1)


def test_autotune_table_and_parity(env):
    F, prm, o, ctx, rk, rk_d = env
    rep = ctx.autotune()
    shapes = rep["shapes"]
    for d in ("forward", "inverse"):
        for p in ("column", "row"):
            assert len(shapes[d][p]) == 4 and all(g in (4, 8, 16) for g in shapes[d][p])
    assert all(t > 0 for t in rep["transform_ms"]["forward"] + rep["transform_ms"]["inverse"])
    l = 30
    rng = xrng(1300)
    a = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    b = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    out = ctx.mult(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])),
                   F.Ciphertext(F.to_device(b[0]), F.to_device(b[1])), rk_d, rescale=True)
    r0, r1 = o.hmult(*a, *b, rk, rescale=True)
    assert eq(out.c0, r0) and eq(out.c1, r1)


def test_bad_shape_rejected(env):
    F, _, _, ctx, _, _ = env
    for args in ((0, 0, 0, 5), (2, 0, 0, 8), (0, 2, 0, 8), (0, 0, 4, 8)):
        with pytest.raises(F.FidesError) as e:
            ctx.set_ntt_shape(*args)
        assert e.value.code == -1


@pytest.mark.parametrize("chunk", [7, 56, 0])
def test_chunked_launches_equal_oracle(env, chunk):
    """A limb list longer than the chunk size runs as balanced chunks (both passes of a chunk
    back to back); the transforms and a batched HMult built on them stay bit-exact."""
    F, prm, o, ctx, rk, rk_d = env
    old = ctx.ntt_chunk()
    try:
        assert ctx.ntt_chunk(chunk) == (chunk or 448)
        polys = 4
        x = np.stack([uniform_limbs(xrng(4100 + i), prm.q, prm.N) for i in range(polys)])  # 120 limbs
        d = F.to_device(x)
        ctx.ntt(d)
        got = F.to_host(d)
        for i in range(polys):
            assert np.array_equal(got[i], o.ntt(x[i], list(range(prm.n_q)))), f"poly {i}"
        ctx.intt(d)
        assert eq(d, x)
        a = [uniform_limbs(xrng(4200 + i), prm.q, prm.N) for i in range(4)]
        out = ctx.mult_batch([(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])),
                               F.Ciphertext(F.to_device(a[2]), F.to_device(a[3])))], rk_d, rescale=True)[0]
        w0, w1 = o.hmult(a[0], a[1], a[2], a[3], rk, rescale=True)
        assert eq(out.c0, w0) and eq(out.c1, w1)
    finally:
        ctx.ntt_chunk(old)
