"""GPU tests of the NTT tile shapes and their autotuner (fides_ctx_autotune).

Every shape (4, 8 or 16 sub-transforms per CTA) and residues per thread (16, or 8: three
butterfly stages per register chunk) only regroup the same butterflies, so the transforms
and the fused key-switch / rescale paths built on them must stay bit-exact against the
oracle whatever the tables hold -- forced entries, and the autotuned ones."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def eq(gpu_t, host):
    import fides_b200 as F
    return np.array_equal(F.to_host(gpu_t), host)


def force(ctx, g, r=16):
    for inv in (0, 1):
        for p in (0, 1):
            for cls in range(4):
                ctx.set_ntt_shape(inv, p, cls, g)
                ctx.set_ntt_residues(inv, p, cls, r)


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o)
    rk = kg.relin_key()
    return fides, prm, o, ctx, rk, fides.to_device(rk)


@pytest.mark.parametrize("r", [16, 8])
@pytest.mark.parametrize("g", [4, 8, 16])
@pytest.mark.parametrize("limbs", [3, 20, 40])
def test_forced_shapes_ntt(env, g, limbs, r):
    F, prm, o, ctx, _, _ = env
    force(ctx, g, r)
    allq = prm.q + prm.p
    ids = [i % len(allq) for i in range(limbs)]
    x = uniform_limbs(xrng(1000 + limbs), [allq[i] for i in ids], prm.N)
    d = F.to_device(x)
    ctx.ntt_limbs([d[i] for i in range(limbs)], ids)
    assert eq(d, o.ntt(x, ids))
    ctx.ntt_limbs([d[i] for i in range(limbs)], ids, inverse=True)
    assert eq(d, x)


@pytest.mark.parametrize("r", [16, 8])
@pytest.mark.parametrize("g", [4, 8])
def test_forced_shapes_hmult(env, g, r):
    F, prm, o, ctx, rk, rk_d = env
    force(ctx, g, r)
    l = 12
    rng = xrng(1200 + g)
    a = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    b = [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]
    out = ctx.mult(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])),
                   F.Ciphertext(F.to_device(b[0]), F.to_device(b[1])), rk_d, rescale=True)
    r0, r1 = o.hmult(*a, *b, rk, rescale=True)
    assert eq(out.c0, r0) and eq(out.c1, r1)


@pytest.fixture(scope="module")
def rot_keys(env):
    F, prm, o, _, _, _ = env
    kg = KeyGen(o, seed_stream=9)
    rot = {s: kg.rotation_key(s) for s in (1, -4)}
    return rot, {s: F.to_device(k) for s, k in rot.items()}


@pytest.mark.parametrize("r", [8, 16])
@pytest.mark.parametrize("level", [30, 7])
def test_forced_residues_every_fused_pass(env, rot_keys, r, level):
    """Every prologue / epilogue variant of the passes with the forced residues per thread:
    HMult with and without rescale (a1 b1 prologue, ModDown + rescale epilogue, conv +
    P SwitchModulus prologue, special-limb epilogue), rotation (ModDown epilogue), rescale
    (SwitchModulus prologue, rescale epilogue), hoisted rotations and a key switch."""
    F, prm, o, ctx, rk, rk_d = env
    force(ctx, 8, r)
    try:
        rot, rot_d = rot_keys
        rng = xrng(5100 + level + r)
        a = [uniform_limbs(rng, prm.q[:level], prm.N) for _ in range(2)]
        b = [uniform_limbs(rng, prm.q[:level], prm.N) for _ in range(2)]
        A = F.Ciphertext(F.to_device(a[0]), F.to_device(a[1]))
        B = F.Ciphertext(F.to_device(b[0]), F.to_device(b[1]))
        for rs in (True, False):
            out = ctx.mult(A, B, rk_d, rescale=rs)
            r0, r1 = o.hmult(*a, *b, rk, rescale=rs)
            assert eq(out.c0, r0) and eq(out.c1, r1), f"hmult rescale={rs}"
        out = ctx.rotate(A, rot_d[1], 1)
        r0, r1 = o.rotate(*a, rot[1], 1)
        assert eq(out.c0, r0) and eq(out.c1, r1)
        assert eq(ctx.rescale_poly(F.to_device(a[0])), o.rescale(a[0]))
        outs = ctx.rotate_hoisted(A, [rot_d[1], rot_d[-4]], [1, -4])
        h0, h1 = o.rotate_hoisted(*a, [rot[1], rot[-4]], [1, -4])
        for k in range(2):
            assert eq(outs[k].c0, h0[k]) and eq(outs[k].c1, h1[k])
        f0, f1 = ctx.keyswitch(F.to_device(a[1]), rk_d)
        g0, g1 = o.keyswitch(a[1], rk)
        assert eq(f0, g0) and eq(f1, g1)
    finally:
        force(ctx, 16, 16)


def test_autotune_table_and_parity(env):
    F, prm, o, ctx, rk, rk_d = env
    rep = ctx.autotune()
    shapes = rep["shapes"]
    for d in ("forward", "inverse"):
        for p in ("column", "row"):
            assert len(shapes[d][p]) == 4 and all(g in (4, 8, 16) for g in shapes[d][p])
            assert all(r in (8, 16) for r in rep["residues_per_thread"][d][p])
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
    for args in ((0, 0, 0, 12), (2, 0, 0, 8), (0, 0, 4, 16)):
        with pytest.raises(F.FidesError) as e:
            ctx.set_ntt_residues(*args)
        assert e.value.code == -1
    from fides_b200 import params as P
    pa = P.config_a()  # N = 2^13: only 16 residues per thread are built
    small = F.Context(pa.logN, pa.q, pa.p, pa.dnum)
    with pytest.raises(F.FidesError):
        small.set_ntt_residues(0, 0, 0, 8)
    small.set_ntt_residues(0, 0, 0, 16)


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
