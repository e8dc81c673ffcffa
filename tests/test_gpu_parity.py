"""GPU parity: every residue of the CUDA path (through the C ABI) equals the CPU oracle
on the same seeded inputs and keys.  Bit-exact: integer arithmetic only."""
import numpy as np
import pytest
import torch

import oracle as O
from ckks_host import KeyGen, decode, encode, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def eq(gpu_t, host):
    import fides_b200 as F
    return np.array_equal(F.to_host(gpu_t), host)


class Setup:
    def __init__(self, F, prm, keys=True, rot=()):
        self.prm = prm
        self.o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
        self.ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
        assert self.ctx.psi == self.o.psi
        self.F = F
        if keys:
            self.kg = KeyGen(self.o)
            self.rk = self.kg.relin_key()
            self.rk_d = F.to_device(self.rk)
            self.rot = {r: self.kg.rotation_key(r) for r in rot}
            self.rot_d = {r: F.to_device(k) for r, k in self.rot.items()}

    def rand_ct(self, l, stream):
        rng = xrng(stream)
        c0 = uniform_limbs(rng, self.prm.q[:l], self.o.N)
        c1 = uniform_limbs(rng, self.prm.q[:l], self.o.N)
        return c0, c1

    def dev_ct(self, c):
        return self.F.Ciphertext(self.F.to_device(c[0]), self.F.to_device(c[1]))


@pytest.fixture(scope="module")
def A(fides):
    from fides_b200 import params as P
    return Setup(fides, P.config_a(), rot=(1, -1, 5))


@pytest.fixture(scope="module")
def Cfg(fides):
    from fides_b200 import params as P
    return Setup(fides, P.config_c(4), rot=(1, -1, 2, 128, -128))


# ---------------------------------------------------------------- NTT (config B)
@pytest.mark.parametrize("batch", [1, 8])
def test_ntt_config_b_bit_exact(fides, batch):
    from fides_b200 import params as P
    prm = P.config_b()
    o = O.Oracle(16, prm.q, [], 1)
    ctx = fides.Context(16, prm.q, [], 1)
    rng = xrng(200 + batch)
    x = np.stack([uniform_limbs(rng, prm.q, o.N) for _ in range(batch)])
    d = fides.to_device(x)
    ctx.ntt(d)
    got = fides.to_host(d)
    ids = list(range(36))
    for b in range(batch):
        assert np.array_equal(got[b], o.ntt(x[b], ids)), f"poly {b}"
    ctx.intt(d)
    assert eq(d, x)


def test_ntt_config_b_batch64_roundtrip(fides):
    """Full 64-polynomial batch: INTT(NTT(x)) == x everywhere, and every 9th polynomial
    bit-exact against the oracle (size-independent check of the whole batch)."""
    from fides_b200 import params as P
    prm = P.config_b()
    o = O.Oracle(16, prm.q, [], 1)
    ctx = fides.Context(16, prm.q, [], 1)
    rng = xrng(264)
    x = np.stack([uniform_limbs(rng, prm.q, o.N) for _ in range(64)])
    d = fides.to_device(x)
    ctx.ntt(d)
    got = fides.to_host(d)
    for b in range(0, 64, 9):
        assert np.array_equal(got[b], o.ntt(x[b], list(range(36))))
    ctx.intt(d)
    assert eq(d, x)


@pytest.mark.parametrize("logN", [10, 11, 12, 13, 14, 15, 17])
def test_ntt_all_sizes(fides, logN):
    q = O.gen_primes(logN, 60, 1) + O.gen_primes(logN, 50, 2)
    o = O.Oracle(logN, q, [], 1)
    ctx = fides.Context(logN, q, [], 1)
    x = uniform_limbs(xrng(logN), q, o.N)
    d = fides.to_device(x)
    ctx.ntt(d)
    assert eq(d, o.ntt(x, [0, 1, 2]))
    ctx.intt(d)
    assert eq(d, x)


def test_ntt_uneven_limb_list(fides):
    """One launch over limbs of different primes and different polynomials."""
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    ids = [3, 0, 7, 7, 1, 8, 2]
    x = np.stack([xrng(i).integers(0, o.primes[p], o.N, dtype=np.uint64) for i, p in enumerate(ids)])
    ts = [fides.to_device(x[i]) for i in range(len(ids))]
    ctx.ntt_limbs(ts, ids)
    for i, p in enumerate(ids):
        assert eq(ts[i], o.ntt(x[i:i + 1], [p])[0])


def test_ntt_reference_primes(fides):
    """The reference's own NTT test moduli (p64 / sp64, up to 62 bits)."""
    import json, os
    from conftest import GOLDEN
    rp = json.load(open(os.path.join(GOLDEN, "ref_params.json")))
    q = rp["p64"][:6] + rp["sp64"][:3]
    for logN in (13, 16):
        o = O.Oracle(logN, q, [], 1)
        ctx = fides.Context(logN, q, [], 1)
        x = uniform_limbs(xrng(77), q, o.N)
        d = fides.to_device(x)
        ctx.ntt(d)
        assert eq(d, o.ntt(x, list(range(len(q)))))
        ctx.intt(d)
        assert eq(d, x)


# ---------------------------------------------------------------- key switching pieces
@pytest.mark.parametrize("level", [30, 16, 6])
def test_modup_ksk_moddown_config_c(Cfg, level):
    F, o = Cfg.F, Cfg.o
    x = Cfg.rand_ct(level, 300 + level)[0]
    xd = F.to_device(x)
    dig = Cfg.ctx.modup(xd)
    dig_ref = o.modup(x)
    assert eq(dig, dig_ref)
    a, b = Cfg.ctx.ksk_inner_product(dig, level, Cfg.rk_d)
    a_ref, b_ref = o.ksk_ip(dig_ref, level, Cfg.rk)
    assert eq(a, a_ref) and eq(b, b_ref)
    assert eq(Cfg.ctx.moddown(a), o.moddown(a_ref))
    f0, f1 = Cfg.ctx.keyswitch(xd, Cfg.rk_d)
    g0, g1 = o.keyswitch(x, Cfg.rk)
    assert eq(f0, g0) and eq(f1, g1)


def test_moddown_of_scaled_input_is_identity(Cfg):
    """ModDown(P * x) == x exactly: special limbs are zero (size-independent property)."""
    F, o, l = Cfg.F, Cfg.o, 30
    x = Cfg.rand_ct(l, 31)[0]
    Pm = []
    for q in Cfg.prm.q[:l]:
        v = 1
        for p in Cfg.prm.p:
            v = v * p % q
        Pm.append(v)
    ext = np.zeros((l + Cfg.prm.K, o.N), dtype=np.uint64)
    ext[:l] = o.mul(x, np.array([[v] * o.N for v in Pm], dtype=np.uint64), list(range(l)))
    assert eq(Cfg.ctx.moddown(F.to_device(ext)), x)


# ---------------------------------------------------------------- ciphertext ops
@pytest.mark.parametrize("level", [30, 16, 6, 2])
def test_rescale(Cfg, level):
    x = Cfg.rand_ct(level, 400 + level)[0]
    assert eq(Cfg.ctx.rescale_poly(Cfg.F.to_device(x)), Cfg.o.rescale(x))


@pytest.mark.parametrize("rescale", [True, False])
def test_hmult_config_a(A, rescale):
    a, b = A.rand_ct(6, 1), A.rand_ct(6, 2)
    out = A.ctx.mult(A.dev_ct(a), A.dev_ct(b), A.rk_d, rescale=rescale)
    r0, r1 = A.o.hmult(*a, *b, A.rk, rescale=rescale)
    assert eq(out.c0, r0) and eq(out.c1, r1)


@pytest.mark.parametrize("level", [30, 16, 6])
def test_hmult_config_c(Cfg, level):
    a, b = Cfg.rand_ct(level, 10 + level), Cfg.rand_ct(level, 20 + level)
    out = Cfg.ctx.mult(Cfg.dev_ct(a), Cfg.dev_ct(b), Cfg.rk_d, rescale=True)
    r0, r1 = Cfg.o.hmult(*a, *b, Cfg.rk, rescale=True)
    assert eq(out.c0, r0) and eq(out.c1, r1)


@pytest.mark.parametrize("r", [1, -1, 5])
def test_rotate_config_a(A, r):
    c = A.rand_ct(6, 50 + r)
    out = A.ctx.rotate(A.dev_ct(c), A.rot_d[r], r)
    r0, r1 = A.o.rotate(*c, A.rot[r], r)
    assert eq(out.c0, r0) and eq(out.c1, r1)


def test_conjugate_config_a(A):
    c = A.rand_ct(6, 60)
    k = 2 * A.o.N - 1
    key = A.kg.auto_key(k)
    out = A.ctx.rotate_auto(A.dev_ct(c), A.F.to_device(key), k)
    r0, r1 = A.o.rotate_auto(*c, key, k)
    assert eq(out.c0, r0) and eq(out.c1, r1)


@pytest.mark.parametrize("level", [30, 16, 6])
def test_rotate_config_c(Cfg, level):
    c = Cfg.rand_ct(level, 70 + level)
    out = Cfg.ctx.rotate(Cfg.dev_ct(c), Cfg.rot_d[1], 1)
    r0, r1 = Cfg.o.rotate(*c, Cfg.rot[1], 1)
    assert eq(out.c0, r0) and eq(out.c1, r1)


@pytest.mark.parametrize("level", [16, 6])
def test_hoisted_config_c(Cfg, level):
    c = Cfg.rand_ct(level, 80 + level)
    rs = [1, -1, 2, 128, -128]
    outs = Cfg.ctx.rotate_hoisted(Cfg.dev_ct(c), [Cfg.rot_d[r] for r in rs], rs)
    h0, h1 = Cfg.o.rotate_hoisted(*c, [Cfg.rot[r] for r in rs], rs)
    for j in range(len(rs)):
        assert eq(outs[j].c0, h0[j]) and eq(outs[j].c1, h1[j])


def test_batched_mixed_levels_equal_singles(Cfg):
    """One batched launch sequence over uneven levels == per-op results == oracle."""
    levels = [30, 7, 16, 2, 23]
    pairs = [(Cfg.dev_ct(Cfg.rand_ct(l, 500 + l)), Cfg.dev_ct(Cfg.rand_ct(l, 600 + l))) for l in levels]
    outs = Cfg.ctx.mult_batch(pairs, Cfg.rk_d, rescale=True)
    for (a, b), o in zip(pairs, outs):
        s = Cfg.ctx.mult(a, b, Cfg.rk_d, rescale=True)
        assert torch.equal(s.c0, o.c0) and torch.equal(s.c1, o.c1)
    l = 7
    a, b = Cfg.rand_ct(l, 500 + l), Cfg.rand_ct(l, 600 + l)
    r0, r1 = Cfg.o.hmult(*a, *b, Cfg.rk, rescale=True)
    assert eq(outs[1].c0, r0) and eq(outs[1].c1, r1)
    jobs = [(Cfg.dev_ct(Cfg.rand_ct(l, 700 + l)), Cfg.rot_d[r], r) for l, r in zip(levels, [1, -1, 2, 128, -128])]
    routs = Cfg.ctx.rotate_batch(jobs)
    for (ct, key, r), o in zip(jobs, routs):
        s = Cfg.ctx.rotate(ct, key, r)
        assert torch.equal(s.c0, o.c0) and torch.equal(s.c1, o.c1)


def test_host_entry_points(Cfg):
    l = 16
    a, b = Cfg.rand_ct(l, 900), Cfg.rand_ct(l, 901)
    key = Cfg.ctx.key_upload(Cfg.rk)
    try:
        o0, o1 = Cfg.ctx.mult_host(*a, *b, key, rescale=True)
        r0, r1 = Cfg.o.hmult(*a, *b, Cfg.rk, rescale=True)
        assert np.array_equal(o0, r0) and np.array_equal(o1, r1)
    finally:
        Cfg.ctx.key_free(key)
    rk = Cfg.ctx.key_upload(Cfg.rot[2])
    try:
        o0, o1 = Cfg.ctx.rotate_host(*a, rk, 2)
        r0, r1 = Cfg.o.rotate(*a, Cfg.rot[2], 2)
        assert np.array_equal(o0, r0) and np.array_equal(o1, r1)
    finally:
        Cfg.ctx.key_free(rk)


@pytest.mark.parametrize("terms,level", [(1, 30), (15, 17), (16, 30), (32, 5)])
def test_dot_plain_config_c(Cfg, terms, level):
    """The fused plaintext inner product of a linear transform's giant step equals the
    oracle's sum of elementwise products, residue for residue (1 term, the 15-term reduction
    boundary, one past it, and the 32-term maximum)."""
    ids = list(range(level))
    cts = [Cfg.rand_ct(level, 1000 + t) for t in range(terms)]
    pts = [uniform_limbs(xrng(1100 + t), Cfg.prm.q[:level], Cfg.o.N) for t in range(terms)]
    ref = [None, None]
    for (c0, c1), pt in zip(cts, pts):
        for k, c in enumerate((c0, c1)):
            m = Cfg.o.mul(c, pt, ids)
            ref[k] = m if ref[k] is None else Cfg.o.add(ref[k], m, ids)
    got = Cfg.ctx.dot_plain([Cfg.dev_ct(c) for c in cts], [Cfg.F.to_device(p) for p in pts])
    assert eq(got.c0, ref[0]) and eq(got.c1, ref[1])


@pytest.mark.parametrize("terms,level", [(1, 30), (15, 17), (16, 5)])
def test_lincomb_config_c(Cfg, terms, level):
    """sum_t s_t * ct_t + add0 with per-limb integer constants equals the oracle's products
    and sums residue for residue (add0 on c0 only)."""
    N, q = Cfg.o.N, Cfg.prm.q[:level]
    ids = list(range(level))
    rng = xrng(1200 + terms)
    cts = [Cfg.rand_ct(level, 1300 + t) for t in range(terms)]
    scal = [[int(rng.integers(0, qi)) for qi in q] for _ in range(terms)]
    add = [int(rng.integers(0, qi)) for qi in q]
    bc = lambda v: np.repeat(np.array(v, dtype=np.uint64)[:, None], N, axis=1)
    ref = [bc(add), np.zeros((level, N), dtype=np.uint64)]
    for (c0, c1), sv in zip(cts, scal):
        ref = [Cfg.o.add(ref[k], Cfg.o.mul(c, bc(sv), ids), ids) for k, c in enumerate((c0, c1))]
    got = Cfg.ctx.lincomb([Cfg.dev_ct(c) for c in cts], scal, add0=add, level=level)
    assert eq(got.c0, ref[0]) and eq(got.c1, ref[1])


def test_lincomb_lanes_and_rescale_batch(Cfg):
    """Lanes of one combination launch equal the combination run lane by lane, and a batched
    rescale of polynomials at mixed levels equals the oracle's rescale of each."""
    F, l = Cfg.F, 12
    rng = xrng(1400)
    lanes = [[Cfg.dev_ct(Cfg.rand_ct(l, 1410 + 4 * a + t)) for t in range(4)] for a in range(3)]
    scal = [[int(rng.integers(0, qi)) for qi in Cfg.prm.q[:l]] for _ in range(4)]
    outs = Cfg.ctx.lincomb_lanes(lanes, scal, add0=7, level=l)
    for lane, o in zip(lanes, outs):
        one = Cfg.ctx.lincomb(lane, scal, add0=7, level=l)
        assert torch.equal(one.c0, o.c0) and torch.equal(one.c1, o.c1)
    polys = [Cfg.rand_ct(lv, 1450 + lv)[0] for lv in (30, 17, 2)]
    got = Cfg.ctx.rescale_many([F.to_device(x) for x in polys])
    for x, g in zip(polys, got):
        assert eq(g, Cfg.o.rescale(x))


def test_dot_plain_rejects_bad_terms(Cfg):
    c = Cfg.dev_ct(Cfg.rand_ct(4, 2))
    with pytest.raises(Cfg.F.FidesError):
        Cfg.ctx.dot_plain([c] * 33, [c.c0] * 33)


def test_error_statuses(Cfg):
    F = Cfg.F
    c = Cfg.dev_ct(Cfg.rand_ct(4, 1))
    with pytest.raises(F.FidesError) as e:
        Cfg.ctx.mult(c, c, None)
    assert e.value.code == -5
    bad = F.Ciphertext(Cfg.ctx.empty(31), Cfg.ctx.empty(31))
    with pytest.raises(F.FidesError) as e:
        Cfg.ctx.rotate(bad, Cfg.rot_d[1], 1)
    assert e.value.code == -4
    Cfg.ctx.set_scratch_limit(1 << 20)
    try:
        with pytest.raises(F.FidesError) as e:
            Cfg.ctx.mult(c, c, Cfg.rk_d)
        assert e.value.code == -3
    finally:
        Cfg.ctx.set_scratch_limit(0)
    out = Cfg.ctx.mult(c, c, Cfg.rk_d)  # context still usable
    assert out.level == 3


def test_decrypt_valid_config_c_k9(fides):
    """K = 9 (reference sizing rule): results decrypt to the FP64 product / rotation."""
    from fides_b200 import params as P
    s = Setup(fides, P.config_c(9), rot=(1,))
    N, D, l = s.o.N, 2.0 ** 50, 30
    rng = xrng(33)
    z1 = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    z2 = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    c = s.kg.encrypt(encode(z1, N, D).astype(np.int64), l)
    d = s.kg.encrypt(encode(z2, N, D).astype(np.int64), l)
    out = s.ctx.mult(s.dev_ct(c), s.dev_ct(d), s.rk_d, rescale=True)
    got = decode(s.kg.decrypt_limb0(fides.to_host(out.c0), fides.to_host(out.c1)), N, D * D / s.prm.q[l - 1])
    assert np.abs(got - z1 * z2).max() < 1e-6
    rot = s.ctx.rotate(s.dev_ct(c), s.rot_d[1], 1)
    got = decode(s.kg.decrypt_limb0(fides.to_host(rot.c0), fides.to_host(rot.c1)), N, D)
    assert np.abs(got - np.roll(z1, -1)).max() < 1e-6


@pytest.mark.parametrize("level", [30, 16, 6])
def test_elementwise_kernels_config_c(Cfg, level):
    """tensor_kernel (fides_tensor, the binomialMult_ counterpart), addsub_kernel's add / sub /
    mul and scalar_kernel's mul / add against the oracle, residue for residue (config C)."""
    F, o, ctx = Cfg.F, Cfg.o, Cfg.ctx
    ids = list(range(level))
    a, b = Cfg.rand_ct(level, 3100 + level), Cfg.rand_ct(level, 3200 + level)
    d = ctx.tensor(Cfg.dev_ct(a), Cfg.dev_ct(b))
    torch.cuda.synchronize()
    for got, want in zip(d, o.tensor(a[0], a[1], b[0], b[1])):
        assert eq(got, want)
    A, B = F.to_device(a[0]), F.to_device(b[1])
    assert eq(ctx.add_poly(A, B), o.add(a[0], b[1], ids))
    assert eq(ctx.sub_poly(A, B), o.sub(a[0], b[1], ids))
    assert eq(ctx.sub_poly(B, A), o.sub(b[1], a[0], ids))
    assert eq(ctx.mul_poly(A, B), o.mul(a[0], b[1], ids))
    # in place (out aliases an input)
    C = F.to_device(a[0])
    ctx.mul_poly(C, B, out=C)
    assert eq(C, o.mul(a[0], b[1], ids))
    sc = [int(v) % Cfg.prm.q[j] for j, v in enumerate(xrng(3300 + level).integers(0, 2**62, level))]
    sc[0] = Cfg.prm.q[0] - 1
    scal = np.array([[v] * Cfg.o.N for v in sc], dtype=np.uint64)
    assert eq(ctx.mul_scalar_poly(A, sc), o.mul(a[0], scal, ids))
    assert eq(ctx.add_scalar_poly(A, sc), o.add(a[0], scal, ids))


@pytest.mark.gpu
def test_mixed_batch_equals_separate_batches_and_oracle(fides):
    """fides_mixed_batch: HMults (rescaled and not) and rotations at uneven levels in one launch
    sequence equal fides_hmult_batch / fides_rotate_batch item for item, and the oracle."""
    import torch
    from fides_b200 import params as P
    F = fides
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=91)
    rk = kg.relin_key()
    keys = {r: kg.rotation_key(r) for r in (1, -3)}
    rk_d = F.to_device(rk)
    keys_d = {r: F.to_device(k) for r, k in keys.items()}
    rng = xrng(4500)
    hl, rl = [30, 9, 17], [6, 30, 12, 21]
    hcts = [[uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(4)] for l in hl]
    rcts = [[uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)] for l in rl]
    dev = lambda c: F.Ciphertext(F.to_device(c[0]), F.to_device(c[1]))
    pairs = [(dev(h[:2]), dev(h[2:])) for h in hcts]
    rsel = [1, -3, 1, -3]
    rots = [(dev(c), keys_d[r], r) for c, r in zip(rcts, rsel)]
    for rescale in (True, False):
        mh, mr = ctx.mixed_batch(pairs, rk_d, rots, rescale=rescale)
        sh = ctx.mult_batch(pairs, rk_d, rescale=rescale)
        sr = ctx.rotate_batch(rots)
        torch.cuda.synchronize()
        for a, b in zip(mh + mr, sh + sr):
            assert torch.equal(a.c0, b.c0) and torch.equal(a.c1, b.c1)
        for h, out in zip(hcts[:2], mh[:2]):
            w0, w1 = o.hmult(*h, rk, rescale=rescale)
            assert np.array_equal(F.to_host(out.c0), w0) and np.array_equal(F.to_host(out.c1), w1)
    for c, r, out in list(zip(rcts, rsel, mr))[:2]:
        w0, w1 = o.rotate(c[0], c[1], keys[r], r)
        assert np.array_equal(F.to_host(out.c0), w0) and np.array_equal(F.to_host(out.c1), w1)
    # only one kind, and neither
    mh, mr = ctx.mixed_batch(pairs[:1], rk_d, [], rescale=True)
    assert len(mh) == 1 and mr == []
    mh, mr = ctx.mixed_batch([], rk_d, rots[:1])
    assert mh == [] and len(mr) == 1
    assert ctx.mixed_batch([], rk_d, []) == ([], [])
    with pytest.raises(F.FidesError):  # HMults need the relinearisation key
        ctx.mixed_batch(pairs[:1], None, [])
