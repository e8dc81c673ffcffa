"""The measurement harness of the reference's own GPU NTT kernels (baseline/ref_kernels) is
valid: on the same primes, root and inputs, the reference kernels' forward and inverse
transforms equal this project's NTT residue for residue (and the oracle's).  The harness is
built from the reference sources, so it is skipped where it was not built."""
import os
import sys

import numpy as np
import pytest

import oracle as O
from ckks_host import uniform_limbs, xrng

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "baseline", "ref_kernels"))
import ref_kernels as R  # noqa: E402

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference kernel harness not built")]


@pytest.mark.parametrize("logN", [16, 13])
def test_reference_ntt_equals_ours(fides, logN):
    import torch
    from fides_b200 import params as P
    q = P.gen_primes(logN, 60, 8)
    ctx = fides.Context(logN, q, [], 1)
    R.init(logN, q, ctx.psi)
    N = 1 << logN
    polys, limbs = 2, len(q)
    x = np.stack([uniform_limbs(xrng(1700 + i), q, N) for i in range(polys)])
    ours = fides.to_device(x)
    ref = fides.to_device(x)
    aux = torch.empty_like(ref)
    ctx.ntt(ours)
    s = torch.cuda.current_stream().cuda_stream
    R.ntt(ref, aux, polys, limbs, False, s)
    torch.cuda.synchronize()
    assert torch.equal(ours, ref)
    o = O.Oracle(logN, q, [], 1)
    assert np.array_equal(fides.to_host(ours)[0], o.ntt(x[0], list(range(limbs))))
    ctx.intt(ours)
    R.ntt(ref, aux, polys, limbs, True, s)
    torch.cuda.synchronize()
    assert torch.equal(ours, ref)
    assert np.array_equal(fides.to_host(ref), x)


@pytest.mark.parametrize("level", [30, 17, 5])
def test_reference_conversions_equal_oracle(fides, level):
    """The reference's ModUp (DecompAndModUpConv) and ModDown (ModDown2) conversions, driven
    by the harness, equal the oracle's ApproxSwitchCRTBasis (config C: N=2^16, 30 Q limbs,
    dnum 3, 4 special primes)."""
    import torch
    from fides_b200 import params as P
    prm = P.config_c(4)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    R.init(prm.logN, prm.q + prm.p, ctx.psi, K=prm.K, dnum=prm.dnum)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    N = prm.N
    x = uniform_limbs(xrng(1800 + level), prm.q[:level], N)
    xd = fides.to_device(x)
    s = torch.cuda.current_stream().cuda_stream
    alpha = -(-prm.n_q // prm.dnum)
    for d in range(-(-level // alpha)):
        lo, hi = d * alpha, min(level, (d + 1) * alpha)
        dst = R.modup_dst(d)
        out = torch.zeros((len(dst), N), dtype=torch.int64, device="cuda").view(torch.uint64)
        R.modup(xd, level, d, out, s)
        torch.cuda.synchronize()
        got = fides.to_host(out)
        active = [j for j, pid in enumerate(dst) if pid < level or pid >= prm.n_q]
        ref = o.switch_basis(x[lo:hi], list(range(lo, hi)), [dst[j] for j in active])
        assert np.array_equal(got[active], ref), f"digit {d}"
    sp = uniform_limbs(xrng(1900 + level), prm.p, N)
    out = torch.empty((level, N), dtype=torch.int64, device="cuda").view(torch.uint64)
    R.moddown(fides.to_device(sp), level, out, s)
    torch.cuda.synchronize()
    ref = o.switch_basis(sp, list(range(prm.n_q, prm.n_q + prm.K)), list(range(level)))
    assert np.array_equal(fides.to_host(out), ref)


@pytest.mark.parametrize("level", [30, 17, 5])
def test_reference_reduced_noise_conversions_equal_oracle(fides, level):
    """With the reference's reduced_noise flag (Parameters::reducedNoise, read by
    DecompAndModUpConv and ModDown2), its conversions equal the oracle's lifted conversion and
    differ from the plain one; this project's ModUp with the flag equals the oracle too."""
    import torch
    from fides_b200 import params as P
    prm = P.config_c(4)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=True)
    R.init(prm.logN, prm.q + prm.p, ctx.psi, K=prm.K, dnum=prm.dnum)
    R.set_reduced_noise(True)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=True)
    N = prm.N
    x = uniform_limbs(xrng(2800 + level), prm.q[:level], N)
    xd = fides.to_device(x)
    s = torch.cuda.current_stream().cuda_stream
    alpha = -(-prm.n_q // prm.dnum)
    for d in range(-(-level // alpha)):
        lo, hi = d * alpha, min(level, (d + 1) * alpha)
        dst = R.modup_dst(d)
        out = torch.zeros((len(dst), N), dtype=torch.int64, device="cuda").view(torch.uint64)
        R.modup(xd, level, d, out, s)
        torch.cuda.synchronize()
        got = fides.to_host(out)
        active = [j for j, pid in enumerate(dst) if pid < level or pid >= prm.n_q]
        ids = [dst[j] for j in active]
        ref = o.switch_basis(x[lo:hi], list(range(lo, hi)), ids, lift=True)
        assert np.array_equal(got[active], ref), f"digit {d}"
        assert not np.array_equal(ref, o.switch_basis(x[lo:hi], list(range(lo, hi)), ids))
    sp = uniform_limbs(xrng(2900 + level), prm.p, N)
    out = torch.empty((level, N), dtype=torch.int64, device="cuda").view(torch.uint64)
    R.moddown(fides.to_device(sp), level, out, s)
    torch.cuda.synchronize()
    ref = o.switch_basis(sp, list(range(prm.n_q, prm.n_q + prm.K)), list(range(level)), lift=True)
    assert np.array_equal(fides.to_host(out), ref)
    R.set_reduced_noise(False)
    # the whole ModUp of this project with the flag (INTT, lifted conversion, NTT)
    x_eval = o.ntt(x, list(range(level)))
    assert np.array_equal(fides.to_host(ctx.modup(fides.to_device(x_eval))), o.modup(x_eval))


# ---------------------------------------------------------------- key switching, automorphism,
# SwitchModulus, tensor and elementwise kernels of the reference, against the oracle and ours
def _config_c(fides):
    import torch
    from fides_b200 import params as P
    prm = P.config_c(4)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    R.init(prm.logN, prm.q + prm.p, ctx.psi, K=prm.K, dnum=prm.dnum)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    return prm, ctx, o, torch.cuda.current_stream().cuda_stream


def _rand_key(prm, seed):
    """A [2][dnum][n_q + K][N] array of uniform residues: the inner products are linear, so
    residue parity needs no valid key."""
    rng = xrng(seed)
    return np.stack([np.stack([uniform_limbs(rng, prm.q + prm.p, prm.N) for _ in range(prm.dnum)])
                     for _ in range(2)])


@pytest.mark.parametrize("level", [30, 16, 6])
def test_reference_ksk_inner_product_equals_oracle_and_ours(fides, level):
    """fusedDotKSK_2_ (ElemenwiseBatchKernels.cu:202-274) over the reference's digit pointer
    tables = the oracle's KSK inner product = ours (ksk_kernel), residue for residue."""
    import torch
    prm, ctx, o, s = _config_c(fides)
    x = uniform_limbs(xrng(2100 + level), prm.q[:level], prm.N)
    key = _rand_key(prm, 2200 + level)
    kd = fides.to_device(key)
    digits = ctx.modup(fides.to_device(x))
    ext = level + prm.K
    ra = torch.zeros((ext, prm.N), dtype=torch.int64, device="cuda").view(torch.uint64)
    rb = torch.zeros_like(ra)
    R.ksk(digits, level, kd, ra, rb, s)
    oa, ob = ctx.ksk_inner_product(digits, level, kd)
    torch.cuda.synchronize()
    wa, wb = o.ksk_ip(fides.to_host(digits), level, key)
    assert np.array_equal(fides.to_host(ra), wa) and np.array_equal(fides.to_host(rb), wb)
    assert torch.equal(oa, ra) and torch.equal(ob, rb)


@pytest.mark.parametrize("level", [30, 16, 6])
def test_reference_hoisted_ksk_equals_oracle(fides, level):
    """hoistedRotateDotKSK_2_ (ElemenwiseBatchKernels.cu:277-377): per rotation r,
    out0 = sigma_k(sum_d D_d b_(r,d) + P c0), out1 = sigma_k(sum_d D_d a_(r,d)) over Q and special
    limbs; the oracle's inner product, P c0 and automorphism give the same residues."""
    import torch
    prm, ctx, o, s = _config_c(fides)
    rng = xrng(2300 + level)
    c0 = uniform_limbs(rng, prm.q[:level], prm.N)
    c1 = uniform_limbs(rng, prm.q[:level], prm.N)
    rots = [1, -2, 128]
    keys = [_rand_key(prm, 2400 + 10 * level + i) for i in range(len(rots))]
    ks = [O.rotation_auto_index(prm.logN, r) for r in rots]
    kd = [fides.to_device(k) for k in keys]
    digits = ctx.modup(fides.to_device(c1))
    c0d = fides.to_device(c0)
    ext = level + prm.K
    z = lambda: torch.zeros((ext, prm.N), dtype=torch.int64, device="cuda").view(torch.uint64)
    out0, out1 = [z() for _ in rots], [z() for _ in rots]
    R.hoisted_ksk(digits, c0d, level, kd, ks, out0, out1, s)
    torch.cuda.synchronize()
    dh = fides.to_host(digits)
    P = [1] * level
    for p in prm.p:
        P = [P[j] * p % prm.q[j] for j in range(level)]
    Pc0 = o.mul(c0, np.array([[P[j]] * prm.N for j in range(level)], dtype=np.uint64), list(range(level)))
    for i, k in enumerate(ks):
        wa, wb = o.ksk_ip(dh, level, keys[i])
        wb[:level] = o.add(wb[:level], Pc0, list(range(level)))
        assert np.array_equal(fides.to_host(out1[i]), o.automorph(wa, k)), f"a side, rotation {rots[i]}"
        assert np.array_equal(fides.to_host(out0[i]), o.automorph(wb, k)), f"b side, rotation {rots[i]}"


def test_reference_automorph_and_switch_modulus_equal_oracle(fides):
    """automorph_ (Rotation.cu:10-12) and SwitchModulus (Rescale.cu:8-13) equal the oracle's
    restatements, on every kind of prime pair the rescale and ModRaise use."""
    import torch
    prm, ctx, o, s = _config_c(fides)
    x = uniform_limbs(xrng(2500), prm.q[:1], prm.N)[0]
    xd = fides.to_device(x)
    out = torch.empty_like(xd)
    for r in (1, -1, 5, 128, -128):
        k = O.rotation_auto_index(prm.logN, r)
        R.automorph(xd, out, k, s)
        torch.cuda.synchronize()
        assert np.array_equal(fides.to_host(out), o.automorph(x[None, :], k)[0]), f"rotation {r}"
    k = 2 * prm.N - 1  # conjugation
    R.automorph(xd, out, k, s)
    torch.cuda.synchronize()
    assert np.array_equal(fides.to_host(out), o.automorph(x[None, :], k)[0])
    n_q = prm.n_q
    for src, dst in ((29, 0), (29, 5), (0, 7), (0, n_q), (n_q + 1, 0), (3, 12)):
        xs = uniform_limbs(xrng(2600 + src), [(prm.q + prm.p)[src]], prm.N)[0]
        xs[:4] = [0, 1, (prm.q + prm.p)[src] // 2, (prm.q + prm.p)[src] // 2 + 1]  # around the centring threshold
        xsd = fides.to_device(xs)
        R.switch_modulus(xsd, src, out, dst, s)
        torch.cuda.synchronize()
        assert np.array_equal(fides.to_host(out), o.switch_modulus(xs, src, dst)), f"{src} -> {dst}"


@pytest.mark.parametrize("level", [30, 16, 6])
def test_reference_tensor_and_elementwise_equal_oracle_and_ours(fides, level):
    """binomialMult_ (ElemenwiseBatchKernels.cu:1363-1398), add_ / sub_ / scalar_add_
    (AddSub.cu:31-111) and mult_ / scalar_mult_ (ModMult.cu:8-21) against the oracle and
    this library's fides_tensor / fides_add / fides_sub / fides_mul / fides_mul_scalar /
    fides_add_scalar on the same inputs."""
    import torch
    prm, ctx, o, s = _config_c(fides)
    ids = list(range(level))
    rng = xrng(2700 + level)
    a0, a1, b0, b1 = (uniform_limbs(rng, prm.q[:level], prm.N) for _ in range(4))
    # tensor product
    c0, c1, d0, d1 = (fides.to_device(v) for v in (a0, a1, b0, b1))
    c2 = torch.empty_like(c0)
    R.tensor(c0, c1, c2, d0, d1, level, s)
    ours = ctx.tensor(fides.Ciphertext(fides.to_device(a0), fides.to_device(a1)),
                      fides.Ciphertext(fides.to_device(b0), fides.to_device(b1)))
    torch.cuda.synchronize()
    want = o.tensor(a0, a1, b0, b1)
    for got, mine, w in zip((c0, c1, c2), ours, want):
        assert np.array_equal(fides.to_host(got), w)
        assert torch.equal(mine, got)
    # elementwise with a second polynomial
    A, B = fides.to_device(a0), fides.to_device(b0)
    for op, mine, w in (("add", ctx.add_poly(A, B), o.add(a0, b0, ids)),
                        ("sub", ctx.sub_poly(A, B), o.sub(a0, b0, ids)),
                        ("mul", ctx.mul_poly(A, B), o.mul(a0, b0, ids))):
        r = fides.to_device(a0)
        R.elementwise(op, r, B, level, s)
        torch.cuda.synchronize()
        assert np.array_equal(fides.to_host(r), w), op
        assert torch.equal(mine, r), op
    # per-limb scalars (reduced residues), including 0, 1 and q - 1
    sc = [int(v) for v in xrng(2800 + level).integers(0, 2**62, level)]
    sc[0], sc[-1] = 1, 0
    if level > 2:
        sc[1] = prm.q[1] - 1
    sc = [v % prm.q[j] for j, v in enumerate(sc)]
    scal = np.array([[v] * prm.N for v in sc], dtype=np.uint64)
    for op, mine, w in (("mul_scalar", ctx.mul_scalar_poly(A, sc), o.mul(a0, scal, ids)),
                        ("add_scalar", ctx.add_scalar_poly(A, sc), o.add(a0, scal, ids))):
        r = fides.to_device(a0)
        R.elementwise(op, r, None, level, s, scalars=sc)
        torch.cuda.synchronize()
        assert np.array_equal(fides.to_host(r), w), op
        assert torch.equal(mine, r), op
