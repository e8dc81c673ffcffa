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
