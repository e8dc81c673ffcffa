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
