"""GPU test of fides_rescale_noalloc, the rescale entry point that allocates no device
memory.  It exists for callers that cannot allocate on the call path -- a host whose HBM
is entirely reserved by another allocator, or a latency-bound loop that cannot take the
synchronisation of cudaMalloc / cudaFree -- and takes its one limb of scratch from a
static array in the library.  It must give exactly what fides_rescale gives, call after
call, and refuse the ring sizes and buffer layouts it does not support.

Collected last on purpose (file name), so that a failure here leaves every other test run.
"""
import numpy as np
import pytest
import torch

from ckks_host import uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def test_noalloc_rescale_matches_rescale_on_consecutive_calls(fides):
    import oracle as O
    from fides_b200 import params as P
    prm = P.config_c(4)  # N = 2^16: the largest ring the static scratch holds
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    # consecutive calls; the third repeats the first input, the last leaves one output limb
    cases = [(30, 4401), (17, 4402), (30, 4401), (2, 4405)]
    free = []
    for level, seed in cases:
        xh = uniform_limbs(xrng(seed), prm.q[:level], prm.N)
        x = fides.to_device(xh)
        want = ctx.rescale_poly(x)
        got = ctx.empty(level - 1)
        torch.cuda.synchronize()
        before = torch.cuda.mem_get_info()[0]
        ctx.rescale_poly_noalloc(x, got)
        torch.cuda.synchronize()
        free.append((before, torch.cuda.mem_get_info()[0]))
        assert torch.equal(got, want), f"level {level}: differs from fides_rescale"
        if level in (17, 2):
            assert np.array_equal(fides.to_host(got), o.rescale(xh)), f"level {level}: differs from the oracle"
    # after the first call (which may load the module), calls leave device memory untouched
    for before, after in free[1:]:
        assert before == after
    assert ctx.scratch_bytes == 0
    assert torch.cuda.current_device() == 0


def test_noalloc_rescale_refuses_unsupported_inputs(fides):
    from fides_b200 import params as P
    import oracle as O
    prm = P.config_a()
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    x = fides.to_device(uniform_limbs(xrng(4403), prm.q, prm.N))
    with pytest.raises(fides.FidesError) as e:
        ctx.rescale_poly_noalloc(x, x[:5])  # output overlapping the input
    assert e.value.code == -1
    q17 = O.gen_primes(17, 50, 3)
    big = fides.Context(17, q17, [], 1)
    xb = fides.to_device(uniform_limbs(xrng(4404), q17, 1 << 17))
    with pytest.raises(fides.FidesError) as e:
        big.rescale_poly_noalloc(xb, big.empty(2))  # ring larger than the static scratch
    assert e.value.code == -1 and "2^16" in str(e.value)
