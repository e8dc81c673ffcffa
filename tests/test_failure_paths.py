"""GPU tests of the failure paths, with every failure made on the host (no kernel is made to
fault, trap or hang):

  * the device status word -> FIDES_ERR_TIMEOUT mapping: the status bit a bounded
    device-side wait sets when it gives up is written from the host
    (fides_ctx_inject_status), and every synchronising call must then fail with
    FIDES_ERR_TIMEOUT until the status is cleared, after which the context works again;
  * the bounded server wait: fides_server_wait_timeout returns FIDES_ERR_TIMEOUT for a
    request still queued behind others, and the ticket stays valid.

The reference has no bounded device waits; its errors surface from CudaCheckErrorMod after a
synchronisation (src/CudaUtils.cuh:706-757), which is the role the status check plays here."""
import numpy as np
import pytest
import torch

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu

TIMEOUT = -6


def test_status_word_maps_to_timeout_until_cleared(fides):
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o)
    rk = kg.relin_key()
    key = ctx.key_upload(rk)
    rng = xrng(7101)
    a = [uniform_limbs(rng, prm.q, o.N) for _ in range(4)]
    want = o.hmult(a[0], a[1], a[2], a[3], rk, rescale=True)

    ctx.synchronize()  # clean context: no error
    ctx.inject_status(1)  # as conv_tc_kernel's bounded mbarrier wait does when it gives up
    with pytest.raises(fides.FidesError) as e:
        ctx.synchronize()
    assert e.value.code == TIMEOUT
    with pytest.raises(fides.FidesError) as e:  # a host entry point synchronises, then checks
        ctx.mult_host(a[0], a[1], a[2], a[3], key)
    assert e.value.code == TIMEOUT
    with pytest.raises(fides.FidesError) as e:  # sticky until cleared
        ctx.synchronize()
    assert e.value.code == TIMEOUT

    assert ctx.device_status(clear=True) & 1
    assert ctx.device_status(clear=False) == 0
    ctx.synchronize()
    r0, r1 = ctx.mult_host(a[0], a[1], a[2], a[3], key)
    assert np.array_equal(r0, want[0]) and np.array_equal(r1, want[1])
    # bit 1 (encode overflow) is reported but is not a timeout
    ctx.inject_status(2)
    ctx.synchronize()
    assert ctx.device_status(clear=True) == 2
    ctx.key_free(key)


def test_server_wait_timeout_leaves_ticket_valid(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=93)
    rk = fides.to_device(kg.relin_key())
    srv = fides.Server(ctx, n_streams=1, max_batch=1)
    srv.set_relin_key(rk)
    rng = xrng(7102)
    x = [fides.to_device(uniform_limbs(rng, prm.q, prm.N)) for _ in range(2)]
    a = fides.Ciphertext(x[0], x[1])
    outs = [fides.Ciphertext(ctx.empty(29), ctx.empty(29)) for _ in range(40)]
    # 40 top-level HMults, one per batch on one stream: the last is queued behind ~40 key
    # switches (milliseconds of work) when its wait starts
    tickets = [srv.submit(fides.OP_HMULT, a, outs[i], b=a) for i in range(40)]
    with pytest.raises(fides.FidesError) as e:
        srv.wait(tickets[-1], timeout_ms=0.0)
    assert e.value.code == TIMEOUT
    for t in tickets:
        st, _ = srv.wait(t, timeout_ms=60000.0)
        assert st == 0
    torch.cuda.synchronize()
    for out in outs[1:]:
        assert torch.equal(out.c0, outs[0].c0) and torch.equal(out.c1, outs[0].c1)
    srv.close()
