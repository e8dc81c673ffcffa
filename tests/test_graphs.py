"""GPU test of CUDA-graph capture of library calls (fides_capture_* / fides_graph_*): a
captured batched HMult + HRotate step replays to the same residues as the direct calls."""
import numpy as np
import pytest
import torch

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def test_captured_step_replays_bit_exact(fides):
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=51)
    rk, k1 = fides.to_device(kg.relin_key()), fides.to_device(kg.rotation_key(1))
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    rng = xrng(52)
    levels = [6, 3, 5]
    cts = [fides.Ciphertext(fides.to_device(uniform_limbs(rng, prm.q[:l], prm.N)),
                            fides.to_device(uniform_limbs(rng, prm.q[:l], prm.N))) for l in levels for _ in range(2)]
    pairs = [(cts[2 * i], cts[2 * i + 1]) for i in range(len(levels))]
    want_m = ctx.mult_batch(pairs, rk, rescale=True)
    want_r = ctx.rotate_batch([(a, k1, 1) for a, _ in pairs])
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g = ctx.capture(s)
        with g:
            got_m = ctx.mult_batch(pairs, rk, rescale=True)
            got_r = ctx.rotate_batch([(a, k1, 1) for a, _ in pairs])
        for o_ in got_m + got_r:  # poison the outputs, then replay twice
            o_.c0.zero_()
            o_.c1.zero_()
        g.launch(s)
        g.launch(s)
    torch.cuda.synchronize()
    for w, x in zip(want_m + want_r, got_m + got_r):
        assert torch.equal(w.c0, x.c0) and torch.equal(w.c1, x.c1)
    g.close()
