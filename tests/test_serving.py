"""GPU tests of the continuous-batching request loop (fides_server_*).

Model: the reference's ConcurrentOpsTests (test/ConcurrentOpsTests.cu:246-420) -- every
request's result must be bit-identical whether it runs alone or mixed with others that
arrive while it is on the GPU; admission by HBM budget must queue, not fail, requests that
fit, and reject those that never can."""
import random
import threading
import time

import numpy as np
import pytest
import torch

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


class Env:
    def __init__(self, F, prm, rots):
        self.F, self.prm = F, prm
        self.o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
        self.ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
        kg = KeyGen(self.o, seed_stream=91)
        self.rk = F.to_device(kg.relin_key())
        self.rot = {r: F.to_device(kg.rotation_key(r)) for r in rots}

    def ct(self, level, seed):
        rng = xrng(seed)
        return self.F.Ciphertext(self.F.to_device(uniform_limbs(rng, self.prm.q[:level], self.prm.N)),
                                 self.F.to_device(uniform_limbs(rng, self.prm.q[:level], self.prm.N)))

    def server(self, **kw):
        s = self.F.Server(self.ctx, **kw)
        s.set_relin_key(self.rk)
        for r, k in self.rot.items():
            s.add_rotation_key(r, k)
        return s

    def requests(self, n, seed, levels):
        rnd = random.Random(seed)
        F = self.F
        out = []
        for i in range(n):
            l = rnd.choice(levels)
            kind = rnd.choices([F.OP_HMULT, F.OP_HMULT_NORESCALE, F.OP_ROTATE], [5, 1, 4])[0]
            a = self.ct(l, seed * 1000 + 2 * i)
            b = self.ct(l, seed * 1000 + 2 * i + 1) if kind != F.OP_ROTATE else None
            r = rnd.choice(list(self.rot)) if kind == F.OP_ROTATE else 0
            lo = l - 1 if kind == F.OP_HMULT else l
            out.append(dict(op=kind, a=a, b=b, rotation=r, level=lo))
        return out

    def alloc_out(self, req):
        return self.F.Ciphertext(self.ctx.empty(req["level"]), self.ctx.empty(req["level"]))


def run_alone(env, srv, reqs):
    res = []
    for q in reqs:
        out = env.alloc_out(q)
        t = srv.submit(q["op"], q["a"], out, q["b"], q["rotation"])
        st, _ = srv.wait(t)
        assert st == 0
        res.append(out)
    return res


def run_mixed(env, srv, reqs, threads=3, max_gap_us=300):
    outs = [env.alloc_out(q) for q in reqs]
    tickets = [None] * len(reqs)
    order = list(range(len(reqs)))
    random.Random(5).shuffle(order)
    chunks = [order[i::threads] for i in range(threads)]

    def worker(k, idx):
        rnd = random.Random(k)
        for i in idx:
            q = reqs[i]
            tickets[i] = srv.submit(q["op"], q["a"], outs[i], q["b"], q["rotation"])
            time.sleep(rnd.random() * max_gap_us * 1e-6)

    ts = [threading.Thread(target=worker, args=(k, c)) for k, c in enumerate(chunks)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    lat = []
    for t in tickets:
        st, l = srv.wait(t)
        assert st == 0
        lat.append(l)
    return outs, lat


@pytest.mark.parametrize("max_inflight", [0, 1])
def test_alone_equals_mixed_config_a(fides, max_inflight):
    """max_inflight = 1: at most one batch per operation type on the device, so requests that
    arrive meanwhile form the next batch (batches grow under load); results are unchanged."""
    from fides_b200 import params as P
    env = Env(fides, P.config_a(), rots=(1, -1, 2))
    reqs = env.requests(40, seed=3, levels=[2, 3, 4, 5, 6])
    srv = env.server(n_streams=3, max_batch=6)
    srv.set_max_inflight(max_inflight)
    try:
        alone = run_alone(env, srv, reqs)
        mixed, lat = run_mixed(env, srv, reqs)
        stats = srv.stats()
    finally:
        srv.close()
    for i, (x, y) in enumerate(zip(alone, mixed)):
        assert torch.equal(x.c0, y.c0) and torch.equal(x.c1, y.c1), f"request {i}"
    assert stats["completed"] == 80 and stats["rejected"] == 0
    assert stats["batches"] < stats["completed"]  # the mix was actually batched
    # the served results are the library's single-op results
    q = reqs[0]
    if q["op"] == fides.OP_ROTATE:
        d = env.ctx.rotate(q["a"], env.rot[q["rotation"]], q["rotation"])
    else:
        d = env.ctx.mult(q["a"], q["b"], env.rk, rescale=q["op"] == fides.OP_HMULT)
    assert torch.equal(d.c0, alone[0].c0) and torch.equal(d.c1, alone[0].c1)


def test_alone_equals_mixed_config_c(fides):
    from fides_b200 import params as P
    env = Env(fides, P.config_c(4), rots=(1, 2))
    reqs = env.requests(12, seed=4, levels=list(range(5, 31)))
    srv = env.server(n_streams=2, max_batch=4)
    try:
        alone = run_alone(env, srv, reqs)
        mixed, lat = run_mixed(env, srv, reqs)
    finally:
        srv.close()
    for i, (x, y) in enumerate(zip(alone, mixed)):
        assert torch.equal(x.c0, y.c0) and torch.equal(x.c1, y.c1), f"request {i}"
    assert all(l > 0 for l in lat)


def test_budget_admission(fides):
    from fides_b200 import params as P
    env = Env(fides, P.config_a(), rots=(1,))
    reqs = env.requests(10, seed=6, levels=[6])
    limb = 8 * env.prm.N
    # room for about one request at a time: everything completes, serialised by memory
    srv = env.server(n_streams=4, max_batch=8, hbm_budget_bytes=100 * limb)
    try:
        outs, _ = run_mixed(env, srv, reqs, threads=2, max_gap_us=0)
        st = srv.stats()
        assert st["completed"] == 10 and st["rejected"] == 0
        assert st["peak_bytes"] <= 100 * limb
    finally:
        srv.close()
    # a budget smaller than any request: rejected with OOM, the server stays usable
    srv = env.server(n_streams=1, max_batch=2, hbm_budget_bytes=limb)
    try:
        out = env.alloc_out(reqs[0])
        t = srv.submit(reqs[0]["op"], reqs[0]["a"], out, reqs[0]["b"], reqs[0]["rotation"])
        st, _ = srv.wait(t)
        assert st == -3
        assert srv.stats()["rejected"] == 1
    finally:
        srv.close()


def test_submit_rejects_malformed_requests(fides):
    from fides_b200 import params as P
    env = Env(fides, P.config_a(), rots=(1,))
    srv = env.server(n_streams=1, max_batch=1)
    try:
        a = env.ct(4, 1)
        out = env.alloc_out(dict(level=4))
        with pytest.raises(fides.FidesError) as e:
            srv.submit(fides.OP_ROTATE, a, out, None, rotation=7)  # no key for 7
        assert e.value.code == -5
        with pytest.raises(fides.FidesError) as e:
            srv.submit(fides.OP_HMULT, a, out, None)  # missing second operand
        assert e.value.code == -1
    finally:
        srv.close()
