"""GPU tests of the pipelined host-buffer batches (fides_hmult_host_batch,
fides_rotate_host_batch): every item equals the one-call-per-op host path and the oracle,
at mixed levels and with more items than the pipeline's buffer slots."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o)
    rk = kg.relin_key()
    rot = {r: kg.rotation_key(r) for r in (1, -2)}
    return fides, prm, o, ctx, rk, rot


def host_ct(F, prm, l, stream):
    rng = xrng(stream)
    out = []
    for _ in range(2):
        a = F.pinned_empty((l, prm.N))
        a[:] = uniform_limbs(rng, prm.q[:l], prm.N)
        out.append(a)
    return out


def test_hmult_host_batch_matches_oracle(env):
    F, prm, o, ctx, rk, _ = env
    key = ctx.key_upload(rk)
    try:
        levels = [6, 3, 5, 6, 2, 4, 6]  # more items than the three pipeline slots
        items, refs = [], []
        for k, l in enumerate(levels):
            a, b = host_ct(F, prm, l, 500 + 2 * k), host_ct(F, prm, l, 501 + 2 * k)
            o0, o1 = F.pinned_empty((l - 1, prm.N)), F.pinned_empty((l - 1, prm.N))
            items.append((a[0], a[1], b[0], b[1], o0, o1))
            refs.append(o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True))
        ctx.mult_host_batch(items, key, True)
        for k, ((*_, o0, o1), (r0, r1)) in enumerate(zip(items, refs)):
            assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"item {k}"
        # the one-call-per-op host path gives the same residues
        s0, s1 = ctx.mult_host(*items[1][:4], key, True)
        assert np.array_equal(s0, refs[1][0]) and np.array_equal(s1, refs[1][1])
    finally:
        ctx.key_free(key)


def test_rotate_host_batch_matches_oracle(env):
    F, prm, o, ctx, _, rot = env
    keys = {r: ctx.key_upload(k) for r, k in rot.items()}
    try:
        spec = [(6, 1), (4, -2), (6, -2), (2, 1), (5, 1)]
        items, refs = [], []
        for k, (l, r) in enumerate(spec):
            c = host_ct(F, prm, l, 700 + k)
            o0, o1 = F.pinned_empty((l, prm.N)), F.pinned_empty((l, prm.N))
            items.append((c[0], c[1], o0, o1, keys[r], r))
            refs.append(o.rotate(c[0], c[1], rot[r], r))
        ctx.rotate_host_batch(items)
        for k, ((_, _, o0, o1, _, _), (r0, r1)) in enumerate(zip(items, refs)):
            assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"item {k}"
    finally:
        for v in keys.values():
            ctx.key_free(v)


def test_mixed_host_batch_matches_oracle(env):
    """HMults and rotations alternated in one pipeline (fides_mixed_host_batch), uneven counts
    and levels: every item equals the oracle."""
    F, prm, o, ctx, rk, rot = env
    key = ctx.key_upload(rk)
    keys = {r: ctx.key_upload(k) for r, k in rot.items()}
    try:
        hm, hrefs = [], []
        for k, l in enumerate([6, 4, 5]):
            a, b = host_ct(F, prm, l, 1500 + 2 * k), host_ct(F, prm, l, 1501 + 2 * k)
            o0, o1 = F.pinned_empty((l - 1, prm.N)), F.pinned_empty((l - 1, prm.N))
            hm.append((a[0], a[1], b[0], b[1], o0, o1))
            hrefs.append(o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True))
        rt, rrefs = [], []
        for k, (l, r) in enumerate([(6, 1), (3, -2), (5, 1), (6, -2), (2, 1)]):
            c = host_ct(F, prm, l, 1600 + k)
            o0, o1 = F.pinned_empty((l, prm.N)), F.pinned_empty((l, prm.N))
            rt.append((c[0], c[1], o0, o1, keys[r], r))
            rrefs.append(o.rotate(c[0], c[1], rot[r], r))
        ctx.mixed_host_batch(hm, key, rt, True)
        for k, ((*_, o0, o1), (r0, r1)) in enumerate(zip(hm, hrefs)):
            assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"hmult item {k}"
        for k, ((_, _, o0, o1, _, _), (r0, r1)) in enumerate(zip(rt, rrefs)):
            assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"rotate item {k}"
    finally:
        ctx.key_free(key)
        for v in keys.values():
            ctx.key_free(v)


def test_host_batch_rejects_bad_level(env):
    F, prm, o, ctx, rk, _ = env
    key = ctx.key_upload(rk)
    try:
        a = host_ct(F, prm, 1, 900)
        o0, o1 = F.pinned_empty((1, prm.N)), F.pinned_empty((1, prm.N))
        with pytest.raises(F.FidesError) as e:
            ctx.mult_host_batch([(a[0], a[1], a[0], a[1], o0, o1)], key, True)  # level 1 cannot rescale
        assert e.value.code == -4
        ctx.mult_host_batch([], key, True)  # empty batch: no-op
    finally:
        ctx.key_free(key)


def test_mixed_host_batch_async_continues_pipeline(env):
    """Calls that return once enqueued (fides_mixed_host_batch_async) continue one pipeline
    across calls: a later call with larger items grows the slots, a rejected call leaves the
    enqueued ones intact, and after fides_host_batch_wait every item equals the oracle."""
    F, prm, o, ctx, rk, rot = env
    key = ctx.key_upload(rk)
    keys = {r: ctx.key_upload(k) for r, k in rot.items()}
    try:
        calls = []  # per call: (hmult items, rotate items, references)
        for c, (hl, rl) in enumerate([([3, 2], [(2, 1)]), ([4], [(3, -2), (4, 1)]), ([6, 5], [(6, -2)])]):
            hm, rt, refs = [], [], []
            for k, l in enumerate(hl):
                a, b = host_ct(F, prm, l, 2500 + 10 * c + 2 * k), host_ct(F, prm, l, 2501 + 10 * c + 2 * k)
                o0, o1 = F.pinned_empty((l - 1, prm.N)), F.pinned_empty((l - 1, prm.N))
                hm.append((a[0], a[1], b[0], b[1], o0, o1))
                refs.append(((o0, o1), o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True)))
            for k, (l, r) in enumerate(rl):
                x = host_ct(F, prm, l, 2600 + 10 * c + k)
                o0, o1 = F.pinned_empty((l, prm.N)), F.pinned_empty((l, prm.N))
                rt.append((x[0], x[1], o0, o1, keys[r], r))
                refs.append(((o0, o1), o.rotate(x[0], x[1], rot[r], r)))
            calls.append((hm, rt, refs))
        ctx.mixed_host_batch(calls[0][0], key, calls[0][1], True, wait=False)
        ctx.mixed_host_batch(calls[1][0], key, calls[1][1], True, wait=False)
        bad = host_ct(F, prm, 1, 2700)
        b0, b1 = F.pinned_empty((1, prm.N)), F.pinned_empty((1, prm.N))
        with pytest.raises(F.FidesError) as e:  # level 1 cannot rescale: rejected before enqueueing
            ctx.mixed_host_batch([(bad[0], bad[1], bad[0], bad[1], b0, b1)], key, [], True, wait=False)
        assert e.value.code == -4
        ctx.mixed_host_batch(calls[2][0], key, calls[2][1], True, wait=False)  # larger slots
        ctx.host_batch_wait()
        for c, (_, _, refs) in enumerate(calls):
            for k, ((o0, o1), (r0, r1)) in enumerate(refs):
                assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"call {c} item {k}"
        # a waiting call after asynchronous ones continues the same slots
        hm, rt, refs = calls[1]
        for (o0, o1), _ in refs:
            o0[:] = 0
            o1[:] = 0
        ctx.mixed_host_batch(hm, key, rt, True)
        for k, ((o0, o1), (r0, r1)) in enumerate(refs):
            assert np.array_equal(o0, r0) and np.array_equal(o1, r1), f"repeat item {k}"
        ctx.host_batch_wait()  # nothing pending: returns at once
    finally:
        ctx.key_free(key)
        for v in keys.values():
            ctx.key_free(v)
