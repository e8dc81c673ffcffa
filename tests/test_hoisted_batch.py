"""GPU tests of batched hoisted rotations (fides_rotate_hoisted_batch): the scope of the
reference's key-switching benchmark -- 16 hoisted rotations by +-{1, 2, 4, ..., 128} at
levels 29, 15 and 5, several ciphertexts per launch sequence -- checked against the
single-ciphertext hoisted path and the oracle."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu

ROTS = [s * (1 << k) for k in range(8) for s in (1, -1)]  # +-1, +-2, ..., +-128


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=41)
    keys = {r: kg.rotation_key(r) for r in ROTS}
    keys_d = {r: fides.to_device(k) for r, k in keys.items()}
    return fides, prm, o, ctx, keys, keys_d


def ct(F, prm, l, stream):
    rng = xrng(stream)
    return [uniform_limbs(rng, prm.q[:l], prm.N) for _ in range(2)]


def test_batch_matches_single_and_oracle(env):
    F, prm, o, ctx, keys, keys_d = env
    levels = [29, 15, 5]
    host = [ct(F, prm, l, 1500 + l) for l in levels]
    dev = [F.Ciphertext(F.to_device(c[0]), F.to_device(c[1])) for c in host]
    outs = ctx.rotate_hoisted_batch(dev, [keys_d[r] for r in ROTS], ROTS)
    for c, res in zip(dev, outs):
        single = ctx.rotate_hoisted(c, [keys_d[r] for r in ROTS], ROTS)
        for a, b in zip(res, single):
            assert np.array_equal(F.to_host(a.c0), F.to_host(b.c0))
            assert np.array_equal(F.to_host(a.c1), F.to_host(b.c1))
    # oracle: the extreme rotations at the smallest level
    sub = [1, -128, 64]
    h0, h1 = o.rotate_hoisted(*host[2], [keys[r] for r in sub], sub)
    for j, r in enumerate(sub):
        k = ROTS.index(r)
        assert np.array_equal(F.to_host(outs[2][k].c0), h0[j])
        assert np.array_equal(F.to_host(outs[2][k].c1), h1[j])


def test_per_ciphertext_rotation_lists(env):
    """Items with their own (different-length) rotation lists, one of them empty."""
    F, prm, o, ctx, keys, keys_d = env
    host = [ct(F, prm, l, 1600 + l) for l in (6, 6, 9)]
    dev = [F.Ciphertext(F.to_device(c[0]), F.to_device(c[1])) for c in host]
    lists = [[1, 2, 4], [], [-8]]
    outs = ctx.rotate_hoisted_batch(dev, [[keys_d[r] for r in rs] for rs in lists], lists)
    assert [len(x) for x in outs] == [3, 0, 1]
    for c, rs, res in zip(host, lists, outs):
        if not rs:
            continue
        h0, h1 = o.rotate_hoisted(*c, [keys[r] for r in rs], rs)
        for j in range(len(rs)):
            assert np.array_equal(F.to_host(res[j].c0), h0[j])
            assert np.array_equal(F.to_host(res[j].c1), h1[j])


def test_batch_of_32_ciphertexts_level_29(env):
    """Config C's largest batch: 32 ciphertexts at level 29, the 16 rotations each, in one
    launch sequence (the KSK pass groups the ciphertexts that share a key, so each key tile is
    read once per group of 4).  Every output equals the single-ciphertext hoisted path; two
    ciphertexts are also checked against the oracle on three rotations."""
    F, prm, o, ctx, keys, keys_d = env
    host = [ct(F, prm, 29, 1700 + i) for i in range(32)]
    dev = [F.Ciphertext(F.to_device(c[0]), F.to_device(c[1])) for c in host]
    outs = ctx.rotate_hoisted_batch(dev, [keys_d[r] for r in ROTS], ROTS)
    assert len(outs) == 32 and all(len(x) == 16 for x in outs)
    for i in (0, 13, 31):
        single = ctx.rotate_hoisted(dev[i], [keys_d[r] for r in ROTS], ROTS)
        for a, b in zip(outs[i], single):
            assert np.array_equal(F.to_host(a.c0), F.to_host(b.c0))
            assert np.array_equal(F.to_host(a.c1), F.to_host(b.c1))
    sub = [2, -32, 128]
    for i in (7, 30):
        h0, h1 = o.rotate_hoisted(*host[i], [keys[r] for r in sub], sub)
        for j, r in enumerate(sub):
            k = ROTS.index(r)
            assert np.array_equal(F.to_host(outs[i][k].c0), h0[j])
            assert np.array_equal(F.to_host(outs[i][k].c1), h1[j])
