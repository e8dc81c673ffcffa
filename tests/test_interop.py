"""Interop with the reference's raw host formats (fides_ct_import / fides_ct_export /
fides_key_import): per-limb host arrays in EVALUATION (bit-reversed or natural order) or
COEFFICIENT format land in the library's layout bit-exactly, and export is the inverse
(Ciphertext::load / store, src/CKKS/Ciphertext.cpp:415-464; RawCipherText with REV = 1 / 0,
src/CKKS/openfhe-interface/RawCiphertext.cu:57-96)."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    return prm, O.Oracle(prm.logN, prm.q, prm.p, prm.dnum), fides.Context(prm.logN, prm.q, prm.p, prm.dnum)


def brev_perm(logN):
    idx = np.arange(1 << logN)
    r = np.zeros_like(idx)
    for b in range(logN):
        r |= ((idx >> b) & 1) << (logN - 1 - b)
    return r


@pytest.mark.parametrize("level", [30, 34, 3])
def test_import_eval_coeff_natural(fides, C, level):
    import torch
    prm, o, ctx = C
    primes = (prm.q + prm.p)[:level]
    ids = list(range(level))
    polys = [uniform_limbs(xrng(2500 + level + k), primes, prm.N) for k in range(2)]
    ev = ctx.import_limbs([list(p) for p in polys])
    assert torch.equal(ev, fides.to_device(np.stack(polys)))
    co = ctx.import_limbs([list(p) for p in polys], format_coeff=True)
    for k in range(2):
        assert np.array_equal(fides.to_host(co[k]), o.ntt(polys[k], ids))
    perm = brev_perm(prm.logN)
    nat = ctx.import_limbs([[limb[perm] for limb in p] for p in polys], natural_order=True)
    assert torch.equal(nat, ev)
    for fc in (False, True):
        for no in (False, True):
            back = ctx.export_limbs(ev, format_coeff=fc, natural_order=no)
            for k in range(2):
                exp = o.ntt(polys[k], ids, inverse=True) if fc else polys[k]
                if no:
                    exp = exp[:, perm]
                assert np.array_equal(np.stack(back[k]), exp), (fc, no)


def test_import_rejects_wrong_moduli(fides, C):
    prm, o, ctx = C
    p = uniform_limbs(xrng(2600), prm.q[:2], prm.N)
    with pytest.raises(fides.FidesError):
        ctx.import_limbs([list(p)], moduli=[prm.q[1], prm.q[0]])


def test_key_import_equals_upload(fides, C):
    """A key imported from per-limb arrays (bit-reversed, or natural order with zero limbs
    given as None) acts exactly like the same key uploaded flat: relinearisation at level 30
    reads every limb of every digit."""
    import torch
    prm, o, ctx = C
    kg = KeyGen(o, seed_stream=77)
    rk = kg.relin_key()  # [2][dnum][n_q + K][N]
    ext = prm.n_q + prm.K
    perm = brev_perm(prm.logN)
    a = fides.Ciphertext(fides.to_device(uniform_limbs(xrng(2601), prm.q, prm.N)),
                         fides.to_device(uniform_limbs(xrng(2602), prm.q, prm.N)))
    zeroed = rk.copy()
    zeroed[:, :, 5] = 0
    keys = []
    try:
        keys.append(ctx.import_key([[[rk[x, d, i] for i in range(ext)] for d in range(prm.dnum)] for x in range(2)]))
        keys.append(ctx.key_upload(rk))
        keys.append(ctx.import_key([[[None if i == 5 else rk[x, d, i][perm] for i in range(ext)]
                                     for d in range(prm.dnum)] for x in range(2)], natural_order=True))
        keys.append(ctx.key_upload(zeroed))
        r = [ctx.mult(a, a, k, rescale=True) for k in keys]
        assert torch.equal(r[0].c0, r[1].c0) and torch.equal(r[0].c1, r[1].c1)
        assert torch.equal(r[2].c0, r[3].c0) and torch.equal(r[2].c1, r[3].c1)
        assert not torch.equal(r[0].c0, r[2].c0)
    finally:
        for k in keys:
            ctx.key_free(k)
