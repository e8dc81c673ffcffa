"""GPU parity of the tensor-core basis conversion (tcgen05 INT8-split product).

ModUp / ModDown / key switching / HMult / rotation with the conversion forced onto the
tensor cores must equal the CPU oracle (ApproxSwitchCRTBasis of the reference,
src/Conv.cu:27-423) and the 64-bit SIMT engine residue for residue, including at the
extremes of the byte-plane sums (every residue q - 1) and for odd destination counts
(padded B rows)."""
import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng

pytestmark = pytest.mark.gpu


def eq(gpu_t, host):
    import fides_b200 as F
    return np.array_equal(F.to_host(gpu_t), host)


class Env:
    def __init__(self, F, prm):
        self.F, self.prm = F, prm
        self.o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
        self.ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
        self.ctx.set_conv_engine("tensor")
        self.kg = KeyGen(self.o)
        self.rk = self.kg.relin_key()
        self.rk_d = F.to_device(self.rk)

    def rand(self, l, stream):
        return uniform_limbs(xrng(stream), self.prm.q[:l], self.o.N)


@pytest.fixture(scope="module")
def C(fides):
    from fides_b200 import params as P
    return Env(fides, P.config_c(4))


@pytest.fixture(scope="module")
def Boot(fides):
    """The bootstrap bench's chain: N=2^16, L+1 = 24, dnum 3, K 7 (K = 8 n_src not a
    multiple of 32 on the ModDown side)."""
    from fides_b200 import params as P
    return Env(fides, P.chain(16, 60, 50, 24, 3, K=7))


@pytest.mark.parametrize("level", [30, 29, 16, 5, 1])
def test_modup_moddown_tensor_equals_oracle(C, level):
    x = C.rand(level, 900 + level)
    dig = C.ctx.modup(C.F.to_device(x))
    dig_ref = C.o.modup(x)
    assert eq(dig, dig_ref)
    ext = uniform_limbs(xrng(950 + level), C.prm.q[:level] + C.prm.p, C.o.N)
    assert eq(C.ctx.moddown(C.F.to_device(ext)), C.o.moddown(ext))
    assert C.ctx.device_status() == 0


@pytest.mark.parametrize("level", [24, 23, 9])
def test_modup_moddown_tensor_k7(Boot, level):
    x = Boot.rand(level, 700 + level)
    assert eq(Boot.ctx.modup(Boot.F.to_device(x)), Boot.o.modup(x))
    ext = uniform_limbs(xrng(750 + level), Boot.prm.q[:level] + Boot.prm.p, Boot.o.N)
    assert eq(Boot.ctx.moddown(Boot.F.to_device(ext)), Boot.o.moddown(ext))
    assert Boot.ctx.device_status() == 0


def test_extreme_residues(C):
    """Every residue q - 1: the largest byte-plane sums the pre-scaled inputs allow."""
    level = 30
    qs = C.prm.q[:level] + C.prm.p
    x = np.array([[q - 1] * C.o.N for q in C.prm.q[:level]], dtype=np.uint64)
    assert eq(C.ctx.modup(C.F.to_device(x)), C.o.modup(x))
    ext = np.array([[q - 1] * C.o.N for q in qs], dtype=np.uint64)
    assert eq(C.ctx.moddown(C.F.to_device(ext)), C.o.moddown(ext))


@pytest.mark.parametrize("level", [30, 17])
def test_keyswitch_hmult_tensor(C, level):
    F = C.F
    x = C.rand(level, 960 + level)
    f0, f1 = C.ctx.keyswitch(F.to_device(x), C.rk_d)
    g0, g1 = C.o.keyswitch(x, C.rk)
    assert eq(f0, g0) and eq(f1, g1)
    a = (C.rand(level, 970), C.rand(level, 971))
    b = (C.rand(level, 972), C.rand(level, 973))
    out = C.ctx.mult(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])),
                     F.Ciphertext(F.to_device(b[0]), F.to_device(b[1])), C.rk_d, rescale=True)
    r0, r1 = C.o.hmult(*a, *b, C.rk, rescale=True)
    assert eq(out.c0, r0) and eq(out.c1, r1)


def test_engines_agree_on_rotation_batch(C):
    """Rotations of a mixed-level batch: tensor engine == SIMT engine."""
    F = C.F
    key = F.to_device(C.kg.rotation_key(3))
    cts = [F.Ciphertext(F.to_device(C.rand(l, 980 + l)), F.to_device(C.rand(l, 990 + l))) for l in (30, 21, 8)]
    outs = {}
    for eng in ("simt", "tensor"):
        C.ctx.set_conv_engine(eng)
        outs[eng] = [C.ctx.rotate(ct, key, 3) for ct in cts]
    C.ctx.set_conv_engine("tensor")
    for s, t in zip(outs["simt"], outs["tensor"]):
        assert np.array_equal(F.to_host(s.c0), F.to_host(t.c0))
        assert np.array_equal(F.to_host(s.c1), F.to_host(t.c1))
    assert C.ctx.device_status() == 0
