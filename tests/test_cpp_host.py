"""GPU test of the C++ host API (fideslib-fork_b200/host/FIDESlibB200.hpp): the compiled
program drives Context / KeySwitchingKey / Ciphertext calls shaped like the reference's
CKKS classes through the C ABI; every residue it stores is compared with the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, uniform_limbs, xrng
from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("reduced_noise", [False, True])
def test_cpp_host_api_matches_oracle(fides, tmp_path, reduced_noise):
    """reduced_noise: Parameters::reducedNoise set on the C++ side, the oracle's flag likewise."""
    from fides_b200 import params as P
    pkg = os.path.join(ROOT, "fideslib-fork_b200")
    subprocess.run(["make", "-s", "-C", pkg, "host_test"], check=True)
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum, reduced_noise=reduced_noise)
    kg = KeyGen(o, seed_stream=71)
    rot = 3
    rk, kr = kg.relin_key(), kg.rotation_key(rot)
    l, N = prm.n_q, prm.N
    rng = xrng(72)
    a = [uniform_limbs(rng, prm.q, N) for _ in range(2)]
    b = [uniform_limbs(rng, prm.q, N) for _ in range(2)]
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        np.array([prm.logN, prm.n_q, prm.K, prm.dnum, l, rot], dtype=np.uint64).tofile(f)
        np.array(prm.q + prm.p, dtype=np.uint64).tofile(f)
        for arr in (rk, kr, a[0], a[1], b[0], b[1]):
            np.ascontiguousarray(arr, dtype=np.uint64).tofile(f)
    r = subprocess.run([os.path.join(pkg, "host_test"), str(inp), str(outp)] + (["rn"] if reduced_noise else []),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr + r.stdout
    data = np.fromfile(outp, dtype=np.uint64)
    pos = 0
    got = []
    for _ in range(6):
        n = int(data[pos])
        pos += 1
        c0 = data[pos:pos + n * N].reshape(n, N)
        pos += n * N
        c1 = data[pos:pos + n * N].reshape(n, N)
        pos += n * N
        got.append((c0, c1))
    ids = list(range(l))
    want = [
        o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True),
        (o.add(a[0], b[0], ids), o.add(a[1], b[1], ids)),
        o.rotate(a[0], a[1], kr, rot),
        o.rotate(a[0], a[1], kr, rot),
    ]
    f0, f1 = o.keyswitch(a[1], rk)
    want.append((o.add(a[0], f0, ids), f1))
    want.append((o.rescale(a[0]), o.rescale(a[1])))
    names = ["mult+rescale", "add", "rotate", "rotate_hoisted", "keySwitch", "rescale"]
    for name, (g0, g1), (w0, w1) in zip(names, got, want):
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), name
