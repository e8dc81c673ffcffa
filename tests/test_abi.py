"""CPU checks of the C-ABI library: it builds for sm_100a, loads, exports every entry
point include/fides_b200.h declares, and rejects bad arguments before touching a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fides_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fides_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def libpath():
    import fides_b200
    return fides_b200.build()


def test_exports_every_declared_symbol(libpath):
    names = declared()
    assert len(names) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (fides_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = C.CDLL(libpath)
    for n in names:
        getattr(L, n)


def test_build_targets_sm100a():
    """The library's build recipe compiles for sm_100a only (the runtime check of the loaded
    code is test_kernels_loaded_as_sm100 below)."""
    mk = open(os.path.join(ROOT, "fideslib-fork_b200", "Makefile")).read()
    arch = re.search(r"^ARCH\s*:=\s*(.*)$", mk, re.M).group(1)
    assert arch.split() == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_kernels_loaded_as_sm100(fides):
    """cudaFuncAttributes::binaryVersion of a library kernel on the GPU: sm_100 code."""
    assert fides.kernel_arch(0) == 100


def test_bad_parameters_are_rejected_without_a_gpu(libpath):
    import fides_b200 as F
    import numpy as np
    L = F.lib()
    primes = np.array([97, 113], dtype=np.uint64)  # not 1 mod 2N for logN = 12
    prm = F._Params(12, 1, 1, 1, primes.ctypes.data_as(F.u64p), None, 0)
    h = C.c_void_p()
    rc = L.fides_ctx_create(C.byref(prm), C.byref(h))
    assert rc == F.FIDES_OK - 1  # FIDES_ERR_ARG
    assert b"prime" in L.fides_last_error()
    assert L.fides_ctx_create(None, C.byref(h)) == -1


def test_rotation_index_matches_oracle(libpath):
    import fides_b200 as F
    import oracle as O
    for logN in (13, 16):
        for r in (1, -1, 7, 128, -128, (1 << logN) * 2 - 1):
            assert F.auto_index(logN, r) == O.rotation_auto_index(logN, r)


def test_params_agree_with_oracle_prime_search():
    import oracle as O
    from fides_b200 import params as P
    a = P.config_a()
    assert a.q[:1] == O.gen_primes(13, 60, 1)
    assert a.p == O.gen_primes(13, 61, len(a.p), exclude=a.q)
    assert len(a.p) == 3  # reference sizing rule for 60 + 2x50-bit digits
