"""ctypes access to the measurement harness of the reference's own GPU NTT kernels
(baseline/_ref/libref_kernels.so, built by baseline/ref_kernels/Makefile from the reference
sources).  Measurement only: used to time the reference kernels beside this project's on the
same GPU and inputs."""
import ctypes as C
import os

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "_ref", "libref_kernels.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB)
        _lib.ref_kernels_init.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        _lib.ref_ntt.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
    return _lib


def init(logN: int, primes, psi):
    n = len(primes)
    rc = lib().ref_kernels_init(logN, n, (C.c_uint64 * n)(*primes), (C.c_uint64 * n)(*psi))
    if rc:
        raise RuntimeError(f"ref_kernels_init failed: {rc}")


def ntt(data, aux, n_polys: int, n_limbs: int, inverse: bool, stream: int):
    """data, aux: device uint64 tensors of [n_polys][n_limbs][N]; limb j uses prime j."""
    rc = lib().ref_ntt(data.data_ptr(), aux.data_ptr(), n_polys, n_limbs, 1 if inverse else 0, stream)
    if rc:
        raise RuntimeError(f"ref_ntt failed: {rc}")
