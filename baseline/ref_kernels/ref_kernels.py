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
        _lib.ref_kernels_init.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                                          C.POINTER(C.c_uint64)]
        _lib.ref_ntt.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.ref_modup_dst.argtypes = [C.c_int, C.POINTER(C.c_int)]
        _lib.ref_modup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.ref_moddown.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    return _lib


def init(logN: int, primes, psi, K: int = 0, dnum: int = 1):
    """primes = the n_q Q primes followed by the K special primes; psi their 2N-th roots."""
    n = len(primes)
    rc = lib().ref_kernels_init(logN, n - K, K, dnum, (C.c_uint64 * n)(*primes), (C.c_uint64 * n)(*psi))
    if rc:
        raise RuntimeError(f"ref_kernels_init failed: {rc}")


def modup_dst(d: int) -> list:
    ids = (C.c_int * 64)()
    n = lib().ref_modup_dst(d, ids)
    if n < 0:
        raise RuntimeError("bad digit")
    return list(ids[:n])


def modup(x, level: int, d: int, out, stream: int):
    """ModUp conversion of digit d at `level`: x [level][N] coefficient-domain Q limbs; out
    [len(modup_dst(d))][N] receives one row per destination prime."""
    rc = lib().ref_modup(x.data_ptr(), level, d, out.data_ptr(), stream)
    if rc:
        raise RuntimeError(f"ref_modup failed: {rc}")


def moddown(sp, level: int, out, stream: int):
    """ModDown conversion: sp [K][N] coefficient-domain special limbs -> out [level][N]."""
    rc = lib().ref_moddown(sp.data_ptr(), level, out.data_ptr(), stream)
    if rc:
        raise RuntimeError(f"ref_moddown failed: {rc}")


def ntt(data, aux, n_polys: int, n_limbs: int, inverse: bool, stream: int):
    """data, aux: device uint64 tensors of [n_polys][n_limbs][N]; limb j uses prime j."""
    rc = lib().ref_ntt(data.data_ptr(), aux.data_ptr(), n_polys, n_limbs, 1 if inverse else 0, stream)
    if rc:
        raise RuntimeError(f"ref_ntt failed: {rc}")
