"""ctypes access to the measurement harness of the reference's own GPU kernels
(baseline/_ref/libref_kernels.so, built by baseline/ref_kernels/Makefile from the reference
sources): NTT / INTT, the ModUp and ModDown conversions, the KSK inner products (plain and
hoisted), the automorphism, SwitchModulus, the tensor product and the elementwise kernels.
Measurement and parity only: used to check the oracle against executed reference code and to
time the reference kernels beside this project's on the same GPU and inputs."""
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
        _lib.ref_kernels_set_reduced_noise.argtypes = [C.c_int]
        _lib.ref_modup.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _lib.ref_moddown.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        vp = C.c_void_p
        _lib.ref_ksk.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, C.POINTER(C.c_float), vp]
        _lib.ref_hoisted_ksk.argtypes = [vp, vp, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(C.c_int),
                                         C.POINTER(vp), C.POINTER(vp), C.c_int, C.POINTER(C.c_float), vp]
        _lib.ref_automorph.argtypes = [vp, vp, C.c_int, vp]
        _lib.ref_switch_modulus.argtypes = [vp, C.c_int, vp, C.c_int, vp]
        _lib.ref_elementwise.argtypes = [C.c_int, vp, vp, C.POINTER(C.c_uint64), C.c_int, vp]
        _lib.ref_tensor.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp]
    return _lib


def init(logN: int, primes, psi, K: int = 0, dnum: int = 1):
    """primes = the n_q Q primes followed by the K special primes; psi their 2N-th roots."""
    n = len(primes)
    rc = lib().ref_kernels_init(logN, n - K, K, dnum, (C.c_uint64 * n)(*primes), (C.c_uint64 * n)(*psi))
    if rc:
        raise RuntimeError(f"ref_kernels_init failed: {rc}")


def set_reduced_noise(on: bool):
    """The reduced-noise conversions (reference Parameters::reducedNoise) on or off."""
    rc = lib().ref_kernels_set_reduced_noise(1 if on else 0)
    if rc:
        raise RuntimeError(f"ref_kernels_set_reduced_noise failed: {rc}")


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


def _rc(rc, what):
    if rc:
        raise RuntimeError(f"{what} failed: {rc}")


def ksk(digits, level: int, key, out_a, out_b, stream: int, reps: int = 0) -> float | None:
    """fusedDotKSK_2_: digits [beta][level+K][N] (ModUp output, own-digit limbs included), key
    [2][dnum][n_q+K][N] -> out_a, out_b [level+K][N].  reps > 0: returns the mean time (ms) of
    `reps` further launches."""
    ms = C.c_float(0)
    _rc(lib().ref_ksk(digits.data_ptr(), level, key.data_ptr(), out_a.data_ptr(), out_b.data_ptr(), reps,
                      C.byref(ms), stream), "ref_ksk")
    return ms.value if reps > 0 else None


def hoisted_ksk(digits, c0, level: int, keys, auto_indices, out0, out1, stream: int, reps: int = 0):
    """hoistedRotateDotKSK_2_: one ModUp output of c1, c0 [level][N], n keys and automorphism
    indices -> out0[r] (b side + P c0) and out1[r] (a side), [level+K][N] each, scattered by the
    automorphism."""
    n = len(keys)
    vp = C.c_void_p
    ms = C.c_float(0)
    _rc(lib().ref_hoisted_ksk(digits.data_ptr(), c0.data_ptr(), level, n, (vp * n)(*[k.data_ptr() for k in keys]),
                              (C.c_int * n)(*auto_indices), (vp * n)(*[o.data_ptr() for o in out0]),
                              (vp * n)(*[o.data_ptr() for o in out1]), reps, C.byref(ms), stream), "ref_hoisted_ksk")
    return ms.value if reps > 0 else None


def automorph(x, out, k: int, stream: int):
    """automorph_ on one limb [N]."""
    _rc(lib().ref_automorph(x.data_ptr(), out.data_ptr(), k, stream), "ref_automorph")


def switch_modulus(x, src_id: int, out, dst_id: int, stream: int):
    """SwitchModulus of one coefficient vector [N] from prime src_id to prime dst_id."""
    _rc(lib().ref_switch_modulus(x.data_ptr(), src_id, out.data_ptr(), dst_id, stream), "ref_switch_modulus")


EW = {"add": 0, "sub": 1, "mul": 2, "mul_scalar": 3, "add_scalar": 4}


def elementwise(op: str, a, b, level: int, stream: int, scalars=None):
    """In place on a [level][N]: add_ / sub_ / mult_ with b, or scalar_mult_ / scalar_add_ with
    one (reduced) scalar per limb."""
    sc = (C.c_uint64 * level)(*scalars) if scalars is not None else None
    _rc(lib().ref_elementwise(EW[op], a.data_ptr(), None if b is None else b.data_ptr(), sc, level, stream),
        "ref_elementwise")


def tensor(c0, c1, c2, d0, d1, level: int, stream: int):
    """binomialMult_ in place: (c0, c1, c2) <- (c0 d0, c0 d1 + c1 d0, c1 d1)."""
    _rc(lib().ref_tensor(c0.data_ptr(), c1.data_ptr(), c2.data_ptr(), d0.data_ptr(), d1.data_ptr(), level, stream),
        "ref_tensor")
