"""ctypes front-end of the CPU oracle (oracle/ckks_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm, always as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

u64p = C.POINTER(C.c_uint64)
i32p = C.POINTER(C.c_int)


def build() -> str:
    """Compile liboracle.so with the system C compiler (idempotent via make)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.or_mulmod.restype = C.c_uint64
        L.or_mulmod.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.or_powmod.restype = C.c_uint64
        L.or_powmod.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.or_invmod.restype = C.c_uint64
        L.or_invmod.argtypes = [C.c_uint64, C.c_uint64]
        L.or_is_prime.restype = C.c_int
        L.or_is_prime.argtypes = [C.c_uint64]
        L.or_gen_primes.restype = C.c_int
        L.or_gen_primes.argtypes = [C.c_int, C.c_int, C.c_int, u64p, C.c_int, u64p]
        L.or_generator.restype = C.c_uint64
        L.or_generator.argtypes = [C.c_uint64]
        L.or_root_2n.restype = C.c_uint64
        L.or_root_2n.argtypes = [C.c_uint64, C.c_int]
        L.or_ctx_create.restype = C.c_void_p
        L.or_ctx_create.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int]
        L.or_ctx_destroy.argtypes = [C.c_void_p]
        L.or_ctx_set_reduced_noise.argtypes = [C.c_void_p, C.c_int]
        L.or_ctx_alpha.restype = C.c_int
        L.or_ctx_alpha.argtypes = [C.c_void_p]
        L.or_ctx_psi.restype = C.c_uint64
        L.or_ctx_psi.argtypes = [C.c_void_p, C.c_int]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        L.or_ntt.argtypes = [C.c_void_p, u64p, C.c_int, i32p, C.c_int]
        L.or_switch_basis.argtypes = [C.c_void_p, u64p, C.c_int, i32p, u64p, C.c_int, i32p]
        L.or_switch_basis_lift.argtypes = L.or_switch_basis.argtypes
        for f in ("or_poly_mul", "or_poly_add", "or_poly_sub"):
            getattr(L, f).argtypes = [C.c_void_p, u64p, u64p, u64p, C.c_int, i32p]
        L.or_tensor.argtypes = [C.c_void_p, u64p, u64p, u64p, u64p, C.c_int, u64p, u64p, u64p]
        L.or_automorph.argtypes = [C.c_void_p, u64p, u64p, C.c_int, C.c_uint32]
        L.or_rotation_auto_index.restype = C.c_uint32
        L.or_rotation_auto_index.argtypes = [C.c_int, C.c_int]
        L.or_num_digits.restype = C.c_int
        L.or_num_digits.argtypes = [C.c_void_p, C.c_int]
        L.or_modup.argtypes = [C.c_void_p, u64p, C.c_int, u64p]
        L.or_ksk_ip.argtypes = [C.c_void_p, u64p, C.c_int, u64p, u64p, u64p]
        L.or_moddown.argtypes = [C.c_void_p, u64p, C.c_int, u64p]
        L.or_keyswitch.argtypes = [C.c_void_p, u64p, C.c_int, u64p, u64p, u64p]
        L.or_rescale.argtypes = [C.c_void_p, u64p, C.c_int, u64p]
        L.or_switch_modulus.argtypes = [C.c_void_p, u64p, C.c_int, C.c_int, C.c_int, u64p]
        L.or_hmult.argtypes = [C.c_void_p, u64p, u64p, u64p, u64p, C.c_int, u64p, C.c_int, u64p, u64p]
        L.or_rotate_auto.argtypes = [C.c_void_p, u64p, u64p, C.c_int, u64p, C.c_uint32, u64p, u64p]
        L.or_accumulate.argtypes = [C.c_void_p, u64p, u64p, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.c_int), C.POINTER(u64p), C.c_int, u64p, u64p]
        L.or_rotate_hoisted.argtypes = [C.c_void_p, u64p, u64p, C.c_int, C.POINTER(u64p), C.POINTER(C.c_uint32),
                                        C.c_int, C.POINTER(u64p), C.POINTER(u64p)]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(u64p)


def _ip(a):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    return a, a.ctypes.data_as(i32p)


def gen_primes(logN: int, bits: int, count: int, exclude=()) -> list[int]:
    ex = np.array(list(exclude) or [0], dtype=np.uint64)
    out = np.zeros(count, dtype=np.uint64)
    got = lib().or_gen_primes(logN, bits, count, _p(ex), len(exclude), _p(out))
    if got != count:
        raise ValueError(f"only {got} primes of {bits} bits for logN={logN}")
    return [int(x) for x in out]


def root_2n(q: int, logN: int) -> int:
    return int(lib().or_root_2n(q, logN))


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def get_threads() -> int:
    return int(lib().or_get_threads())


def rotation_auto_index(logN: int, r: int) -> int:
    return int(lib().or_rotation_auto_index(logN, r))


class Oracle:
    """CPU restatement of the CKKS evaluation path on one parameter set."""

    def __init__(self, logN: int, q_primes, p_primes, dnum: int, psi=None, reduced_noise: bool = False):
        self.logN, self.N = logN, 1 << logN
        self.q = [int(x) for x in q_primes]
        self.p = [int(x) for x in p_primes]
        self.n_q, self.K, self.dnum = len(self.q), len(self.p), dnum
        primes = np.array(self.q + self.p, dtype=np.uint64)
        ps = np.zeros(len(primes), dtype=np.uint64) if psi is None else np.array(psi, dtype=np.uint64)
        self._h = lib().or_ctx_create(logN, self.n_q, self.K, _p(primes), _p(ps), dnum)
        self.alpha = lib().or_ctx_alpha(self._h)
        self.psi = [int(lib().or_ctx_psi(self._h, i)) for i in range(len(primes))]
        self.primes = [int(x) for x in primes]
        self.reduced_noise = bool(reduced_noise)
        lib().or_ctx_set_reduced_noise(self._h, int(self.reduced_noise))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            try:
                _lib.or_ctx_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- helpers --
    def ids(self, l: int) -> list[int]:
        return list(range(l))

    def ext_ids(self, l: int) -> list[int]:
        return list(range(l)) + [self.n_q + k for k in range(self.K)]

    def beta(self, l: int) -> int:
        return int(lib().or_num_digits(self._h, l))

    def _new(self, rows: int) -> np.ndarray:
        return np.zeros((rows, self.N), dtype=np.uint64)

    # -- transforms --
    def ntt(self, a: np.ndarray, prime_ids, inverse=False) -> np.ndarray:
        out = np.ascontiguousarray(a, dtype=np.uint64).copy()
        ids, ip = _ip(prime_ids)
        assert out.shape == (len(ids), self.N)
        lib().or_ntt(self._h, _p(out), len(ids), ip, 1 if inverse else 0)
        return out

    def switch_basis(self, a: np.ndarray, src_ids, dst_ids, lift: bool = False) -> np.ndarray:
        """ApproxSwitchCRTBasis; lift=True: the reduced-noise form (sources above q_i / 2 taken
        as y_i - q_i)."""
        a = np.ascontiguousarray(a, dtype=np.uint64)
        s, sp = _ip(src_ids)
        d, dp = _ip(dst_ids)
        out = self._new(len(d))
        fn = lib().or_switch_basis_lift if lift else lib().or_switch_basis
        fn(self._h, _p(a), len(s), sp, _p(out), len(d), dp)
        return out

    def _elt(self, fn, a, b, prime_ids):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        ids, ip = _ip(prime_ids)
        out = self._new(len(ids))
        getattr(lib(), fn)(self._h, _p(a), _p(b), _p(out), len(ids), ip)
        return out

    def mul(self, a, b, prime_ids):
        return self._elt("or_poly_mul", a, b, prime_ids)

    def add(self, a, b, prime_ids):
        return self._elt("or_poly_add", a, b, prime_ids)

    def sub(self, a, b, prime_ids):
        return self._elt("or_poly_sub", a, b, prime_ids)

    def tensor(self, a0, a1, b0, b1):
        l = a0.shape[0]
        d = [self._new(l) for _ in range(3)]
        args = [np.ascontiguousarray(x, dtype=np.uint64) for x in (a0, a1, b0, b1)]
        lib().or_tensor(self._h, *[_p(x) for x in args], l, *[_p(x) for x in d])
        return d

    def automorph(self, a, k: int):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        out = np.zeros_like(a)
        lib().or_automorph(self._h, _p(a), _p(out), a.shape[0], k)
        return out

    def switch_modulus(self, a, src_id: int, dst_id: int) -> np.ndarray:
        """SwitchModulus of a coefficient vector from prime src_id to prime dst_id."""
        a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1)
        out = np.empty_like(a)
        lib().or_switch_modulus(self._h, _p(a), a.size, src_id, dst_id, _p(out))
        return out

    def auto_index(self, r: int) -> int:
        return rotation_auto_index(self.logN, r)

    # -- key switching --
    def modup(self, x: np.ndarray) -> np.ndarray:
        l = x.shape[0]
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros((self.beta(l), l + self.K, self.N), dtype=np.uint64)
        lib().or_modup(self._h, _p(x), l, _p(out))
        return out

    def ksk_ip(self, digits: np.ndarray, l: int, key: np.ndarray):
        a, b = self._new(l + self.K), self._new(l + self.K)
        lib().or_ksk_ip(self._h, _p(np.ascontiguousarray(digits)), l, _p(key), _p(a), _p(b))
        return a, b

    def moddown(self, x_ext: np.ndarray) -> np.ndarray:
        l = x_ext.shape[0] - self.K
        out = self._new(l)
        lib().or_moddown(self._h, _p(np.ascontiguousarray(x_ext, dtype=np.uint64)), l, _p(out))
        return out

    def keyswitch(self, d: np.ndarray, key: np.ndarray):
        l = d.shape[0]
        f0, f1 = self._new(l), self._new(l)
        lib().or_keyswitch(self._h, _p(np.ascontiguousarray(d, dtype=np.uint64)), l, _p(key), _p(f0), _p(f1))
        return f0, f1

    # -- ciphertext ops --
    def rescale(self, x: np.ndarray) -> np.ndarray:
        l = x.shape[0]
        out = self._new(l - 1)
        lib().or_rescale(self._h, _p(np.ascontiguousarray(x, dtype=np.uint64)), l, _p(out))
        return out

    def hmult(self, a0, a1, b0, b1, key, rescale=True):
        l = a0.shape[0]
        lo = l - 1 if rescale else l
        o0, o1 = self._new(lo), self._new(lo)
        args = [np.ascontiguousarray(x, dtype=np.uint64) for x in (a0, a1, b0, b1)]
        lib().or_hmult(self._h, *[_p(x) for x in args], l, _p(key), 1 if rescale else 0, _p(o0), _p(o1))
        return o0, o1

    def rotate_auto(self, c0, c1, key, k: int):
        l = c0.shape[0]
        o0, o1 = self._new(l), self._new(l)
        lib().or_rotate_auto(self._h, _p(np.ascontiguousarray(c0)), _p(np.ascontiguousarray(c1)), l, _p(key), k,
                             _p(o0), _p(o1))
        return o0, o1

    def rotate(self, c0, c1, key, r: int):
        return self.rotate_auto(c0, c1, key, self.auto_index(r))

    def accumulate(self, c0, c1, radix: int, stride: int, size: int, keys: dict):
        """Rotation sum (reference Accumulate); keys: rotation index -> switching key."""
        l = c0.shape[0]
        rots = list(keys)
        karr = [np.ascontiguousarray(keys[r], dtype=np.uint64) for r in rots]
        kp = (u64p * max(1, len(rots)))(*[_p(k) for k in karr])
        kr = (C.c_int * max(1, len(rots)))(*rots)
        o0, o1 = self._new(l), self._new(l)
        rc = lib().or_accumulate(self._h, _p(np.ascontiguousarray(c0)), _p(np.ascontiguousarray(c1)), l, radix, stride,
                                 size, kr, kp, len(rots), _p(o0), _p(o1))
        if rc:
            raise ValueError(f"or_accumulate: bad arguments or a missing key ({rc})")
        return o0, o1

    def rotate_hoisted(self, c0, c1, keys, rs):
        l, n = c0.shape[0], len(rs)
        o0 = [self._new(l) for _ in range(n)]
        o1 = [self._new(l) for _ in range(n)]
        kp = (u64p * n)(*[_p(k) for k in keys])
        ks = (C.c_uint32 * n)(*[self.auto_index(r) for r in rs])
        p0 = (u64p * n)(*[_p(x) for x in o0])
        p1 = (u64p * n)(*[_p(x) for x in o1])
        lib().or_rotate_hoisted(self._h, _p(np.ascontiguousarray(c0)), _p(np.ascontiguousarray(c1)), l, kp, ks, n, p0,
                                p1)
        return o0, o1
