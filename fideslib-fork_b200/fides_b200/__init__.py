"""Python binding of the B200 CKKS evaluation core (libfides_b200.so, C ABI in
include/fides_b200.h).

The library is the product; this module only marshals arguments.  Device memory comes
from torch (uint64 CUDA tensors); every call runs the CUDA kernels on the caller's
current torch stream.  There is no CPU fallback: a missing library or GPU raises.

Names follow the reference's CKKS ciphertext API (src/CKKS/Ciphertext.cuh: mult, rescale,
rotate, rotate_hoisted, keySwitch) and engine plug-in (api/engine/Engine.hpp:75-408:
evalMult, evalRotate, evalFastRotation).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import torch

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "libfides_b200.so")
_lib = None

u64p = C.POINTER(C.c_uint64)
vp = C.c_void_p

FIDES_OK = 0
ERRORS = {-1: "ARG", -2: "CUDA", -3: "OOM", -4: "LEVEL", -5: "KEY", -6: "TIMEOUT", -7: "STATE"}


class FidesError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"fides error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class _Params(C.Structure):
    _fields_ = [("logN", C.c_int), ("n_q", C.c_int), ("n_special", C.c_int), ("dnum", C.c_int),
                ("primes", u64p), ("psi", u64p), ("device", C.c_int)]


class _HMultItem(C.Structure):
    _fields_ = [("a0", vp), ("a1", vp), ("b0", vp), ("b1", vp), ("out0", vp), ("out1", vp), ("level", C.c_int)]


class _ServerConfig(C.Structure):
    _fields_ = [("n_streams", C.c_int), ("max_batch", C.c_int), ("hbm_budget_bytes", C.c_size_t)]


class _Request(C.Structure):
    _fields_ = [("op", C.c_int), ("level", C.c_int), ("c0", vp), ("c1", vp), ("d0", vp), ("d1", vp),
                ("out0", vp), ("out1", vp), ("rotation", C.c_int)]


class _ServerStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "rejected", "batches", "batched_requests",
                                          "peak_bytes")]


OP_HMULT, OP_HMULT_NORESCALE, OP_ROTATE, OP_BOOTSTRAP = 0, 1, 2, 3


class _HMultHostItem(C.Structure):
    _fields_ = [("a0", vp), ("a1", vp), ("b0", vp), ("b1", vp), ("out0", vp), ("out1", vp), ("level", C.c_int)]


class _HoistItem(C.Structure):
    _fields_ = [("c0", vp), ("c1", vp), ("level", C.c_int), ("n", C.c_int), ("keys", C.POINTER(vp)),
                ("rotations", C.POINTER(C.c_int)), ("out0", C.POINTER(vp)), ("out1", C.POINTER(vp))]


class _RotateHostItem(C.Structure):
    _fields_ = [("c0", vp), ("c1", vp), ("out0", vp), ("out1", vp), ("key", vp), ("level", C.c_int),
                ("rotation", C.c_int)]


class _RotateItem(C.Structure):
    _fields_ = [("c0", vp), ("c1", vp), ("out0", vp), ("out1", vp), ("key", vp), ("level", C.c_int),
                ("auto_index", C.c_uint32)]


class _BootParams(C.Structure):
    _fields_ = [("level_budget_cts", C.c_int), ("level_budget_stc", C.c_int), ("top_level", C.c_int),
                ("top_scale", C.c_double), ("msg_scale", C.c_double), ("K", C.c_int), ("r", C.c_int),
                ("degree", C.c_int), ("baby", C.c_int), ("prescale_bits", C.c_int), ("sparse_encapsulation", C.c_int),
                ("correction_bits", C.c_int), ("double_hoist", C.c_int)]


def build(force: bool = False) -> str:
    """Compile libfides_b200.so for sm_100a with nvcc (make, in-tree)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", _PKG], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FidesError(-7, f"{LIB_PATH} is not built (run build())")
        L = C.CDLL(LIB_PATH)
        L.fides_last_error.restype = C.c_char_p
        L.fides_ctx_create.argtypes = [C.POINTER(_Params), C.POINTER(vp)]
        L.fides_ctx_destroy.argtypes = [vp]
        L.fides_ctx_psi.argtypes = [vp, u64p]
        L.fides_ctx_alpha.argtypes = [vp]
        L.fides_ctx_scratch_bytes.argtypes = [vp]
        L.fides_ctx_scratch_bytes.restype = C.c_size_t
        L.fides_ctx_set_scratch_limit.argtypes = [vp, C.c_size_t]
        L.fides_ctx_launch_count.argtypes = [vp]
        L.fides_ctx_launch_count.restype = C.c_uint64
        L.fides_ctx_profile.argtypes = [vp, C.c_int]
        L.fides_ctx_set_conv_engine.argtypes = [vp, C.c_int]
        L.fides_ctx_set_reduced_noise.argtypes = [vp, C.c_int]
        L.fides_int_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
        L.fides_f64_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
        L.fides_ctx_ntt_counts.argtypes = [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.fides_ctx_autotune.argtypes = [vp, C.POINTER(C.c_float)]
        L.fides_ctx_reserve_scratch.argtypes = [vp, C.c_size_t]
        L.fides_server_add_bootstrap.argtypes = [vp, vp, vp, vp, C.c_int, vp, vp, C.c_int]
        L.fides_server_add_bootstrap_batch.argtypes = [vp, vp, C.c_int, C.POINTER(vp), C.POINTER(vp), C.c_int,
                                                       C.POINTER(vp), C.POINTER(vp), C.c_int]
        L.fides_server_set_max_inflight.argtypes = [vp, C.c_int]
        L.fides_rotate_hoisted_batch.argtypes = [vp, C.POINTER(_HoistItem), C.c_int, vp]
        L.fides_ctx_ntt_shapes.argtypes = [vp, C.POINTER(C.c_uint8)]
        L.fides_ctx_set_ntt_shape.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.fides_ctx_ntt_residues.argtypes = [vp, C.POINTER(C.c_uint8)]
        L.fides_ctx_set_ntt_residues.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
        L.fides_ctx_device_status.argtypes = [vp, C.POINTER(C.c_uint32), C.c_int]
        L.fides_ctx_synchronize.argtypes = [vp, vp]
        L.fides_ctx_ntt_chunk.argtypes = [vp, C.c_int]
        L.fides_boot_create.argtypes = [vp, C.POINTER(_BootParams), C.POINTER(vp)]
        L.fides_accumulate.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(vp), C.c_int, vp, vp, vp]
        L.fides_accumulate_rotations.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int]
        L.fides_eval_chebyshev.argtypes = [vp, vp, C.c_double, vp, vp, C.c_int, C.c_double,
                                           C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, vp, vp,
                                           C.POINTER(C.c_int), C.POINTER(C.c_double), vp]
        L.fides_boot_destroy.argtypes = [vp]
        L.fides_boot_rotations.argtypes = [vp, C.POINTER(C.c_int), C.c_int]
        L.fides_boot_set_keys.argtypes = [vp, vp, vp, vp, vp]
        L.fides_boot_set_rotation_key.argtypes = [vp, C.c_int, vp]
        L.fides_boot_prepare.argtypes = [vp, vp]
        L.fides_boot_levels.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.fides_bootstrap.argtypes = [vp, vp, vp, vp, vp, vp]
        L.fides_bootstrap_batch.argtypes = [vp, C.c_int, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), vp]
        L.fides_boot_chebyshev.argtypes = [vp, C.POINTER(C.c_double), C.c_int]
        L.fides_boot_matrices.argtypes = [vp, C.c_int]
        L.fides_boot_plaintext.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
        L.fides_boot_table.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int, vp]
        L.fides_ctx_inject_status.argtypes = [vp, C.c_uint32]
        L.fides_kernel_arch.argtypes = [C.c_int, C.POINTER(C.c_int)]
        L.fides_server_wait_timeout.argtypes = [vp, C.c_uint64, C.c_double, C.POINTER(C.c_double),
                                                C.POINTER(C.c_int)]
        L.fides_ctx_profile_read.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                             C.POINTER(C.c_uint64)]
        L.fides_rotation_auto_index.argtypes = [C.c_int, C.c_int]
        L.fides_rotation_auto_index.restype = C.c_uint32
        L.fides_ntt_limbs.argtypes = [vp, C.POINTER(vp), C.POINTER(C.c_int), C.c_int, C.c_int, vp]
        L.fides_ntt_polys.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, vp]
        L.fides_modup.argtypes = [vp, vp, C.c_int, vp, vp]
        L.fides_ksk_inner_product.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp]
        L.fides_moddown.argtypes = [vp, vp, C.c_int, vp, vp]
        L.fides_keyswitch.argtypes = [vp, vp, C.c_int, vp, vp, vp, vp]
        L.fides_tensor.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp]
        L.fides_rescale.argtypes = [vp, vp, C.c_int, vp, vp]
        L.fides_hmult.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp, C.c_int, vp, vp, vp]
        L.fides_rotate.argtypes = [vp, vp, vp, C.c_int, vp, C.c_int, vp, vp, vp]
        L.fides_rotate_auto.argtypes = [vp, vp, vp, C.c_int, vp, C.c_uint32, vp, vp, vp]
        L.fides_rotate_hoisted.argtypes = [vp, vp, vp, C.c_int, C.POINTER(vp), C.POINTER(C.c_int), C.c_int,
                                           C.POINTER(vp), C.POINTER(vp), vp]
        L.fides_hmult_batch.argtypes = [vp, C.POINTER(_HMultItem), C.c_int, vp, C.c_int, vp]
        L.fides_rotate_batch.argtypes = [vp, C.POINTER(_RotateItem), C.c_int, vp]
        L.fides_mixed_batch.argtypes = [vp, C.POINTER(_HMultItem), C.c_int, vp, C.c_int, C.POINTER(_RotateItem),
                                        C.c_int, vp]
        L.fides_key_upload.argtypes = [vp, u64p, C.POINTER(vp)]
        L.fides_key_free.argtypes = [vp, vp]
        L.fides_hmult_host.argtypes = [vp, u64p, u64p, u64p, u64p, C.c_int, vp, C.c_int, u64p, u64p]
        L.fides_rotate_host.argtypes = [vp, u64p, u64p, C.c_int, vp, C.c_int, u64p, u64p]
        L.fides_hmult_host_batch.argtypes = [vp, C.POINTER(_HMultHostItem), C.c_int, vp, C.c_int]
        L.fides_rotate_host_batch.argtypes = [vp, C.POINTER(_RotateHostItem), C.c_int]
        L.fides_mixed_host_batch.argtypes = [vp, C.POINTER(_HMultHostItem), C.c_int, vp, C.c_int,
                                             C.POINTER(_RotateHostItem), C.c_int]
        L.fides_mixed_host_batch_async.argtypes = L.fides_mixed_host_batch.argtypes
        L.fides_host_batch_wait.argtypes = [vp]
        L.fides_rescale_noalloc.argtypes = [vp, vp, C.c_int, vp, vp]
        L.fides_add.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        L.fides_mul.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        L.fides_mul_scalar.argtypes = [vp, vp, C.c_int, u64p, vp, vp]
        L.fides_dot_plain.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int, vp, vp, vp]
        L.fides_dot_plain_ext.argtypes = L.fides_dot_plain.argtypes
        L.fides_add_ext.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        L.fides_dot_plain_bsgs.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.c_int, C.POINTER(vp), C.c_int, C.c_int,
                                           C.c_int, C.POINTER(vp), C.POINTER(vp), vp]
        L.fides_encode_ext.argtypes = [vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, vp, vp]
        L.fides_rotate_hoisted_ext.argtypes = [vp, vp, C.c_int, vp, C.c_int, C.POINTER(vp), C.POINTER(C.c_int),
                                               C.c_int, C.POINTER(vp), C.POINTER(vp), vp]
        L.fides_lincomb.argtypes = [vp, C.c_int, vp, vp, u64p, u64p, C.c_int, C.c_int, vp, vp, vp]
        L.fides_rescale_batch.argtypes = [vp, vp, vp, vp, C.c_int, vp]
        L.fides_encode.argtypes = [vp, vp, C.c_int, C.c_int, C.c_double, C.c_int, vp, vp]
        L.fides_ct_import.argtypes = [vp, C.c_int, vp, u64p, C.c_int, C.c_int, C.c_int, vp, vp]
        L.fides_ct_export.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, vp]
        L.fides_key_import.argtypes = [vp, vp, C.c_int, C.POINTER(vp)]
        L.fides_decode.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_double, vp, vp]
        L.fides_add_scalar.argtypes = [vp, vp, C.c_int, u64p, vp, vp]
        L.fides_mod_raise.argtypes = [vp, vp, C.c_int, vp, vp]
        L.fides_sub.argtypes = [vp, vp, vp, C.c_int, vp, vp]
        L.fides_capture_begin.argtypes = [vp, vp]
        L.fides_capture_end.argtypes = [vp, vp, C.POINTER(vp)]
        L.fides_graph_launch.argtypes = [vp, vp]
        L.fides_graph_destroy.argtypes = [vp]
        L.fides_server_create.argtypes = [vp, C.POINTER(_ServerConfig), C.POINTER(vp)]
        L.fides_server_set_relin_key.argtypes = [vp, vp]
        L.fides_server_add_rotation_key.argtypes = [vp, C.c_int, vp]
        L.fides_server_submit.argtypes = [vp, C.POINTER(_Request), C.POINTER(C.c_uint64)]
        L.fides_server_wait.argtypes = [vp, C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.fides_server_get_stats.argtypes = [vp, C.POINTER(_ServerStats)]
        L.fides_server_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != FIDES_OK:
        raise FidesError(rc, lib().fides_last_error().decode())


def _ptr(t) -> int | None:
    if t is None:
        return None
    if isinstance(t, int):
        return t
    assert t.dtype == torch.uint64 and t.is_contiguous(), "expected a contiguous uint64 tensor"
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def int_peak(device: int = 0) -> float:
    """Butterflies per second the GPU sustains on the NTT's forward butterfly with
    register-resident data (the integer-pipe roofline of the NTT passes)."""
    v = C.c_double()
    _check(lib().fides_int_peak(device, C.byref(v)))
    return float(v.value)


def f64_peak(device: int = 0) -> float:
    """Butterflies per second of the FP64 butterfly the NTT uses for primes below 2^50,
    register-resident (the FP64-pipe roofline of those limbs' passes)."""
    v = C.c_double()
    _check(lib().fides_f64_peak(device, C.byref(v)))
    return float(v.value)


def kernel_arch(device: int = 0) -> int:
    """cudaFuncAttributes::binaryVersion of the library's kernels as loaded on `device`
    (100 = sm_100a code)."""
    v = C.c_int()
    _check(lib().fides_kernel_arch(device, C.byref(v)))
    return int(v.value)


def auto_index(logN: int, rotation: int) -> int:
    return int(lib().fides_rotation_auto_index(logN, rotation))


@dataclass
class Ciphertext:
    """Device ciphertext (c0, c1) in EVALUATION format at `level` active Q limbs."""
    c0: torch.Tensor
    c1: torch.Tensor

    @property
    def level(self) -> int:
        return int(self.c0.shape[0])


class Context:
    """One parameter set on one GPU (reference: CKKS::Context / ContextData)."""

    def __init__(self, logN: int, q_primes, p_primes, dnum: int, psi=None, device: int = 0,
                 reduced_noise: bool = False):
        import numpy as np
        self.logN, self.N = logN, 1 << logN
        self.q, self.p = [int(x) for x in q_primes], [int(x) for x in p_primes]
        self.n_q, self.K, self.dnum = len(self.q), len(self.p), dnum
        self.device = device
        self._primes = np.array(self.q + self.p, dtype=np.uint64)
        self._psi = None if psi is None else np.array(psi, dtype=np.uint64)
        prm = _Params(logN, self.n_q, self.K, dnum, self._primes.ctypes.data_as(u64p),
                      None if self._psi is None else self._psi.ctypes.data_as(u64p), device)
        h = vp()
        _check(lib().fides_ctx_create(C.byref(prm), C.byref(h)))
        self._h = h
        self.alpha = int(lib().fides_ctx_alpha(h))
        ps = np.zeros(len(self._primes), dtype=np.uint64)
        _check(lib().fides_ctx_psi(h, ps.ctypes.data_as(u64p)))
        self.psi = [int(x) for x in ps]
        if reduced_noise:
            self.set_reduced_noise(True)

    def close(self):
        if getattr(self, "_h", None):
            lib().fides_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- bookkeeping --
    def beta(self, l: int) -> int:
        return (l + self.alpha - 1) // self.alpha

    def ntt_counts(self) -> tuple[int, int]:
        """(FP64-form, integer-form) limb transforms submitted since creation."""
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().fides_ctx_ntt_counts(self._h, C.byref(a), C.byref(b)))
        return int(a.value), int(b.value)

    @property
    def launch_count(self) -> int:
        return int(lib().fides_ctx_launch_count(self._h))

    @property
    def scratch_bytes(self) -> int:
        return int(lib().fides_ctx_scratch_bytes(self._h))

    def reserve_scratch(self, nbytes: int):
        """Grow the scratch pool to `nbytes` once, up front."""
        _check(lib().fides_ctx_reserve_scratch(self._h, nbytes))

    def set_scratch_limit(self, nbytes: int):
        _check(lib().fides_ctx_set_scratch_limit(self._h, nbytes))

    CONV_ENGINES = {"auto": 0, "simt": 1, "tensor": 2}
    NTT_SIZE_CLASSES = (8, 32, 128, None)  # upper bounds of limbs per launch

    def autotune(self) -> dict:
        """Time the NTT tile shapes and residues per thread on the device and keep the fastest
        (fides_ctx_autotune).  Returns both tables and each class's representative transform
        time."""
        ms = (C.c_float * 8)()
        _check(lib().fides_ctx_autotune(self._h, ms))
        return {"shapes": self.ntt_shapes(), "residues_per_thread": self.ntt_residues(),
                "transform_ms": {"forward": list(ms[0:4]), "inverse": list(ms[4:8])}, "chunk_limbs": self.ntt_chunk()}

    def ntt_chunk(self, set_limbs: int = -1) -> int:
        """Limbs per NTT launch pair (fides_ctx_ntt_chunk): set_limbs > 0 sets it, 0 restores
        the largest launch, -1 only reads.  Returns the current value."""
        rc = lib().fides_ctx_ntt_chunk(self._h, set_limbs)
        if rc < 0:
            _check(rc)
        return int(rc)

    def ntt_shapes(self) -> dict:
        """Sub-transforms per CTA by direction / pass / launch-size class."""
        v = (C.c_uint8 * 16)()
        _check(lib().fides_ctx_ntt_shapes(self._h, v))
        return {d: {p: list(v[8 * i + 4 * j: 8 * i + 4 * j + 4]) for j, p in enumerate(("column", "row"))}
                for i, d in enumerate(("forward", "inverse"))}

    def set_ntt_shape(self, inverse: bool, pass_: int, size_class: int, subs_per_cta: int):
        _check(lib().fides_ctx_set_ntt_shape(self._h, int(inverse), pass_, size_class, subs_per_cta))

    def ntt_residues(self) -> dict:
        """Residues per thread (16 or 8) by direction / pass / launch-size class."""
        v = (C.c_uint8 * 16)()
        _check(lib().fides_ctx_ntt_residues(self._h, v))
        return {d: {p: list(v[8 * i + 4 * j: 8 * i + 4 * j + 4]) for j, p in enumerate(("column", "row"))}
                for i, d in enumerate(("forward", "inverse"))}

    def set_ntt_residues(self, inverse: bool, pass_: int, size_class: int, residues_per_thread: int):
        _check(lib().fides_ctx_set_ntt_residues(self._h, int(inverse), pass_, size_class, residues_per_thread))

    def set_conv_engine(self, engine: str):
        """Basis-conversion engine for ModUp/ModDown: 'auto', 'simt' (64-bit integer
        units) or 'tensor' (exact INT8-split product on the tcgen05 tensor cores)."""
        _check(lib().fides_ctx_set_conv_engine(self._h, self.CONV_ENGINES[engine]))

    @staticmethod
    def accumulate_rotations(radix: int, stride: int, size: int) -> list:
        """Rotation indices accumulate() needs (fides_accumulate_rotations)."""
        n = lib().fides_accumulate_rotations(radix, stride, size, None, 0)
        if n < 0:
            _check(n)
        out = (C.c_int * max(1, n))()
        lib().fides_accumulate_rotations(radix, stride, size, out, n)
        return list(out[:n])

    def accumulate(self, ct: "Ciphertext", radix: int, stride: int, size: int, keys: dict) -> "Ciphertext":
        """Rotation sum (fides_accumulate, the reference's AccumulateSum): slot i gathers
        slots i + j stride, j < size.  keys: rotation index -> device key."""
        l = ct.c0.shape[0]
        rots = list(keys)
        kr = (C.c_int * max(1, len(rots)))(*rots)
        kp = (vp * max(1, len(rots)))(*[_ptr(keys[r]) for r in rots])
        o0, o1 = self.empty(l), self.empty(l)
        _check(lib().fides_accumulate(self._h, _ptr(ct.c0), _ptr(ct.c1), l, radix, stride, size, kr, kp, len(rots),
                                      _ptr(o0), _ptr(o1), _stream()))
        return Ciphertext(o0, o1)

    def eval_chebyshev(self, ct: "Ciphertext", relin_key, top_scale: float, scale: float, coeffs, lo=-1.0,
                       hi=1.0):
        """Chebyshev series of ct (fides_eval_chebyshev; OpenFHE's convention c_0 / 2 + sum c_k T_k
        on [lo, hi]) on the canonical scale chain of top_scale.  ct at its level with scale
        `scale`.  Returns (Ciphertext at the output level, its scale)."""
        import numpy as np
        l = ct.c0.shape[0]
        cf = np.ascontiguousarray(coeffs, dtype=np.float64)
        o0, o1 = self.empty(l), self.empty(l)
        lvl, sc = C.c_int(0), C.c_double(0)
        _check(lib().fides_eval_chebyshev(self._h, _ptr(relin_key), top_scale, _ptr(ct.c0), _ptr(ct.c1), l, scale,
                                          cf.ctypes.data_as(C.POINTER(C.c_double)), len(cf), lo, hi, _ptr(o0),
                                          _ptr(o1), C.byref(lvl), C.byref(sc), _stream()))
        return Ciphertext(o0[:lvl.value], o1[:lvl.value]), sc.value

    def set_reduced_noise(self, on: bool):
        """Reduced-noise ModUp/ModDown conversions (reference Parameters::reducedNoise): pre-scaled
        source residues above q_i / 2 are converted as y_i - q_i.  Off by default."""
        _check(lib().fides_ctx_set_reduced_noise(self._h, 1 if on else 0))

    def device_status(self, clear: bool = True) -> int:
        """Synchronises and returns the device status word (bit 0: a bounded device wait
        gave up)."""
        st = C.c_uint32()
        _check(lib().fides_ctx_device_status(self._h, C.byref(st), 1 if clear else 0))
        return int(st.value)

    def synchronize(self, stream=None):
        """Synchronises `stream` (default: torch's current stream) and raises FidesError
        TIMEOUT when a bounded device-side wait gave up since the status was last cleared."""
        _check(lib().fides_ctx_synchronize(self._h, _stream() if stream is None else stream))

    def inject_status(self, bits: int):
        """Host-side fault injection: ORs `bits` into the device status word, as a kernel
        whose bounded wait gave up would (tests of the failure path)."""
        _check(lib().fides_ctx_inject_status(self._h, bits))

    KERNEL_FAMILIES = {"ntt": 0, "conv": 1, "ksk": 2, "elem": 3}

    def profile(self, enable: bool = True):
        _check(lib().fides_ctx_profile(self._h, 1 if enable else 0))

    def profile_read(self, family: str) -> dict:
        ms, by, n = C.c_double(), C.c_double(), C.c_uint64()
        _check(lib().fides_ctx_profile_read(self._h, self.KERNEL_FAMILIES[family], C.byref(ms), C.byref(by),
                                            C.byref(n)))
        return {"ms": ms.value, "bytes": by.value, "launches": int(n.value)}

    def capture(self, stream) -> "Graph":
        """Capture the calls made on `stream` (a torch.cuda.Stream that is current) into a graph."""
        return Graph(self, stream)

    def empty(self, *shape) -> torch.Tensor:
        return torch.empty(*shape, self.N, dtype=torch.uint64, device=f"cuda:{self.device}")

    # -- transforms --
    def ntt_limbs(self, limbs, prime_ids, inverse=False):
        n = len(limbs)
        ptrs = (vp * n)(*[_ptr(t) for t in limbs])
        ids = (C.c_int * n)(*prime_ids)
        _check(lib().fides_ntt_limbs(self._h, ptrs, ids, n, 1 if inverse else 0, _stream()))

    def ntt(self, polys: torch.Tensor, inverse=False):
        """In-place NTT of [n_polys][n_limbs][N] (or [n_limbs][N]) Q-limb polynomials."""
        t = polys if polys.dim() == 3 else polys.unsqueeze(0)
        _check(lib().fides_ntt_polys(self._h, _ptr(t), t.shape[0], t.shape[1], 1 if inverse else 0, _stream()))
        return polys

    def intt(self, polys):
        return self.ntt(polys, inverse=True)

    # -- key switching pieces --
    def modup(self, x: torch.Tensor) -> torch.Tensor:
        l = x.shape[0]
        out = self.empty(self.beta(l), l + self.K)
        _check(lib().fides_modup(self._h, _ptr(x), l, _ptr(out), _stream()))
        return out

    def ksk_inner_product(self, digits, l, key):
        a, b = self.empty(l + self.K), self.empty(l + self.K)
        _check(lib().fides_ksk_inner_product(self._h, _ptr(digits), l, _ptr(key), _ptr(a), _ptr(b), _stream()))
        return a, b

    def moddown(self, x_ext):
        l = x_ext.shape[0] - self.K
        out = self.empty(l)
        _check(lib().fides_moddown(self._h, _ptr(x_ext), l, _ptr(out), _stream()))
        return out

    def keyswitch(self, d, key):
        l = d.shape[0]
        f0, f1 = self.empty(l), self.empty(l)
        _check(lib().fides_keyswitch(self._h, _ptr(d), l, _ptr(key), _ptr(f0), _ptr(f1), _stream()))
        return f0, f1

    # -- ciphertext ops --
    def tensor(self, a: Ciphertext, b: Ciphertext):
        l = a.level
        d = [self.empty(l) for _ in range(3)]
        _check(lib().fides_tensor(self._h, _ptr(a.c0), _ptr(a.c1), _ptr(b.c0), _ptr(b.c1), l,
                                  *[_ptr(x) for x in d], _stream()))
        return d

    def rescale_poly(self, x):
        l = x.shape[0]
        out = self.empty(l - 1)
        _check(lib().fides_rescale(self._h, _ptr(x), l, _ptr(out), _stream()))
        return out

    def rescale_poly_noalloc(self, x, out):
        """fides_rescale_noalloc: same result as rescale_poly, scratch from the library's
        static array (no device allocation); `out` is caller-owned, l - 1 limbs."""
        _check(lib().fides_rescale_noalloc(self._h, _ptr(x), x.shape[0], _ptr(out), _stream()))
        return out

    def rescale(self, ct: Ciphertext) -> Ciphertext:
        return Ciphertext(*self.rescale_many([ct.c0, ct.c1]))

    def rescale_many(self, polys) -> list:
        """Rescale of several polynomials (any levels >= 2) in one launch sequence."""
        n = len(polys)
        if n == 0:
            return []
        outs = [self.empty(x.shape[0] - 1) for x in polys]
        xs = (vp * n)(*[_ptr(x) for x in polys])
        os_ = (vp * n)(*[_ptr(o) for o in outs])
        ls = (C.c_int * n)(*[x.shape[0] for x in polys])
        _check(lib().fides_rescale_batch(self._h, xs, ls, os_, n, _stream()))
        return outs

    def mult(self, a: Ciphertext, b: Ciphertext, relin_key, rescale=True, out: Ciphertext | None = None) -> Ciphertext:
        l = a.level
        lo = l - 1 if rescale else l
        out = out or Ciphertext(self.empty(lo), self.empty(lo))
        _check(lib().fides_hmult(self._h, _ptr(a.c0), _ptr(a.c1), _ptr(b.c0), _ptr(b.c1), l, _ptr(relin_key),
                                 1 if rescale else 0, _ptr(out.c0), _ptr(out.c1), _stream()))
        return out

    def rotate(self, ct: Ciphertext, key, rotation: int, out: Ciphertext | None = None) -> Ciphertext:
        l = ct.level
        out = out or Ciphertext(self.empty(l), self.empty(l))
        _check(lib().fides_rotate(self._h, _ptr(ct.c0), _ptr(ct.c1), l, _ptr(key), rotation, _ptr(out.c0),
                                  _ptr(out.c1), _stream()))
        return out

    def rotate_auto(self, ct: Ciphertext, key, k: int) -> Ciphertext:
        l = ct.level
        out = Ciphertext(self.empty(l), self.empty(l))
        _check(lib().fides_rotate_auto(self._h, _ptr(ct.c0), _ptr(ct.c1), l, _ptr(key), k, _ptr(out.c0),
                                       _ptr(out.c1), _stream()))
        return out

    def rotate_hoisted(self, ct: Ciphertext, keys, rotations) -> list[Ciphertext]:
        n, l = len(rotations), ct.level
        outs = [Ciphertext(self.empty(l), self.empty(l)) for _ in range(n)]
        kp = (vp * n)(*[_ptr(k) for k in keys])
        rs = (C.c_int * n)(*rotations)
        o0 = (vp * n)(*[_ptr(o.c0) for o in outs])
        o1 = (vp * n)(*[_ptr(o.c1) for o in outs])
        _check(lib().fides_rotate_hoisted(self._h, _ptr(ct.c0), _ptr(ct.c1), l, kp, rs, n, o0, o1, _stream()))
        return outs

    def rotate_hoisted_ext(self, ct: Ciphertext, keys, rotations, c0_ext=None) -> list[Ciphertext]:
        """Hoisted rotations left in the extended basis: each result has level + K limbs per
        component (P times the rotation, before ModDown); moddown() of both gives
        rotate_hoisted's results.  c0_ext: an extended c0 added instead of P ct.c0 (ct.c0 is
        then ignored)."""
        n, l = len(rotations), ct.c1.shape[0]
        e = l + self.K
        outs = [Ciphertext(self.empty(e), self.empty(e)) for _ in range(n)]
        kp = (vp * n)(*[_ptr(k) for k in keys])
        rs = (C.c_int * n)(*rotations)
        o0 = (vp * n)(*[_ptr(o.c0) for o in outs])
        o1 = (vp * n)(*[_ptr(o.c1) for o in outs])
        c0, x = (ct.c0, 0) if c0_ext is None else (c0_ext, 1)
        _check(lib().fides_rotate_hoisted_ext(self._h, _ptr(c0), x, _ptr(ct.c1), l, kp, rs, n, o0, o1, _stream()))
        return outs

    def rotate_hoisted_batch(self, cts, keys, rotations) -> list[list[Ciphertext]]:
        """Hoisted rotations of several ciphertexts (any levels) in one launch sequence per
        stage.  keys / rotations: per-ciphertext lists (or one list shared by all)."""
        if rotations and not isinstance(rotations[0], (list, tuple)):
            rotations, keys = [rotations] * len(cts), [keys] * len(cts)
        items = (_HoistItem * max(1, len(cts)))()
        outs, keep = [], []
        for i, (ct, ks, rs) in enumerate(zip(cts, keys, rotations)):
            n, l = len(rs), ct.level
            o = [Ciphertext(self.empty(l), self.empty(l)) for _ in range(n)]
            kp = (vp * max(1, n))(*[_ptr(k) for k in ks])
            rp = (C.c_int * max(1, n))(*rs)
            o0 = (vp * max(1, n))(*[_ptr(x.c0) for x in o])
            o1 = (vp * max(1, n))(*[_ptr(x.c1) for x in o])
            keep += [kp, rp, o0, o1]
            items[i] = _HoistItem(_ptr(ct.c0), _ptr(ct.c1), l, n, kp, rp, o0, o1)
            outs.append(o)
        _check(lib().fides_rotate_hoisted_batch(self._h, items, len(cts), _stream()))
        return outs

    # -- elementwise RNS ops (polynomials of `level` Q limbs) --
    def add_poly(self, a, b, out=None):
        out = self.empty(a.shape[0]) if out is None else out
        _check(lib().fides_add(self._h, _ptr(a), _ptr(b), a.shape[0], _ptr(out), _stream()))
        return out

    def sub_poly(self, a, b, out=None):
        out = self.empty(a.shape[0]) if out is None else out
        _check(lib().fides_sub(self._h, _ptr(a), _ptr(b), a.shape[0], _ptr(out), _stream()))
        return out

    def mul_poly(self, a, b, out=None):
        out = self.empty(a.shape[0]) if out is None else out
        _check(lib().fides_mul(self._h, _ptr(a), _ptr(b), a.shape[0], _ptr(out), _stream()))
        return out

    def dot_plain(self, cts, pts, level=None, out=None):
        """sum_t pts[t] * cts[t] (both components, EVAL) in one launch: the plaintext inner
        product of a linear transform's giant step.  cts: Ciphertexts, pts: polynomials with at
        least `level` limbs (level defaults to the first ciphertext's)."""
        n = len(cts)
        l = cts[0].level if level is None else level
        out = Ciphertext(self.empty(l), self.empty(l)) if out is None else out
        c0 = (vp * n)(*[_ptr(c.c0) for c in cts])
        c1 = (vp * n)(*[_ptr(c.c1) for c in cts])
        pp = (vp * n)(*[_ptr(p) for p in pts])
        _check(lib().fides_dot_plain(self._h, c0, c1, pp, n, l, _ptr(out.c0), _ptr(out.c1), _stream()))
        return out

    def add_ext(self, a, b, level: int, out=None):
        """a + b over extended-basis polynomials ([level + K, N])."""
        out = self.empty(level + self.K) if out is None else out
        _check(lib().fides_add_ext(self._h, _ptr(a), _ptr(b), level, _ptr(out), _stream()))
        return out

    def dot_plain_bsgs(self, babies, pts, level: int, ext: bool = False):
        """Every giant step's inner product in one launch: pts[i][k] (None: no term) times
        babies[k], summed over k, for each giant step i.  ext: Q.P operands and results."""
        nb, ng = len(babies), len(pts)
        e = level + (self.K if ext else 0)
        outs = [Ciphertext(self.empty(e), self.empty(e)) for _ in range(ng)]
        x0 = (vp * nb)(*[_ptr(b.c0) for b in babies])
        x1 = (vp * nb)(*[_ptr(b.c1) for b in babies])
        pp = (vp * (nb * ng))(*[None if p is None else _ptr(p) for row in pts for p in row])
        o0 = (vp * ng)(*[_ptr(o.c0) for o in outs])
        o1 = (vp * ng)(*[_ptr(o.c1) for o in outs])
        _check(lib().fides_dot_plain_bsgs(self._h, x0, x1, nb, pp, ng, level, int(ext), o0, o1, _stream()))
        return outs

    def dot_plain_ext(self, cts, pts, level: int, out=None):
        """dot_plain over extended-basis operands: cts and pts carry level Q limbs followed by
        the K special limbs (rotate_hoisted_ext, encode_ext); out has level + K limbs."""
        n, e = len(cts), level + self.K
        out = Ciphertext(self.empty(e), self.empty(e)) if out is None else out
        c0 = (vp * n)(*[_ptr(c.c0) for c in cts])
        c1 = (vp * n)(*[_ptr(c.c1) for c in cts])
        pp = (vp * n)(*[_ptr(p) for p in pts])
        _check(lib().fides_dot_plain_ext(self._h, c0, c1, pp, n, level, _ptr(out.c0), _ptr(out.c1), _stream()))
        return out

    # -- interop with per-limb host arrays (the reference's RawCipherText / RawKeySwitchKey) --
    def import_limbs(self, polys, format_coeff=False, natural_order=False, check_moduli=True, moduli=None):
        """polys: list of polynomials, each a list of `level` numpy uint64 arrays of N residues
        (one per limb, any host memory).  Returns a device tensor [n_polys, level, N] in
        bit-reversed EVALUATION form."""
        import numpy as np
        n, level = len(polys), len(polys[0])
        arrs = [np.ascontiguousarray(a, dtype=np.uint64) for p in polys for a in p]
        ptrs = (vp * len(arrs))(*[a.ctypes.data for a in arrs])
        if moduli is not None:
            mod = np.array(moduli, dtype=np.uint64)
        else:
            mod = np.array((self.q + self.p)[:level], dtype=np.uint64) if check_moduli else None
        out = torch.empty((n, level, self.N), dtype=torch.int64, device=self.device).view(torch.uint64)
        _check(lib().fides_ct_import(self._h, n, ptrs, None if mod is None else mod.ctypes.data_as(u64p), level,
                                     1 if format_coeff else 0, 1 if natural_order else 0, _ptr(out), _stream()))
        torch.cuda.current_stream(self.device).synchronize()  # the host arrays may go away
        return out

    def export_limbs(self, dev, format_coeff=False, natural_order=False):
        """Device [n_polys, level, N] (bit-reversed EVAL) -> list of lists of numpy limbs."""
        import numpy as np
        d = dev if dev.dim() == 3 else dev.unsqueeze(0)
        n, level = d.shape[0], d.shape[1]
        outs = [[np.empty(self.N, dtype=np.uint64) for _ in range(level)] for _ in range(n)]
        ptrs = (vp * (n * level))(*[a.ctypes.data for p in outs for a in p])
        _check(lib().fides_ct_export(self._h, n, _ptr(d.contiguous()), level, 1 if format_coeff else 0,
                                     1 if natural_order else 0, ptrs, _stream()))
        return outs

    def import_key(self, r_key, natural_order=False):
        """r_key[a/b][digit][limb] numpy arrays (None = zero limb) -> device key pointer (int),
        freed with key_free."""
        import numpy as np
        flat, keep = [], []
        for ab in range(2):
            for d in range(self.dnum):
                for i in range(self.n_q + self.K):
                    a = r_key[ab][d][i]
                    if a is None:
                        flat.append(None)
                    else:
                        a = np.ascontiguousarray(a, dtype=np.uint64)
                        keep.append(a)
                        flat.append(a.ctypes.data)
        ptrs = (vp * len(flat))(*flat)
        out = vp()
        _check(lib().fides_key_import(self._h, ptrs, 1 if natural_order else 0, C.byref(out)))
        return int(out.value)

    # -- slot encode / decode on the device --
    def encode(self, slots, scale: float, level: int):
        """Complex slots -> EVALUATION-form plaintext(s).  slots: complex tensor of shape
        [n_slots] or [n_pts, n_slots] (any device; copied to this GPU as complex128).  Returns
        a uint64 tensor [level, N] (or [n_pts, level, N])."""
        z = torch.as_tensor(slots).to(device=self.device, dtype=torch.complex128).contiguous()
        single = z.dim() == 1
        z = z.reshape(1, -1) if single else z
        n_pts, n = z.shape
        out = torch.empty((n_pts, level, self.N), dtype=torch.int64, device=self.device).view(torch.uint64)
        _check(lib().fides_encode(self._h, torch.view_as_real(z).data_ptr(), n, n_pts, float(scale), level, _ptr(out),
                                  _stream()))
        return out[0] if single else out

    def encode_ext(self, slots, scale: float, level: int):
        """encode over the extended basis (MakeCKKSPackedPlaintextExtended): [level + K, N] (or
        [n_pts, level + K, N]), the level Q limbs then the K special limbs of one integer
        polynomial."""
        z = torch.as_tensor(slots).to(device=self.device, dtype=torch.complex128).contiguous()
        single = z.dim() == 1
        z = z.reshape(1, -1) if single else z
        n_pts, n = z.shape
        out = torch.empty((n_pts, level + self.K, self.N), dtype=torch.int64, device=self.device).view(torch.uint64)
        _check(lib().fides_encode_ext(self._h, torch.view_as_real(z).data_ptr(), n, n_pts, float(scale), level,
                                      _ptr(out), _stream()))
        return out[0] if single else out

    def decode(self, pts, scale: float, n_slots=None):
        """EVALUATION-form plaintext(s) [level, N] or [n_pts, level, N] -> complex128 slots
        (limb 0 is read)."""
        single = pts.dim() == 2
        p = pts.reshape(1, *pts.shape) if single else pts
        p = p.contiguous()
        n_pts, level = p.shape[0], p.shape[1]
        n = self.N // 2 if n_slots is None else n_slots
        z = torch.empty((n_pts, n), dtype=torch.complex128, device=self.device)
        _check(lib().fides_decode(self._h, _ptr(p), level, n_pts, n, float(scale), torch.view_as_real(z).data_ptr(),
                                  _stream()))
        return z[0] if single else z

    def lincomb(self, cts, scalars, add0=None, level=None):
        """sum_t scalars[t] * cts[t] (+ add0 on c0) over `level` limbs in one launch.  scalars[t]
        and add0: an integer (reduced mod every q_i) or one residue per limb."""
        return self.lincomb_lanes([cts], scalars, add0, level)[0]

    def lincomb_lanes(self, lanes, scalars, add0=None, level=None):
        """The same combination over several lanes (lists of ciphertexts, one list per lane,
        all of the same length): one launch, one output Ciphertext per lane."""
        import numpy as np
        n, m = len(lanes[0]), len(lanes)
        l = min(c.level for cts in lanes for c in cts) if level is None else level
        outs = [Ciphertext(self.empty(l), self.empty(l)) for _ in range(m)]
        s = np.stack([self._scalars(v, l) for v in scalars])
        a = None if add0 is None else self._scalars(add0, l)
        c0 = (vp * (n * m))(*[_ptr(c.c0) for cts in lanes for c in cts])
        c1 = (vp * (n * m))(*[_ptr(c.c1) for cts in lanes for c in cts])
        o0 = (vp * m)(*[_ptr(o.c0) for o in outs])
        o1 = (vp * m)(*[_ptr(o.c1) for o in outs])
        _check(lib().fides_lincomb(self._h, m, c0, c1, s.ctypes.data_as(u64p),
                                   None if a is None else a.ctypes.data_as(u64p), n, l, o0, o1, _stream()))
        return outs

    def _scalars(self, values, l):
        import numpy as np
        v = np.array([int(values[i]) % self.q[i] if hasattr(values, "__len__") else int(values) % self.q[i]
                      for i in range(l)], dtype=np.uint64)
        return v

    def mul_scalar_poly(self, a, values, out=None):
        """a_i * values_i mod q_i (values: one int, or one residue per limb)."""
        out = self.empty(a.shape[0]) if out is None else out
        v = self._scalars(values, a.shape[0])
        _check(lib().fides_mul_scalar(self._h, _ptr(a), a.shape[0], v.ctypes.data_as(u64p), _ptr(out), _stream()))
        return out

    def add_scalar_poly(self, a, values, out=None):
        out = self.empty(a.shape[0]) if out is None else out
        v = self._scalars(values, a.shape[0])
        _check(lib().fides_add_scalar(self._h, _ptr(a), a.shape[0], v.ctypes.data_as(u64p), _ptr(out), _stream()))
        return out

    def mod_raise_poly(self, x, level: int):
        """Level-1 polynomial (limb q_0) -> `level` limbs with the centred residues."""
        out = self.empty(level)
        _check(lib().fides_mod_raise(self._h, _ptr(x), level, _ptr(out), _stream()))
        return out

    # -- batched forms --
    def mult_batch(self, pairs, relin_key, rescale=True) -> list[Ciphertext]:
        n = len(pairs)
        outs, items = [], (_HMultItem * n)()
        for i, (a, b) in enumerate(pairs):
            lo = a.level - 1 if rescale else a.level
            o = Ciphertext(self.empty(lo), self.empty(lo))
            outs.append(o)
            items[i] = _HMultItem(_ptr(a.c0), _ptr(a.c1), _ptr(b.c0), _ptr(b.c1), _ptr(o.c0), _ptr(o.c1), a.level)
        _check(lib().fides_hmult_batch(self._h, items, n, _ptr(relin_key), 1 if rescale else 0, _stream()))
        return outs

    def rotate_batch(self, jobs) -> list[Ciphertext]:
        """jobs: list of (ciphertext, key, rotation)."""
        n = len(jobs)
        outs, items = [], (_RotateItem * n)()
        for i, (ct, key, r) in enumerate(jobs):
            o = Ciphertext(self.empty(ct.level), self.empty(ct.level))
            outs.append(o)
            items[i] = _RotateItem(_ptr(ct.c0), _ptr(ct.c1), _ptr(o.c0), _ptr(o.c1), _ptr(key), ct.level,
                                   auto_index(self.logN, r))
        _check(lib().fides_rotate_batch(self._h, items, n, _stream()))
        return outs

    def mixed_batch(self, pairs, relin_key, rots, rescale=True) -> tuple[list[Ciphertext], list[Ciphertext]]:
        """HMults of `pairs` and rotations `rots` ((ciphertext, key, rotation) jobs) in one launch
        sequence (fides_mixed_batch); returns (products, rotated)."""
        nh, nr = len(pairs), len(rots)
        hout, rout = [], []
        hitems, ritems = (_HMultItem * max(nh, 1))(), (_RotateItem * max(nr, 1))()
        for i, (a, b) in enumerate(pairs):
            lo = a.level - 1 if rescale else a.level
            o = Ciphertext(self.empty(lo), self.empty(lo))
            hout.append(o)
            hitems[i] = _HMultItem(_ptr(a.c0), _ptr(a.c1), _ptr(b.c0), _ptr(b.c1), _ptr(o.c0), _ptr(o.c1), a.level)
        for i, (ct, key, r) in enumerate(rots):
            o = Ciphertext(self.empty(ct.level), self.empty(ct.level))
            rout.append(o)
            ritems[i] = _RotateItem(_ptr(ct.c0), _ptr(ct.c1), _ptr(o.c0), _ptr(o.c1), _ptr(key), ct.level,
                                    auto_index(self.logN, r))
        _check(lib().fides_mixed_batch(self._h, hitems, nh, _ptr(relin_key), 1 if rescale else 0, ritems, nr,
                                       _stream()))
        return hout, rout

    # -- host-buffer path --
    def key_upload(self, host_key) -> int:
        import numpy as np
        hk = np.ascontiguousarray(host_key, dtype=np.uint64)
        assert hk.shape == (2, self.dnum, self.n_q + self.K, self.N)
        d = vp()
        _check(lib().fides_key_upload(self._h, hk.ctypes.data_as(u64p), C.byref(d)))
        return int(d.value)

    def key_free(self, dev_key: int):
        _check(lib().fides_key_free(self._h, dev_key))

    def mult_host(self, a0, a1, b0, b1, dev_key: int, rescale=True, out0=None, out1=None):
        import numpy as np
        l = a0.shape[0]
        lo = l - 1 if rescale else l
        out0 = np.empty((lo, self.N), dtype=np.uint64) if out0 is None else out0
        out1 = np.empty((lo, self.N), dtype=np.uint64) if out1 is None else out1
        P = lambda a: a.ctypes.data_as(u64p)
        _check(lib().fides_hmult_host(self._h, P(a0), P(a1), P(b0), P(b1), l, dev_key, 1 if rescale else 0,
                                      P(out0), P(out1)))
        return out0, out1

    def rotate_host(self, c0, c1, dev_key: int, rotation: int, out0=None, out1=None):
        import numpy as np
        l = c0.shape[0]
        out0 = np.empty((l, self.N), dtype=np.uint64) if out0 is None else out0
        out1 = np.empty((l, self.N), dtype=np.uint64) if out1 is None else out1
        P = lambda a: a.ctypes.data_as(u64p)
        _check(lib().fides_rotate_host(self._h, P(c0), P(c1), l, dev_key, rotation, P(out0), P(out1)))
        return out0, out1


    def mult_host_batch(self, items, dev_key: int, rescale=True):
        """Pipelined HMult of host ciphertexts.  items: (a0, a1, b0, b1, out0, out1) tuples of
        contiguous uint64 arrays (pinned for overlap); outputs are written in place."""
        arr = (_HMultHostItem * max(1, len(items)))()
        for k, (a0, a1, b0, b1, o0, o1) in enumerate(items):
            arr[k] = _HMultHostItem(a0.ctypes.data, a1.ctypes.data, b0.ctypes.data, b1.ctypes.data,
                                    o0.ctypes.data, o1.ctypes.data, a0.shape[0])
        _check(lib().fides_hmult_host_batch(self._h, arr, len(items), dev_key, 1 if rescale else 0))

    def rotate_host_batch(self, items):
        """Pipelined rotations of host ciphertexts.  items: (c0, c1, out0, out1, dev_key,
        rotation) tuples; outputs are written in place."""
        arr = (_RotateHostItem * max(1, len(items)))()
        for k, (c0, c1, o0, o1, key, r) in enumerate(items):
            arr[k] = _RotateHostItem(c0.ctypes.data, c1.ctypes.data, o0.ctypes.data, o1.ctypes.data, key,
                                     c0.shape[0], r)
        _check(lib().fides_rotate_host_batch(self._h, arr, len(items)))

    def mixed_host_batch(self, hmult_items, dev_key: int, rotate_items, rescale=True, wait=True):
        """HMults and rotations of host ciphertexts through one pipeline (items as in
        mult_host_batch / rotate_host_batch, alternated); outputs are written in place.
        With wait=False the call returns once everything is enqueued and consecutive calls
        continue one pipeline: the arrays must stay alive and unchanged, and the outputs
        unread, until host_batch_wait()."""
        ha = (_HMultHostItem * max(1, len(hmult_items)))()
        for k, (a0, a1, b0, b1, o0, o1) in enumerate(hmult_items):
            ha[k] = _HMultHostItem(a0.ctypes.data, a1.ctypes.data, b0.ctypes.data, b1.ctypes.data,
                                   o0.ctypes.data, o1.ctypes.data, a0.shape[0])
        ra = (_RotateHostItem * max(1, len(rotate_items)))()
        for k, (c0, c1, o0, o1, key, r) in enumerate(rotate_items):
            ra[k] = _RotateHostItem(c0.ctypes.data, c1.ctypes.data, o0.ctypes.data, o1.ctypes.data, key,
                                    c0.shape[0], r)
        fn = lib().fides_mixed_host_batch if wait else lib().fides_mixed_host_batch_async
        _check(fn(self._h, ha, len(hmult_items), dev_key, 1 if rescale else 0, ra, len(rotate_items)))

    def host_batch_wait(self):
        """Waits for every pipelined host batch of this context (fides_host_batch_wait)."""
        _check(lib().fides_host_batch_wait(self._h))


def pinned_empty(shape) -> "np.ndarray":
    """A uint64 host array in page-locked memory (for asynchronous host <-> device copies)."""
    import numpy as np
    n = int(np.prod(shape))
    t = torch.empty(n, dtype=torch.int64, pin_memory=True)
    return t.numpy().view(np.uint64).reshape(shape)  # the array's base chain keeps t alive


def to_device(a, device: int = 0) -> torch.Tensor:
    """Host uint64 array -> device uint64 tensor (copied through an int64 view)."""
    import numpy as np
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64)).to(f"cuda:{device}").view(torch.uint64)


def to_host(t: torch.Tensor):
    import numpy as np
    return t.contiguous().view(torch.int64).cpu().numpy().view(np.uint64)


class Graph:
    """A captured sequence of library calls (fides_capture_* / fides_graph_*).

    Usage:  with ctx.capture(stream) as g: ...calls on `stream`...;  then g.launch(stream).
    """

    def __init__(self, ctx: "Context", stream):
        self.ctx, self.stream, self._h = ctx, stream, None

    def __enter__(self):
        _check(lib().fides_capture_begin(self.ctx._h, self.stream.cuda_stream))
        return self

    def __exit__(self, et, ev, tb):
        h = vp()
        rc = lib().fides_capture_end(self.ctx._h, self.stream.cuda_stream, C.byref(h))
        if et is None:
            _check(rc)
            self._h = h
        return False

    def launch(self, stream=None):
        s = (stream or self.stream).cuda_stream
        _check(lib().fides_graph_launch(self._h, s))

    def close(self):
        if self._h:
            lib().fides_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NativeBootstrapper:
    """The library's C++ bootstrapper (fides_boot_*): tables derived at creation, device keys set
    by the caller (kept referenced here), full packing (N/2 slots).  bootstrap() reads limb q_0
    of (c0, c1) and returns the output Ciphertext at out_level limbs, scale out_scale."""

    def __init__(self, ctx: "Context", top_level: int, top_scale: float, msg_scale: float, budget=(3, 3),
                 K: int = 12, r: int = 3, degree: int = 31, baby: int = 8, prescale_bits: int = 0,
                 encapsulation: bool = False, correction_bits: int = 0, double_hoist: bool = True):
        self.ctx = ctx
        p = _BootParams(budget[0], budget[1], top_level, float(top_scale), float(msg_scale), K, r, degree, baby,
                        prescale_bits, 1 if encapsulation else 0, correction_bits, 1 if double_hoist else 0)
        h = vp()
        _check(lib().fides_boot_create(ctx._h, C.byref(p), C.byref(h)))
        self._h = h
        self._keys = []

    def close(self):
        if getattr(self, "_h", None):
            lib().fides_boot_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rotations(self) -> list[int]:
        n = lib().fides_boot_rotations(self._h, None, 0)
        buf = (C.c_int * max(1, n))()
        lib().fides_boot_rotations(self._h, buf, n)
        return list(buf[:n])

    def set_keys(self, relin, conj, to_sparse=None, to_dense=None):
        self._keys += [relin, conj, to_sparse, to_dense]
        _check(lib().fides_boot_set_keys(self._h, _ptr(relin), _ptr(conj), _ptr(to_sparse), _ptr(to_dense)))

    def set_rotation_key(self, rotation: int, key):
        self._keys.append(key)
        _check(lib().fides_boot_set_rotation_key(self._h, rotation, _ptr(key)))

    def prepare(self):
        _check(lib().fides_boot_prepare(self._h, _stream()))

    @property
    def out_level(self) -> int:
        lv, sc = C.c_int(), C.c_double()
        _check(lib().fides_boot_levels(self._h, C.byref(lv), C.byref(sc)))
        return int(lv.value)

    @property
    def out_scale(self) -> float:
        lv, sc = C.c_int(), C.c_double()
        _check(lib().fides_boot_levels(self._h, C.byref(lv), C.byref(sc)))
        return float(sc.value)

    def bootstrap(self, ct: "Ciphertext") -> "Ciphertext":
        lo = self.out_level
        out = Ciphertext(self.ctx.empty(lo), self.ctx.empty(lo))
        _check(lib().fides_bootstrap(self._h, _ptr(ct.c0), _ptr(ct.c1), _ptr(out.c0), _ptr(out.c1), _stream()))
        return out

    def bootstrap_batch(self, cts) -> list:
        n, lo = len(cts), self.out_level
        outs = [Ciphertext(self.ctx.empty(lo), self.ctx.empty(lo)) for _ in cts]
        arr = lambda xs: (vp * n)(*xs)
        _check(lib().fides_bootstrap_batch(self._h, n, arr([_ptr(c.c0) for c in cts]), arr([_ptr(c.c1) for c in cts]),
                                           arr([_ptr(o.c0) for o in outs]), arr([_ptr(o.c1) for o in outs]),
                                           _stream()))
        return outs

    def chebyshev(self):
        import numpy as np
        n = lib().fides_boot_chebyshev(self._h, None, 0)
        buf = np.empty(n, dtype=np.float64)
        lib().fides_boot_chebyshev(self._h, buf.ctypes.data_as(C.POINTER(C.c_double)), n)
        return buf

    def plaintext(self, which: str, m: int, i: int, j: int, level: int):
        """The encoded diagonal (giant step i, baby step j) of matrix m, `level` limbs."""
        out = self.ctx.empty(level)
        _check(lib().fides_boot_plaintext(self._h, {"cts": 0, "stc": 1}[which], m, i, j, _ptr(out), _stream()))
        return out

    def matrices(self, which: str) -> list:
        """The composed special-FFT matrices of 'cts' (CoeffsToSlots) or 'stc' (SlotsToCoeffs)
        as dicts slot offset -> complex diagonal (numpy)."""
        import numpy as np
        w = {"cts": 0, "stc": 1}[which]
        mats = []
        n = self.ctx.N // 2
        for m in range(lib().fides_boot_matrices(self._h, w)):
            cnt = lib().fides_boot_table(self._h, w, m, None, 0, None)
            offs = (C.c_int * cnt)()
            d = np.empty((cnt, n), dtype=np.complex128)
            lib().fides_boot_table(self._h, w, m, offs, cnt, d.ctypes.data)
            mats.append({int(o): d[k] for k, o in enumerate(offs)})
        return mats


class Server:
    """Continuous-batching request loop (fides_server_*): submit() enqueues, wait() blocks."""

    def __init__(self, ctx: "Context", n_streams: int = 2, max_batch: int = 8, hbm_budget_bytes: int = 0):
        self.ctx = ctx
        cfg = _ServerConfig(n_streams, max_batch, hbm_budget_bytes)
        h = vp()
        _check(lib().fides_server_create(ctx._h, C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = []

    def set_relin_key(self, key):
        self._keep.append(key)
        _check(lib().fides_server_set_relin_key(self._h, _ptr(key)))

    def add_rotation_key(self, rotation: int, key):
        self._keep.append(key)
        _check(lib().fides_server_add_rotation_key(self._h, rotation, _ptr(key)))

    def add_bootstrap(self, graph, static_in: Ciphertext, static_out: Ciphertext):
        """Register a bootstrap engine: a torch.cuda.CUDAGraph that bootstraps static_in into
        static_out (see fides_b200.bootstrap.make_engine).  Engines run concurrently."""
        self._keep += [graph, static_in, static_out]
        _check(lib().fides_server_add_bootstrap(self._h, graph.raw_cuda_graph_exec(), _ptr(static_in.c0),
                                                _ptr(static_in.c1), static_in.level, _ptr(static_out.c0),
                                                _ptr(static_out.c1), static_out.level))

    def add_bootstrap_batch(self, graph, static_ins: list, static_outs: list):
        """Register an engine that bootstraps len(static_ins) ciphertexts per graph launch (see
        fides_b200.bootstrap.make_batch_engine); the scheduler fills it from the queue."""
        n = len(static_ins)
        self._keep += [graph, static_ins, static_outs]
        arr = lambda xs: (vp * n)(*xs)
        _check(lib().fides_server_add_bootstrap_batch(
            self._h, graph.raw_cuda_graph_exec(), n, arr([_ptr(c.c0) for c in static_ins]),
            arr([_ptr(c.c1) for c in static_ins]), static_ins[0].level, arr([_ptr(c.c0) for c in static_outs]),
            arr([_ptr(c.c1) for c in static_outs]), static_outs[0].level))

    def set_max_inflight(self, k: int):
        """At most k batches of one operation type on the device at once (0 = n_streams)."""
        _check(lib().fides_server_set_max_inflight(self._h, k))

    def submit(self, op: int, a: Ciphertext, out: Ciphertext, b: Ciphertext | None = None, rotation: int = 0) -> int:
        r = _Request(op, a.level, _ptr(a.c0), _ptr(a.c1), _ptr(b.c0) if b else None, _ptr(b.c1) if b else None,
                     _ptr(out.c0), _ptr(out.c1), rotation)
        t = C.c_uint64()
        _check(lib().fides_server_submit(self._h, C.byref(r), C.byref(t)))
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: float | None = None):
        """(status, latency_ms) of a request; with timeout_ms, raises FidesError TIMEOUT
        when it has not completed in time (the ticket stays valid)."""
        lat, st = C.c_double(), C.c_int()
        if timeout_ms is None:
            _check(lib().fides_server_wait(self._h, ticket, C.byref(lat), C.byref(st)))
        else:
            _check(lib().fides_server_wait_timeout(self._h, ticket, float(timeout_ms), C.byref(lat), C.byref(st)))
        return int(st.value), float(lat.value)

    def stats(self) -> dict:
        s = _ServerStats()
        _check(lib().fides_server_get_stats(self._h, C.byref(s)))
        return {n: int(getattr(s, n)) for n, _ in _ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _check(lib().fides_server_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

