"""CKKS bootstrapping on the B200 core: ModRaise -> CoeffsToSlots -> EvalMod -> SlotsToCoeffs.

Mirrors the reference's CKKS::Bootstrap (src/CKKS/Bootstrap.cu:437-648): ModRaise (:708+),
EvalCoeffsToSlots / EvalLinearTransform (src/CKKS/CoeffsToSlots.cu:26-151, BSGS linear
transforms in src/CKKS/LinearTransform.cu), approxModReduction with a Chebyshev series and
double-angle iterations (src/CKKS/ApproxModEval.cu:45-167, :527, :873).  OpenFHE's own
coefficient tables are not available, so every table here is derived from the mathematics:

  * Slots.  Slot j of a plaintext m(X) at scale S is m(zeta^(5^j)) / S, zeta = exp(i pi / N);
    with w_k = m_k + i m_(k+N/2) this is z = U0 w / S, U0[j, k] = zeta^(5^j k), n = N/2 slots,
    and U0^H U0 = n I.
  * Special FFT.  z = U0 w is a radix-2 decimation-in-time transform on bit-reversed input:
    z = F (P w), F = S_(n/2) ... S_2 S_1, where S_h combines entries p, p + h of each block of
    2h with the twiddle rho^(5^r), rho = exp(i pi / (4h)), r = p mod h.  Each S_h has three
    slot diagonals (offsets 0, +h, -h), so CoeffsToSlots applies F^-1 = S_1^-1 ... S_(n/2)^-1
    and SlotsToCoeffs applies F, each grouped into a few levels of composed diagonals
    evaluated baby-step / giant-step with hoisted rotations.  Data stay in bit-reversed
    order between the two transforms; everything in between is slot-wise.
  * EvalMod.  After CoeffsToSlots the real slots hold t = m'_k / (K q0), m' = m + q0 I; the
    Chebyshev interpolant of cos(2 pi K t / 2^r - pi / 2^(r+1)) on [-1, 1] followed by r
    double-angle steps c <- 2 c^2 - 1 gives sin(2 pi m'_k / q0) = sin(2 pi m_k / q0).
  * Scales.  Level l has scale S_l with S_(l-1) = S_l^2 / q_(l-1) (products of two level-l
    ciphertexts land exactly on the next level's scale); a ciphertext moved down several
    levels is first multiplied by an integer constant that re-targets its scale.
"""
from __future__ import annotations

import math

import numpy as np


# ------------------------------------------------------------------------------ encoding
def encode_coeffs(z: np.ndarray, N: int, scale: float) -> np.ndarray:
    """Complex slot vector (N/2) -> integer coefficients (int64) of m with m(zeta^(5^j)) = scale z_j."""
    n = N // 2
    M = 2 * N
    e = np.empty(n, dtype=np.int64)
    e[0] = 1
    for j in range(1, n):
        e[j] = (e[j - 1] * 5) % M
    t_pos = (e - 1) // 2
    t_neg = ((M - e) - 1) // 2
    Mv = np.zeros(N, dtype=np.complex128)
    Mv[t_pos] = z
    Mv[t_neg] = np.conj(z)
    k = np.arange(N)
    m = np.fft.fft(Mv) / N * np.exp(-1j * np.pi * k / N)
    c = np.round(m.real * scale)
    if np.abs(c).max() >= 2.0 ** 62:
        raise ValueError("encoded coefficients exceed 62 bits")
    return c.astype(np.int64)


def decode_coeffs(coeff: np.ndarray, N: int, scale: float) -> np.ndarray:
    n = N // 2
    M = 2 * N
    e = np.empty(n, dtype=np.int64)
    e[0] = 1
    for j in range(1, n):
        e[j] = (e[j - 1] * 5) % M
    k = np.arange(N)
    Mv = np.fft.ifft(np.asarray(coeff, dtype=np.float64) * np.exp(1j * np.pi * k / N)) * N
    return Mv[(e - 1) // 2] / scale


def to_limbs(coeff: np.ndarray, primes) -> np.ndarray:
    c = np.asarray(coeff, dtype=np.int64)
    return np.stack([np.mod(c, np.int64(q)).astype(np.uint64) for q in primes])


def bit_reverse_perm(n: int) -> np.ndarray:
    b = n.bit_length() - 1
    return np.array([int(format(i, f"0{b}b")[::-1], 2) if b else 0 for i in range(n)], dtype=np.int64)


# ------------------------------------------------------------------------------ special FFT
def stage(n: int, h: int, inverse: bool) -> dict[int, np.ndarray]:
    """Slot diagonals of S_h (or S_h^-1): out = sum_r D_r * roll(a, -r)."""
    p = np.arange(n)
    r = p % (2 * h)
    lo = r < h
    idx = np.where(lo, r, r - h)
    e = np.array([pow(5, int(i), 8 * h) for i in range(h)], dtype=np.float64)
    tw = np.exp(1j * np.pi * e / (4 * h))[idx]
    d0 = np.zeros(n, dtype=np.complex128)
    dp = np.zeros(n, dtype=np.complex128)
    dm = np.zeros(n, dtype=np.complex128)
    if not inverse:
        # lo: a[p] + tw a[p+h]; hi: a[p-h] - tw a[p]
        d0[lo] = 1
        dp[lo] = tw[lo]
        d0[~lo] = -tw[~lo]
        dm[~lo] = 1
    else:
        # lo: (a[p] + a[p+h]) / 2; hi: (a[p-h] - a[p]) / (2 tw)
        d0[lo] = 0.5
        dp[lo] = 0.5
        d0[~lo] = -0.5 / tw[~lo]
        dm[~lo] = 0.5 / tw[~lo]
    out = {0: d0}
    if h < n:
        out[h % n] = out.get(h % n, 0) + dp
        out[(-h) % n] = out.get((-h) % n, 0) + dm
    return out


def compose(A: dict[int, np.ndarray], B: dict[int, np.ndarray], n: int) -> dict[int, np.ndarray]:
    """Diagonals of A @ B: (A B) v = sum_{r,s} (A_r * roll(B_s, -r)) * roll(v, -(r + s))."""
    out: dict[int, np.ndarray] = {}
    for r, Ar in A.items():
        for s, Bs in B.items():
            k = (r + s) % n
            out[k] = out.get(k, 0) + Ar * np.roll(Bs, -r)
    return {k: v for k, v in out.items() if np.abs(v).max() > 0}


def apply_diags(D: dict[int, np.ndarray], v: np.ndarray) -> np.ndarray:
    return sum(d * np.roll(v, -r) for r, d in D.items())


def fft_levels(n: int, n_levels: int, inverse: bool, unnormalized: bool = False) -> list[dict[int, np.ndarray]]:
    """F (or F^-1) as `n_levels` composed matrices, in application order.  With
    `unnormalized`, the inverse stages are 2 S_h^-1 (unit-modulus entries), i.e. the product
    is n F^-1."""
    hs = [1 << i for i in range(n.bit_length() - 1)]  # S_1 .. S_(n/2)
    order = hs if not inverse else hs[::-1]           # F applies S_1 first; F^-1 applies S_(n/2)^-1 first
    groups = np.array_split(np.arange(len(order)), n_levels)
    mats = []
    for g in groups:
        M = None
        for i in g:
            S = stage(n, order[i], inverse)
            if inverse and unnormalized:
                S = {k: 2 * v for k, v in S.items()}
            M = S if M is None else compose(S, M, n)  # later stages on the left
        mats.append(M)
    return mats


# ------------------------------------------------------------------------------ evaluator
class Ct:
    """Ciphertext handle with its scale (level = number of limbs)."""

    def __init__(self, c0, c1, scale: float):
        self.c0, self.c1, self.scale = c0, c1, scale

    @property
    def level(self) -> int:
        return int(self.c0.shape[0])


class Evaluator:
    """CKKS arithmetic with exact per-level scale bookkeeping over the GPU core."""

    def __init__(self, F, ctx, relin_key, rot_keys: dict, conj_key, top_scale: float):
        self.F, self.ctx, self.rk = F, ctx, relin_key
        self.rot_keys, self.conj_key = rot_keys, conj_key
        self.q = ctx.q
        L = ctx.n_q
        self.S = [0.0] * (L + 1)
        self.S[L] = top_scale
        for l in range(L, 1, -1):
            self.S[l - 1] = self.S[l] ** 2 / self.q[l - 1]

    # -- level / scale management --
    def drop(self, a: Ct, level: int) -> Ct:
        """Discard limbs (the value is kept modulo the smaller modulus; scale unchanged)."""
        return Ct(a.c0[:level], a.c1[:level], a.scale)

    def to_level(self, a: Ct, level: int) -> Ct:
        """Bring `a` to `level` at that level's canonical scale S_level."""
        return self.to_level_many([a], level)[0]

    def to_level_many(self, cts: list, level: int) -> list:
        """to_level on several ciphertexts of one level and scale: discard down to level + 1
        limbs, multiply by the integer c with scale * c / q_level = S_level, rescale by q_level
        (one combination launch and one batched rescale for all of them)."""
        a = cts[0]
        if a.level == level and abs(a.scale / self.S[level] - 1) < 1e-15:
            return list(cts)
        if a.level <= level:
            raise ValueError(f"cannot raise level {a.level} -> {level}")
        c = round(self.S[level] * self.q[level] / a.scale)
        return self._rescale_many_to(self.lincomb_many([[self.drop(b, level + 1)] for b in cts], [c]), self.S[level])

    def _rescale_to(self, a: Ct, new_scale: float) -> Ct:
        return self._rescale_many_to([a], new_scale)[0]

    def _rescale_many_to(self, cts: list, new_scale: float) -> list:
        outs = self.ctx.rescale_many([p for a in cts for p in (a.c0, a.c1)])
        return [Ct(outs[2 * i], outs[2 * i + 1], new_scale) for i in range(len(cts))]

    def rescale(self, a: Ct) -> Ct:
        return self._rescale_to(a, a.scale / self.q[a.level - 1])

    # -- arithmetic --
    def add(self, a: Ct, b: Ct) -> Ct:
        l = min(a.level, b.level)
        a = self.to_level(a, l) if (a.level != l or abs(a.scale / self.S[l] - 1) > 1e-12) else a
        b = self.to_level(b, l) if (b.level != l or abs(b.scale / self.S[l] - 1) > 1e-12) else b
        return Ct(self.ctx.add_poly(a.c0, b.c0), self.ctx.add_poly(a.c1, b.c1), a.scale)

    def add_raw(self, a: Ct, b: Ct) -> Ct:
        """a + b for operands already at the same level and scale."""
        return Ct(self.ctx.add_poly(a.c0, b.c0), self.ctx.add_poly(a.c1, b.c1), a.scale)

    def sub_raw(self, a: Ct, b: Ct) -> Ct:
        return Ct(self.ctx.sub_poly(a.c0, b.c0), self.ctx.sub_poly(a.c1, b.c1), a.scale)

    def add_const(self, a: Ct, value: float) -> Ct:
        v = round(value * a.scale)
        return Ct(self.ctx.add_scalar_poly(a.c0, [v % q for q in self.q[:a.level]]), a.c1, a.scale)

    def lincomb(self, terms, const: float = 0.0) -> Ct:
        """sum_t c_t * a_t + const for integer c_t, operands at one level and scale (one
        launch; the scale is kept)."""
        return self.lincomb_many([[a for a, _ in terms]], [c for _, c in terms], const)[0]

    def lincomb_many(self, lanes: list, ints: list, const: float = 0.0) -> list:
        """The same integer combination sum_t ints[t] * lane[t] + const on every lane (a list of
        ciphertexts of one level and scale per lane): one launch for all lanes."""
        a = lanes[0][0]
        l = min(b.level for lane in lanes for b in lane)
        add = round(const * a.scale) if const else None
        outs = self.ctx.lincomb_lanes(lanes, ints, add0=add, level=l)
        return [Ct(o.c0, o.c1, a.scale) for o in outs]

    def add_many(self, xs: list, ys: list) -> list:
        """x + y lane by lane (same level and scale), one launch."""
        return self.lincomb_many([[x, y] for x, y in zip(xs, ys)], [1, 1])

    def lincomb_to(self, terms, const: float, target: int) -> Ct:
        return self.lincomb_to_many([[a for a, _ in terms]], [v for _, v in terms], const, target)[0]

    def lincomb_to_many(self, lanes: list, coefs: list, const: float, target: int) -> list:
        """sum_t coefs[t] * lane[t] + const for real coefficients, landing at `target` limbs
        with scale S_target on every lane: operand t (any level > target, any scale, the same
        on every lane) is read on its first target + 1 limbs and multiplied by the integer
        round(coefs[t] S_target q_target / scale_t); the sum is rescaled by q_target (one
        combination launch and one batched rescale for all lanes)."""
        qt, S = self.q[target], self.S[target]
        keep, ints = [], []
        for t, v in enumerate(coefs):
            a = lanes[0][t]
            if a.level <= target:
                raise ValueError(f"operand at level {a.level} cannot land at level {target}")
            c = round(v * S * qt / a.scale)
            if c:
                keep.append(t)
                ints.append(c)
        if not keep:  # constant only: a zero combination of the first operand carries it
            keep, ints = [0], [0]
        add = round(const * S * qt)
        outs = self.ctx.lincomb_lanes([[lane[t] for t in keep] for lane in lanes], ints,
                                      add0=add if add else None, level=target + 1)
        return self._rescale_many_to([Ct(o.c0, o.c1, 0.0) for o in outs], S)

    def mul_many(self, pairs) -> list[Ct]:
        """a * b (relinearised, rescaled) for several pairs in one batched launch sequence;
        each pair is brought to its lower level first."""
        F = self.F
        ab = []
        for a, b in pairs:
            l = min(a.level, b.level)
            ab.append((self.to_level(a, l), self.to_level(b, l)))
        outs = self.ctx.mult_batch([(F.Ciphertext(a.c0, a.c1), F.Ciphertext(b.c0, b.c1)) for a, b in ab], self.rk)
        return [Ct(o.c0, o.c1, self.S[a.level - 1]) for o, (a, _) in zip(outs, ab)]

    def mul_int(self, a: Ct, c: int) -> Ct:
        vals = [c % q for q in self.q[:a.level]]
        return Ct(self.ctx.mul_scalar_poly(a.c0, vals), self.ctx.mul_scalar_poly(a.c1, vals), a.scale)

    def mul_const(self, a: Ct, value: float, target_level: int) -> Ct:
        """value * a, landing at `target_level` (< a.level) with scale S_target."""
        qt = self.q[a.level - 1]
        c = round(value * self.S[target_level] * qt / a.scale)
        b = self.mul_int(a, c)
        b = self._rescale_to(b, self.S[target_level])
        return self.drop(b, target_level)

    def mul(self, a: Ct, b: Ct) -> Ct:
        l = min(a.level, b.level)
        a = self.to_level(a, l)
        b = self.to_level(b, l)
        out = self.ctx.mult(self.F.Ciphertext(a.c0, a.c1), self.F.Ciphertext(b.c0, b.c1), self.rk, rescale=True)
        return Ct(out.c0, out.c1, self.S[l - 1])

    def square(self, a: Ct) -> Ct:
        return self.mul(a, a)

    def mul_plain(self, a: Ct, pt, pt_scale: float) -> Ct:
        """a * pt (EVAL limbs at a.level), then rescale."""
        c0 = self.ctx.mul_poly(a.c0, pt[:a.level])
        c1 = self.ctx.mul_poly(a.c1, pt[:a.level])
        return self._rescale_to(Ct(c0, c1, 0), a.scale * pt_scale / self.q[a.level - 1])

    def mul_plain_int(self, a: Ct, pt) -> Ct:
        """a * pt for an integer plaintext (scale 1), no rescale."""
        return Ct(self.ctx.mul_poly(a.c0, pt[:a.level]), self.ctx.mul_poly(a.c1, pt[:a.level]), a.scale)

    def conjugate(self, a: Ct) -> Ct:
        k = 2 * self.ctx.N - 1
        out = self.ctx.rotate_auto(self.F.Ciphertext(a.c0, a.c1), self.conj_key, k)
        return Ct(out.c0, out.c1, a.scale)

    def rotate_many(self, a: Ct, rs: list[int]) -> list[Ct]:
        rs2 = [r for r in rs if r % (self.ctx.N // 2) != 0]
        res = {}
        if rs2:
            outs = self.ctx.rotate_hoisted(self.F.Ciphertext(a.c0, a.c1), [self.rot_keys[r] for r in rs2], rs2)
            res = {r: Ct(o.c0, o.c1, a.scale) for r, o in zip(rs2, outs)}
        return [a if r % (self.ctx.N // 2) == 0 else res[r] for r in rs]

    def rotate(self, a: Ct, r: int) -> Ct:
        return self.rotate_many(a, [r])[0]

    def rotate_batch(self, jobs) -> list[Ct]:
        """Rotations of several ciphertexts (jobs: (ciphertext, rotation), rotation != 0 mod
        slots) in one batched key switch."""
        if not jobs:
            return []
        F = self.F
        outs = self.ctx.rotate_batch([(F.Ciphertext(a.c0, a.c1), self.rot_keys[r], r) for a, r in jobs])
        return [Ct(o.c0, o.c1, a.scale) for o, (a, _) in zip(outs, jobs)]


# ------------------------------------------------------------------------------ bootstrapper
class Bootstrapper:
    """Precomputed CoeffsToSlots / SlotsToCoeffs diagonals and EvalMod constants."""

    def __init__(self, ev: Evaluator, K: int = 12, r: int = 3, degree: int = 31, cts_levels: int = 3,
                 stc_levels: int = 3, baby: int = 8, prescale_bits: int = 0, encapsulation=None):
        self.ev = ev
        # sparse-secret encapsulation (Bootstrap.cu keySwitchSparse): device switching keys
        # (dense -> sparse, sparse -> dense).  The level-1 input is switched to the sparse
        # secret before ModRaise, so the overflow I of ModRaise stays small, and switched
        # back right after it, so CoeffsToSlots / EvalMod / SlotsToCoeffs run under the dense
        # secret with its ordinary keys.  None: the input is already under a sparse secret.
        self.encapsulation = encapsulation
        ctx = ev.ctx
        self.N = ctx.N
        self.n = self.N // 2
        self.K, self.r, self.degree = K, r, degree
        # the input is multiplied by 2^prescale_bits before ModRaise so that the message fills
        # more of q0 (a correction factor); SlotsToCoeffs divides it back out
        self.prescale = 1 << prescale_bits
        self.cts_levels, self.stc_levels, self.baby = cts_levels, stc_levels, baby
        self.q0 = ctx.q[0]
        # Chebyshev interpolant of cos(2 pi K t / 2^r - pi / 2^(r+1)) on [-1, 1]
        f = lambda t: np.cos(2 * np.pi * K * t / 2 ** r - np.pi / 2 ** (r + 1))
        self.cheb = np.polynomial.chebyshev.chebinterpolate(f, degree)
        self.cts = fft_levels(self.n, cts_levels, inverse=True, unnormalized=True)
        self.stc = fft_levels(self.n, stc_levels, inverse=False)
        self.rotations = sorted({r for M in self.cts + self.stc for r in self._bsgs_rotations(M)} - {0})
        self.pt_int = {}

    # --- BSGS plan of one composed matrix
    def _plan(self, M: dict):
        n, g = self.n, self.baby
        offs = sorted(M)
        step = math.gcd(*[o for o in offs if o] + [n]) if any(offs) else n
        ts = sorted({((o + n // 2) % n - n // 2) // step for o in offs})  # signed multiples of step
        giant = {}
        for t in ts:
            i, j = divmod(t, g)
            giant.setdefault(i, []).append(j)
        return step, giant

    def _bsgs_rotations(self, M: dict):
        step, giant = self._plan(M)
        g = self.baby
        rs = {step * j for js in giant.values() for j in js}
        rs |= {step * g * i for i in giant}
        return {r % self.n for r in rs}

    def needed_rotations(self) -> list[int]:
        return self.rotations

    # --- plaintext preparation (encoding on the GPU: torch FFT, then the library's NTT)
    def _encode_pt(self, z, level: int, scale: float):
        """Slots -> EVALUATION-form plaintext on the device (fides_encode)."""
        import torch
        return self.ev.ctx.encode(torch.from_numpy(np.ascontiguousarray(z, dtype=np.complex128)), scale, level)

    def _int_pt(self, coeff, level: int):
        F, ctx = self.ev.F, self.ev.ctx
        limbs = F.to_device(to_limbs(coeff, ctx.q[:level]))
        ctx.ntt(limbs)
        return limbs

    def prepare(self, top_level: int, msg_scale: float):
        """Encode the transform diagonals for a bootstrap raising to `top_level`, for input
        ciphertexts whose slots are encoded at `msg_scale`."""
        ev, n = self.ev, self.n
        in_scale = ev.S[top_level]  # the scale given to the raised ciphertext (free choice)
        msg_scale = msg_scale * self.prescale
        self.top, self.in_scale, self.msg_scale = top_level, in_scale, msg_scale
        # CoeffsToSlots: slots -> c' P w / S with c' = S / (2 K q0).  The matrices are the
        # unnormalised stages (product n F^-1, unit-modulus entries) and the factor c' / n is
        # spread evenly over them, so every encoded diagonal keeps ~42 significant bits.
        gfac = (in_scale / (2 * self.K * self.q0) / n) ** (1.0 / len(self.cts))
        self.cts_pts = []
        level, scale = top_level, in_scale
        for m, M in enumerate(self.cts):
            self.cts_pts.append(self._prepare_matrix(M, gfac, level, scale))
            level -= 1
            scale = ev.S[level]
        self.cts_out_level = level
        # EvalMod levels: ceil(log2 degree) + 1 (series sum) + r (double angle)
        depth = math.ceil(math.log2(self.degree)) + 1 + self.r
        self.stc_in_level = self.cts_out_level - depth
        # SlotsToCoeffs: c'' = q0 / (2 pi msg_scale), spread evenly over the matrices
        sfac = (self.q0 / (2 * np.pi * msg_scale)) ** (1.0 / len(self.stc))
        self.stc_pts = []
        level = self.stc_in_level
        for m, M in enumerate(self.stc):
            fac = sfac
            self.stc_pts.append(self._prepare_matrix(M, fac, level, ev.S[level]))
            level -= 1
        self.out_level = level
        N = self.N
        mono = np.zeros(N, dtype=np.int64)
        mono[N // 2] = 1  # X^(N/2): slots * i
        self.pt_i = self._int_pt(mono, top_level)
        self.pt_minus_i = self._int_pt(-mono, top_level)
        if ev.ctx.device_status(clear=False) & 2:
            raise ValueError("an encoded diagonal coefficient exceeded 2^62 in magnitude")

    def _prepare_matrix(self, M: dict, fac: float, level: int, scale: float):
        """Pre-rotated, encoded diagonals for BSGS at `level` (input scale `scale`)."""
        ev, n, g = self.ev, self.n, self.baby
        step, giant = self._plan(M)
        target = ev.S[level - 1]
        pt_scale = target * ev.q[level - 1] / scale  # so that rescale lands on S_(level-1)
        out = {}
        for i, js in giant.items():
            for j in js:
                off = (step * (g * i + j)) % n
                d = M.get(off)
                if d is None:
                    continue
                d = np.roll(d * fac, step * g * i)  # rot^{-g i}(D)
                out[(i, j)] = self._encode_pt(d, level, pt_scale)
        return {"step": step, "giant": giant, "pts": out, "pt_scale": pt_scale, "level": level}

    # --- homomorphic linear transform
    def _apply(self, a: Ct, P: dict) -> Ct:
        ev, g = self.ev, self.baby
        step, giant = P["step"], P["giant"]
        assert a.level == P["level"], (a.level, P["level"])
        js = sorted({j for v in giant.values() for j in v})
        baby = dict(zip(js, ev.rotate_many(a, [(step * j) % self.n for j in js])))
        parts, turns = [], []
        for i, jl in sorted(giant.items()):
            terms = [(baby[j], P["pts"][(i, j)]) for j in jl if (i, j) in P["pts"]]
            if not terms:
                continue
            inner = None
            for k in range(0, len(terms), 32):  # one fused launch per 32 diagonals
                chunk = terms[k:k + 32]
                d = ev.ctx.dot_plain([t[0] for t in chunk], [t[1] for t in chunk], level=a.level)
                d = Ct(d.c0, d.c1, a.scale)
                inner = d if inner is None else ev.add_many([inner], [d])[0]
            r = (step * g * i) % self.n
            (turns if r else parts).append((inner, r))
        # every giant-step rotation in one batched key switch, then one sum and one rescale
        parts = [p for p, _ in parts] + ev.rotate_batch(turns)
        while len(parts) > 1:
            parts = [ev.lincomb_many([parts[k:k + 16]], [1] * len(parts[k:k + 16]))[0] if len(parts[k:k + 16]) > 1
                     else parts[k] for k in range(0, len(parts), 16)]
        return ev._rescale_to(parts[0], ev.S[a.level - 1])

    # --- EvalMod
    # Paterson-Stockmeyer leaves: Chebyshev series of degree < 16.  The error of a power
    # computed by doubling grows ~4x per doubling (T_8 is 2 bits worse than T_4), and with
    # leaves of degree < 8 the large coefficients c_8..c_15 of the EvalMod cosine would ride on
    # the error of T_8 (1.2 bits lost at N = 2^16); with 16 they multiply powers computed
    # directly, as in a term-by-term sum, at 3 more HMults.
    PS_BABY = 16

    def _cheb_powers(self, ts: list) -> dict:
        """T_1..T_16 and the giant powers T_32, T_64, ... (<= degree) of every lane, each at its
        natural level: T_2k = 2 T_k^2 - 1, T_2k+1 = 2 T_k T_k+1 - T_1 (one batched HMult and
        one combination launch over the lanes per power)."""
        ev = self.ev
        T = {1: list(ts)}

        def make(k):
            if k % 2 == 0:
                x = ev.mul_many([(a, a) for a in T[k // 2]])
                T[k] = ev.lincomb_many([[p] for p in x], [2], const=-1.0)
            else:
                x = ev.mul_many(list(zip(T[k // 2], T[k // 2 + 1])))
                one = self._t_at(T, 1, x[0].level)
                T[k] = ev.lincomb_many([[p, o] for p, o in zip(x, one)], [2, -1])

        for k in range(2, self.PS_BABY + 1):
            make(k)
        m = 2 * self.PS_BABY
        while m <= self.degree:
            make(m)
            m *= 2
        return T

    def _t_at(self, T: dict, k: int, level: int) -> list:
        """T_k of every lane brought to `level` at its canonical scale (cached)."""
        cache = T.setdefault("at", {})
        if (k, level) not in cache:
            cache[(k, level)] = self.ev.to_level_many(T[k], level)
        return cache[(k, level)]

    def _ps(self, coeffs: np.ndarray, level_out: int, T: dict, lanes: int) -> list:
        """Chebyshev series sum_i coeffs[i] T_i at `level_out` (scale S_level_out) by
        Paterson-Stockmeyer (innerEvalChebyshevPS, src/CKKS/ApproxModEval.cu:341): split
        p = q T_m + r at the largest power of two m < deg p + 1 using T_(m+j) = 2 T_m T_j - T_(m-j);
        q lands one level higher and is multiplied by T_m, r lands at level_out; series of degree
        < PS_BABY are one weighted sum of T_0..T_(PS_BABY-1) (evalPartialLinearWSum,
        ApproxModEval.cu:328)."""
        ev, n = self.ev, len(coeffs)
        if n <= self.PS_BABY:
            ks = list(range(1, n)) or [1]
            cf = [float(coeffs[k]) if k < n else 0.0 for k in ks]
            return ev.lincomb_to_many([[T[k][i] for k in ks] for i in range(lanes)], cf, float(coeffs[0]), level_out)
        m = 1 << ((n - 1).bit_length() - 1)
        q = np.zeros(n - m)
        r = np.array(coeffs[:m], dtype=np.float64)
        q[0] = coeffs[m]
        for j in range(1, n - m):
            q[j] = 2 * coeffs[m + j]
            r[m - j] -= coeffs[m + j]
        qc = self._ps(q, level_out + 1, T, lanes)
        prod = ev.mul_many(list(zip(qc, self._t_at(T, m, level_out + 1))))
        rc = self._ps(r, level_out, T, lanes)
        return ev.add_many(prod, rc)

    def _chebyshev_many(self, ts: list) -> list:
        """The EvalMod series at every lane (one ciphertext per lane, same level and scale)."""
        T = self._cheb_powers(ts)
        depth = math.ceil(math.log2(self.degree)) + 1
        return self._ps(np.asarray(self.cheb, dtype=np.float64), ts[0].level - depth, T, len(ts))

    def _chebyshev(self, t: Ct) -> Ct:
        return self._chebyshev_many([t])[0]

    def _eval_mod_many(self, ts: list) -> list:
        """EvalMod (Chebyshev series of the scaled cosine, then r double-angle steps
        c -> 2 c^2 - 1) on several ciphertexts at once, each step batched over them."""
        ev = self.ev
        cs = self._chebyshev_many(ts)
        for _ in range(self.r):
            cs = ev.lincomb_many([[x] for x in ev.mul_many([(c, c) for c in cs])], [2], const=-1.0)
        return cs

    def _eval_mod(self, t: Ct) -> Ct:
        return self._eval_mod_many([t])[0]

    # --- the bootstrap
    def _switch(self, a: Ct, key) -> Ct:
        """(c0, c1) under the key's payload secret -> (c0 + f0, f1) under its target secret."""
        f0, f1 = self.ev.ctx.keyswitch(a.c1, key)
        return Ct(self.ev.ctx.add_poly(a.c0, f0), f1, a.scale)

    def bootstrap(self, ct: Ct) -> Ct:
        ev = self.ev
        F = ev.F
        x = Ct(ct.c0[:1], ct.c1[:1], ct.scale)
        if self.encapsulation:
            x = self._switch(x, self.encapsulation[0])  # dense -> sparse, at level 1
        if self.prescale != 1:
            x = ev.mul_int(x, self.prescale)
        # ModRaise: m -> m + q0 I at every limb of the top level
        a = Ct(ev.ctx.mod_raise_poly(x.c0[:1], self.top), ev.ctx.mod_raise_poly(x.c1[:1], self.top), self.in_scale)
        if self.encapsulation:
            a = self._switch(a, self.encapsulation[1])  # sparse -> dense, at the top level
        # CoeffsToSlots
        for P in self.cts_pts:
            a = self._apply(a, P)
        # real / imaginary parts: t_re = a + conj(a), t_im = -i (a - conj(a))
        cj = ev.conjugate(a)
        t_re = ev.add_raw(a, cj)
        t_im = ev.mul_plain_int(ev.sub_raw(a, cj), self.pt_minus_i)
        # EvalMod on both, then recombine u = s_re + i s_im
        s_re, s_im = self._eval_mod_many([t_re, t_im])
        s_re = ev.to_level(s_re, self.stc_in_level)
        s_im = ev.to_level(s_im, self.stc_in_level)
        u = ev.add_raw(s_re, ev.mul_plain_int(s_im, self.pt_i))
        # SlotsToCoeffs
        for P in self.stc_pts:
            u = self._apply(u, P)
        return u


def bootstrap_concurrent(bs: Bootstrapper, cts: list, streams=None) -> list:
    """Bootstrap several ciphertexts at once, each on its own CUDA stream forked from and
    joined back to the current stream, so that their kernels overlap on the device (one
    bootstrap at N = 2^16 spends most of its time at low levels, where a single ciphertext
    fills few SMs).  Captured inside torch.cuda.graph, the batch becomes one graph with a
    parallel branch per ciphertext.  Results are those of bs.bootstrap, ciphertext by
    ciphertext."""
    import torch
    main = torch.cuda.current_stream()
    streams = streams or [torch.cuda.Stream() for _ in cts]
    outs = [None] * len(cts)
    for i, (ct, s) in enumerate(zip(cts, streams)):
        s.wait_stream(main)
        with torch.cuda.stream(s):
            outs[i] = bs.bootstrap(ct)
    for s in streams:
        main.wait_stream(s)
    for o in outs:  # the outputs are handed to the current stream
        o.c0.record_stream(main)
        o.c1.record_stream(main)
    return outs


def make_engine(bs: Bootstrapper, scale: float):
    """A bootstrap engine for the request loop (fides_server_add_bootstrap): static device
    buffers for a one-limb input ciphertext (bootstrapping reads limb 0 only) and a CUDA
    graph, captured once, that bootstraps them into a static output.  Returns (graph,
    static input, static output) as (torch.cuda.CUDAGraph, Ciphertext, Ciphertext); the
    graph's private memory pool keeps every intermediate resident."""
    import torch
    F, ctx = bs.ev.F, bs.ev.ctx
    c0, c1 = ctx.empty(1), ctx.empty(1)
    c0.view(torch.int64).zero_()
    c1.view(torch.int64).zero_()
    static = Ct(c0, c1, scale)
    bs.bootstrap(static)  # warm-up outside the capture (lazy kernel loading, tables)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        out = bs.bootstrap(static)
    torch.cuda.synchronize()
    return g, F.Ciphertext(c0, c1), F.Ciphertext(out.c0, out.c1)


def make_batch_engine(bs: Bootstrapper, scale: float, capacity: int):
    """A bootstrap engine holding `capacity` ciphertexts (fides_server_add_bootstrap_batch): one
    CUDA graph, captured once, that bootstraps `capacity` static one-limb inputs on parallel
    branches (bootstrap_concurrent) into static outputs.  Returns (graph, inputs, outputs)."""
    import torch
    F, ctx = bs.ev.F, bs.ev.ctx
    ins = []
    for _ in range(capacity):
        c0, c1 = ctx.empty(1), ctx.empty(1)
        c0.view(torch.int64).zero_()
        c1.view(torch.int64).zero_()
        ins.append(Ct(c0, c1, scale))
    streams = [torch.cuda.Stream() for _ in range(capacity)]
    bootstrap_concurrent(bs, ins, streams)  # warm-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        outs = bootstrap_concurrent(bs, ins, streams)
    torch.cuda.synchronize()
    return (g, [F.Ciphertext(c.c0, c.c1) for c in ins], [F.Ciphertext(o.c0, o.c1) for o in outs])


def make_native_engine(nb, capacity: int = 1):
    """A bootstrap engine for the request loop backed by the library's C++ bootstrapper
    (NativeBootstrapper): `capacity` static one-limb inputs and one CUDA graph, captured once,
    that bootstraps them into static outputs -- fides_bootstrap for capacity 1,
    fides_bootstrap_batch (the whole batch in one launch sequence) otherwise.  Returns
    (graph, input, output) for capacity 1 (Server.add_bootstrap) and (graph, inputs, outputs)
    otherwise (Server.add_bootstrap_batch)."""
    import torch
    from . import Ciphertext
    ctx = nb.ctx
    ins = []
    for _ in range(capacity):
        c0, c1 = ctx.empty(1), ctx.empty(1)
        c0.view(torch.int64).zero_()
        c1.view(torch.int64).zero_()
        ins.append(Ciphertext(c0, c1))
    run = (lambda: [nb.bootstrap(ins[0])]) if capacity == 1 else (lambda: nb.bootstrap_batch(ins))
    run()  # warm-up outside the capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        outs = run()
    torch.cuda.synchronize()
    return (g, ins[0], outs[0]) if capacity == 1 else (g, ins, outs)
