"""Client-side CKKS helpers for tests and benchmarks: encode/decode, key generation,
encryption and decryption, all computed with the CPU oracle.

TEST INFRASTRUCTURE ONLY (it drives the checker and builds synthetic inputs); the
GPU library never imports it.

Conventions (shared with the GPU library's C ABI):
  * ciphertext limbs are limb-major uint64 in EVALUATION (bit-reversed NTT) order;
  * a switching key is [2][dnum][n_q + K][N]: [0] = a (feeds c1), [1] = b (feeds c0);
  * key for digit d encrypts P * s_payload on the digit's Q limbs only (OpenFHE hybrid
    key generation): b_d = -a_d * s_key + e_d + [i in digit d] (P mod q_i) * s_payload;
  * rotation by r uses automorphism index k = 5^(2N - r) mod 2N applied as a scatter
    (reference src/CKKS/RNSPoly.cpp:656, src/Rotation.cuh:14-35), so the rotation key
    encrypts s under tau_k^-1(s) (a gather by the same slot map);
  * encoding: slot j <-> evaluation at zeta^(5^j), zeta = exp(i pi / N).
"""
from __future__ import annotations

import numpy as np

from oracle import Oracle

MASTER_SEED = 20261203


def xrng(stream: int = 0) -> np.random.Generator:
    """Seeded generator for one input stream (master seed xor stream id)."""
    return np.random.default_rng(MASTER_SEED ^ stream)


def uniform_limbs(rng, primes, N) -> np.ndarray:
    return np.stack([rng.integers(0, q, N, dtype=np.uint64) for q in primes])


def small_to_limbs(coeffs: np.ndarray, primes) -> np.ndarray:
    """Signed small integer coefficients -> residues per prime (coefficient domain)."""
    c = np.asarray(coeffs, dtype=np.int64)
    return np.stack([np.where(c < 0, np.uint64(q) - (-c).astype(np.uint64), c.astype(np.uint64)) % np.uint64(q)
                     for q in primes]).astype(np.uint64)


def bigint_to_limbs(values, primes) -> np.ndarray:
    """Python-int (possibly > 2^63) coefficients -> residues per prime."""
    return np.stack([np.array([int(v) % q for v in values], dtype=np.uint64) for q in primes])


def slot_map(N: int):
    """Index t of zeta^(2t+1) for slot j and for its conjugate."""
    M = 2 * N
    e = np.ones(N // 2, dtype=np.int64)
    for j in range(1, N // 2):
        e[j] = (e[j - 1] * 5) % M
    t_pos = (e - 1) // 2
    t_neg = ((M - e) - 1) // 2
    return t_pos, t_neg


def encode(z: np.ndarray, N: int, scale: float) -> np.ndarray:
    """Complex slots (N/2) -> integer coefficients (python ints as object array)."""
    t_pos, t_neg = slot_map(N)
    Mv = np.zeros(N, dtype=np.complex128)
    Mv[t_pos] = z
    Mv[t_neg] = np.conj(z)
    # m_k = (1/N) zeta^-k sum_t M_t omega^-tk, omega = zeta^2
    k = np.arange(N)
    m = np.fft.fft(Mv) / N * np.exp(-1j * np.pi * k / N)
    coeff = np.round(m.real * scale)
    return coeff


def decode(coeff: np.ndarray, N: int, scale: float) -> np.ndarray:
    t_pos, _ = slot_map(N)
    k = np.arange(N)
    # M_t = sum_k (m_k zeta^k) omega^tk
    Mv = np.fft.ifft(np.asarray(coeff, dtype=np.float64) * np.exp(1j * np.pi * k / N)) * N
    return Mv[t_pos] / scale


class KeyGen:
    """Secret key and switching keys over one oracle parameter set."""

    def __init__(self, o: Oracle, seed_stream: int = 1, hamming_weight: int = 0, sigma: float = 3.2):
        self.o = o
        self.rng = xrng(seed_stream)
        self.sigma = sigma
        N = o.N
        if hamming_weight:
            s = np.zeros(N, dtype=np.int64)
            pos = self.rng.choice(N, hamming_weight, replace=False)
            s[pos] = self.rng.choice([-1, 1], hamming_weight)
        else:
            s = self.rng.integers(-1, 2, N).astype(np.int64)
        self.s_coeff = s
        ids = o.ext_ids(o.n_q)
        self.s_eval = o.ntt(small_to_limbs(s, o.primes[:o.n_q] + o.primes[o.n_q:]), ids)

    def _err_eval(self, ids):
        e = np.round(self.rng.normal(0, self.sigma, self.o.N)).astype(np.int64)
        return self.o.ntt(small_to_limbs(e, [self.o.primes[i] for i in ids]), ids)

    def switching_key(self, s_key_eval: np.ndarray, s_payload_eval: np.ndarray) -> np.ndarray:
        """[2][dnum][n_q+K][N] key switching from s_payload to s_key."""
        o = self.o
        ids = o.ext_ids(o.n_q)
        L = len(ids)
        key = np.zeros((2, o.dnum, L, o.N), dtype=np.uint64)
        Pmod = []
        for i in range(o.n_q):
            P = 1
            for pk in o.p:
                P = P * pk % o.q[i]
            Pmod.append(P)
        for d in range(o.dnum):
            a = uniform_limbs(self.rng, [o.primes[i] for i in ids], o.N)
            e = self._err_eval(ids)
            b = o.sub(e, o.mul(a, s_key_eval, ids), ids)
            lo, hi = d * o.alpha, min((d + 1) * o.alpha, o.n_q)
            for i in range(lo, hi):
                pay = o.mul(s_payload_eval[i:i + 1], np.full((1, o.N), Pmod[i], dtype=np.uint64), [i])
                b[i:i + 1] = o.add(b[i:i + 1], pay, [i])
            key[0, d], key[1, d] = a, b
        return key

    def relin_key(self) -> np.ndarray:
        ids = self.o.ext_ids(self.o.n_q)
        s2 = self.o.mul(self.s_eval, self.s_eval, ids)
        return self.switching_key(self.s_eval, s2)

    def rotation_key(self, r: int) -> np.ndarray:
        return self.auto_key(self.o.auto_index(r))

    def auto_key(self, k: int) -> np.ndarray:
        o = self.o
        # tau_k scatters out[sigma(j)] = in[j]; its inverse gathers in[sigma(j)].
        probe = np.arange(o.N, dtype=np.uint64)[None, :]
        sig = o.automorph(probe, k)[0]  # sig[sigma(j)] = j
        inv = np.empty(o.N, dtype=np.int64)
        inv[sig.astype(np.int64)] = np.arange(o.N)  # inv[j] = sigma(j)
        s_key = np.ascontiguousarray(self.s_eval[:, inv])
        return self.switching_key(s_key, self.s_eval)

    def encrypt(self, m_coeff, l: int):
        """Symmetric encryption of integer coefficients at level l -> (c0, c1) EVAL."""
        o = self.o
        ids = o.ids(l)
        primes = o.q[:l]
        m = bigint_to_limbs(m_coeff, primes) if np.asarray(m_coeff).dtype == object else small_to_limbs(m_coeff, primes)
        m_eval = o.ntt(m, ids)
        c1 = uniform_limbs(self.rng, primes, o.N)
        e = self._err_eval(ids)
        c0 = o.add(o.sub(m_eval, o.mul(c1, self.s_eval[:l], ids), ids), e, ids)
        return c0, c1

    def decrypt_limb0(self, c0, c1) -> np.ndarray:
        """Centered coefficients of c0 + c1 s modulo q_0 (valid while |m| < q_0 / 2)."""
        o = self.o
        m = o.add(c0[:1], o.mul(c1[:1], self.s_eval[:1], [0]), [0])
        m = o.ntt(m, [0], inverse=True)[0].astype(object)
        q0 = o.q[0]
        return np.array([int(v) - q0 if int(v) > q0 // 2 else int(v) for v in m], dtype=np.float64)
