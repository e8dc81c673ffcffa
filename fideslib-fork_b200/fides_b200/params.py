"""Parameter sets of the CKKS evaluation path and their deterministic moduli.

Moduli are NTT-friendly primes q = 1 (mod 2N) found by a descending search from 2^bits
(OpenFHE's own prime choice is not reproducible without OpenFHE; this rule is the
documented synthetic stand-in).  Special-prime count K follows the reference's sizing
rule (src/CKKS/Context.cu:355-370) unless a configuration fixes it.
"""
from __future__ import annotations

from dataclasses import dataclass, field


def _powmod(a, e, m):
    return pow(a, e, m)


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = _powmod(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def gen_primes(logN: int, bits: int, count: int, exclude=()) -> list[int]:
    m = 2 << logN
    q = ((1 << bits) // m) * m + 1
    if q >= 1 << bits:
        q -= m
    out, ex = [], set(exclude)
    while len(out) < count and q > m:
        if q not in ex and is_prime(q):
            out.append(q)
        q -= m
    if len(out) != count:
        raise ValueError("not enough primes")
    return out


def special_count(q_bits: list[int], dnum: int, p_bits: int) -> int:
    """Reference K sizing: sum(bits(p_k) - 1) >= bits of the largest digit (Context.cu:355-370)."""
    alpha = -(-len(q_bits) // dnum)
    digits = [sum(q_bits[i:i + alpha]) for i in range(0, len(q_bits), alpha)]
    need, k, have = max(digits), 0, 0
    while have < need:
        k += 1
        have += p_bits - 1
    return k


@dataclass
class CKKSParams:
    name: str
    logN: int
    q: list[int]
    p: list[int]
    dnum: int
    notes: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def N(self) -> int:
        return 1 << self.logN

    @property
    def n_q(self) -> int:
        return len(self.q)

    @property
    def K(self) -> int:
        return len(self.p)

    @property
    def alpha(self) -> int:
        return -(-self.n_q // self.dnum)


def chain(logN: int, first_bits: int, scale_bits: int, n_q: int, dnum: int, K: int | None = None,
          p_bits: int = 61, name: str = "") -> CKKSParams:
    q = gen_primes(logN, first_bits, 1)
    q += gen_primes(logN, scale_bits, n_q - 1, exclude=q)
    if K is None:
        K = special_count([x.bit_length() for x in q], dnum, p_bits)
    p = gen_primes(logN, p_bits, K, exclude=q)
    return CKKSParams(name, logN, q, p, dnum)


def config_a() -> CKKSParams:
    """HMult/HRotate parity case: N=2^13, FIXEDMANUAL, multDepth 5 (L+1 = 6: 60-bit + 5x50-bit),
    dnum 2, K by the sizing rule (61-bit special primes)."""
    return chain(13, 60, 50, 6, 2, name="A: N=2^13 L+1=6 dnum=2")


def config_b(batch: int = 1) -> CKKSParams:
    """NTT microbench: N=2^16, 36 distinct primes < 2^60 with q = 1 mod 2^17."""
    q = gen_primes(16, 60, 36)
    return CKKSParams("B: N=2^16 36 limbs NTT", 16, q, [], 1, extra={"batch": batch})


def config_c(K: int = 4) -> CKKSParams:
    """Key switching / hoisted rotation: N=2^16, L+1 = 30 (60-bit + 29x50-bit), dnum 3,
    K special primes (4 as specified; 9 = sizing rule, decrypt-valid)."""
    return chain(16, 60, 50, 30, 3, K=K, name=f"C: N=2^16 L+1=30 dnum=3 K={K}")
