"""Rotation sum (fides_accumulate; the reference's Accumulate, src/CKKS/AccumulateBroadcast.cu:
122-160, behind CryptoContext::AccumulateSum): rounds of hoisted rotations summed in the extended
basis, c0 kept there until one final ModDown, c1 brought down every round.

CPU: the rotation list equals the reference's GetAccumulateRotationIndices formula, and the
oracle's restatement decrypts to the slot sums.  GPU: the device result equals the oracle residue
for residue at several radices, strides and sizes, and the C++ facade's AccumulateSum equals it."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, decode, encode, uniform_limbs, xrng


def reference_indices(radix, stride, size):
    """GetAccumulateRotationIndices (AccumulateBroadcast.cu:86-96) restated."""
    out, s = [], stride
    shift = radix.bit_length() - 1
    while s < stride * size:
        idx = s
        while idx < s * radix and idx < stride * size:
            out.append(idx)
            idx += s
        s <<= shift
    return out


@pytest.mark.parametrize("radix,stride,size", [(4, 1, 16), (2, 2, 8), (4, 1, 5), (8, 3, 20), (4, 1, 1)])
def test_rotation_list_matches_reference(radix, stride, size):
    import fides_b200 as F
    assert F.Context.accumulate_rotations(radix, stride, size) == reference_indices(radix, stride, size)


def small_env(seed=5):
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=seed)
    return prm, o, kg


def test_oracle_accumulate_decrypts_to_slot_sums():
    import fides_b200 as F
    prm, o, kg = small_env()
    N, l = prm.N, prm.n_q
    n = N // 2
    radix, stride, size = 4, 2, 12
    keys = {r: kg.rotation_key(r) for r in F.Context.accumulate_rotations(radix, stride, size)}
    rng = xrng(600)
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    delta = 2.0 ** 40
    c0, c1 = kg.encrypt(encode(z, N, delta).astype(np.int64), l)
    r0, r1 = o.accumulate(c0, c1, radix, stride, size, keys)
    got = decode(kg.decrypt_limb0(r0, r1), N, delta)
    want = sum(np.roll(z, -j * stride) for j in range(size))
    assert np.abs(got - want).max() < 1e-6
    with pytest.raises(ValueError):  # a missing key is reported, not guessed
        o.accumulate(c0, c1, radix, stride, size, {1: keys[2]})


@pytest.fixture(scope="module")
def gpu_env(fides):
    prm, o, kg = small_env(seed=7)
    ctx = fides.Context(prm.logN, prm.q, prm.p, prm.dnum)
    return fides, prm, o, kg, ctx, {}


def keys_for(env, rots):
    F, prm, o, kg, ctx, cache = env
    for r in rots:
        if r not in cache:
            k = kg.rotation_key(r)
            cache[r] = (k, F.to_device(k))
    return {r: cache[r][0] for r in rots}, {r: cache[r][1] for r in rots}


@pytest.mark.gpu
@pytest.mark.parametrize("radix,stride,size,level", [(4, 1, 16, 6), (2, 2, 8, 6), (4, 1, 5, 3), (8, 3, 20, 6),
                                                     (4, 1, 1, 6)])
def test_accumulate_equals_oracle(gpu_env, radix, stride, size, level):
    F, prm, o, kg, ctx, _ = gpu_env
    rots = F.Context.accumulate_rotations(radix, stride, size)
    hk, dk = keys_for(gpu_env, rots)
    rng = xrng(700 + size + level)
    a = [uniform_limbs(rng, prm.q[:level], prm.N) for _ in range(2)]
    out = ctx.accumulate(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])), radix, stride, size, dk)
    w0, w1 = o.accumulate(a[0], a[1], radix, stride, size, hk)
    assert np.array_equal(F.to_host(out.c0), w0) and np.array_equal(F.to_host(out.c1), w1)


@pytest.mark.gpu
def test_accumulate_missing_key_refused(gpu_env):
    F, prm, o, kg, ctx, _ = gpu_env
    hk, dk = keys_for(gpu_env, [1, 2, 3])
    rng = xrng(750)
    a = [uniform_limbs(rng, prm.q, prm.N) for _ in range(2)]
    with pytest.raises(F.FidesError) as e:
        ctx.accumulate(F.Ciphertext(F.to_device(a[0]), F.to_device(a[1])), 4, 1, 16, dk)  # 4, 8, 12 missing
    assert e.value.code == -5


@pytest.mark.gpu
def test_facade_accumulate_sum_equals_abi(gpu_env):
    F, prm, o, kg, ctx, _ = gpu_env
    from test_bootstrap import _facade_lib
    lib = _facade_lib()
    u64p = C.POINTER(C.c_uint64)
    lib.facade_accumulate.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, C.c_int,
                                      C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_int, u64p, u64p, C.c_int,
                                      C.c_int, u64p, C.c_char_p, C.c_int]
    size, stride, l, N = 16, 1, prm.n_q, prm.N
    rots = F.Context.accumulate_rotations(4, stride, size)
    hk, dk = keys_for(gpu_env, rots)
    rng = xrng(760)
    a = [uniform_limbs(rng, prm.q, N) for _ in range(2)]
    w0, w1 = o.accumulate(a[0], a[1], 4, stride, size, hk)
    out = np.zeros(2 * l * N, dtype=np.uint64)
    err = C.create_string_buffer(512)
    u64 = lambda x: np.ascontiguousarray(x, dtype=np.uint64).ctypes.data_as(u64p)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    kr = (C.c_int * len(rots))(*rots)
    kp = (C.c_void_p * len(rots))(*[dk[r].data_ptr() for r in rots])
    rc = lib.facade_accumulate(prm.logN, l, prm.K, prm.dnum, u64(primes), 2.0 ** 40, len(rots), kr, kp, l, u64(a[0]),
                               u64(a[1]), size, stride, u64(out), err, 512)
    assert rc == 0, err.value.decode()
    assert np.array_equal(out[:l * N].reshape(l, N), w0) and np.array_equal(out[l * N:].reshape(l, N), w1)
