"""LinearTransform over the extended basis Q.P (the reference's LinearTransform with ext = true,
src/CKKS/LinearTransform.cu:84-196, fed by MakeCKKSPackedPlaintextExtended): the baby steps are
P ct and the hoisted rotations before ModDown (Ciphertext::rotate_hoisted with ext,
Ciphertext.cpp:1221-1300), each giant step's plaintext inner product is taken in Q.P, and the
giant-step fold keeps c0 there (c1 brought down before each rotation without ModDown), so that
one ModDown per component closes the transform.

CPU: the restatement below, composed from the oracle's ModUp / KSK inner product / automorphism /
ModDown, decrypts to the FP64 transform.  GPU: the four entry points it uses (fides_encode_ext,
fides_rotate_hoisted_ext, fides_dot_plain_ext, fides_add_ext) and the C++ facade's extended path
equal that restatement residue for residue."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, decode, encode, small_to_limbs, uniform_limbs, xrng


def p_mod_q(prm, l):
    P = 1
    for p in prm.p:
        P *= p
    return [P % q for q in prm.q[:l]]


def times_p(o, prm, x):
    """P x in Q.P: the Q limbs times P mod q_i, the special limbs zero."""
    l = x.shape[0]
    out = np.zeros((l + o.K, o.N), dtype=np.uint64)
    pm = np.array(p_mod_q(prm, l), dtype=np.uint64)
    out[:l] = o.mul(x, np.repeat(pm[:, None], o.N, axis=1), o.ids(l))
    return out


def rot_ext(o, c0e, c1, key, r):
    """A rotation left in Q.P: automorph(B + c0e), automorph(A) for (A, B) the key-switch
    outputs of c1 (hoistedRotateDotKSK_2_ without the ModDown)."""
    l = c1.shape[0]
    a, b = o.ksk_ip(o.modup(c1), l, key)
    b = o.add(b, c0e, o.ext_ids(l))
    k = o.auto_index(r)
    return o.automorph(b, k), o.automorph(a, k)


def dot_ext(o, xs, pts, l):
    ids = o.ext_ids(l)
    s0 = s1 = None
    for (x0, x1), p in zip(xs, pts):
        m0, m1 = o.mul(x0, p, ids), o.mul(x1, p, ids)
        s0 = m0 if s0 is None else o.add(s0, m0, ids)
        s1 = m1 if s1 is None else o.add(s1, m1, ids)
    return s0, s1


def lt_ext_oracle(o, prm, c0, c1, pts, row, bstep, stride, offset, keys):
    l, N = c0.shape[0], o.N
    ids = o.ext_ids(l)
    nb, gs = min(bstep, row), (row + bstep - 1) // bstep
    baby = [(times_p(o, prm, c0), times_p(o, prm, c1))]
    baby += [rot_ext(o, times_p(o, prm, c0), c1, keys[j * stride], j * stride) for j in range(1, nb)]

    def rot_sum(a, r):
        return rot_ext(o, a[0], o.moddown(a[1]), keys[r], r)

    acc = None
    for g in reversed(range(gs)):
        js = [j for j in range(nb) if g * bstep + j < row]
        inner = dot_ext(o, [baby[j] for j in js], [pts[g * bstep + j] for j in js], l)
        if acc is None:
            acc = inner
            continue
        if (bstep * stride) % (N // 2):
            acc = rot_sum(acc, bstep * stride)
        acc = (o.add(acc[0], inner[0], ids), o.add(acc[1], inner[1], ids))
    if offset:
        acc = rot_sum(acc, offset)
    return o.moddown(acc[0]), o.moddown(acc[1])


def encode_ext_host(o, z, scale, l):
    coeff = encode(z, o.N, scale).astype(np.int64)
    primes = [o.primes[i] for i in o.ext_ids(l)]
    return o.ntt(small_to_limbs(coeff, primes), o.ext_ids(l))


def problem(N, row, bstep, stride, offset, seed):
    n = N // 2
    rng = xrng(seed)
    x = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    D = rng.uniform(-1, 1, (row, n)) + 1j * rng.uniform(-1, 1, (row, n))
    pre = [np.roll(D[k], bstep * (k // bstep) * stride + offset) for k in range(row)]
    want = sum(np.roll(x, -(k * stride + offset)) * D[k] for k in range(row))
    return x, pre, want


def test_oracle_lt_ext_decrypts_to_fp64():
    from fides_b200 import params as P
    prm = P.config_a()
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=31)
    N, l = prm.N, 4
    row, bstep, stride, offset = 6, 4, 1, 2
    rots = sorted(set([j * stride for j in range(1, bstep + 1)] + [offset]))
    keys = {r: kg.rotation_key(r) for r in rots}
    x, pre, want = problem(N, row, bstep, stride, offset, 32)
    ds, dp = 2.0 ** 30, 2.0 ** 20
    c0, c1 = kg.encrypt(encode(x, N, ds).astype(np.int64), l)
    pts = [encode_ext_host(o, p, dp, l) for p in pre]
    r0, r1 = lt_ext_oracle(o, prm, c0, c1, pts, row, bstep, stride, offset, keys)
    got = decode(kg.decrypt_limb0(r0, r1), N, ds * dp)
    assert np.abs(got - want).max() < 1e-3


@pytest.fixture(scope="module")
def env(fides):
    from fides_b200 import params as P
    prm = P.chain(12, 60, 50, 8, 2, name="lt_ext")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=41)
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
@pytest.mark.parametrize("level", [8, 3])
def test_encode_ext_is_the_plain_encoding_over_qp(env, level):
    """The Q limbs equal fides_encode's; every special limb holds the same signed integer
    coefficients (checked through the oracle's inverse NTT against limb 0)."""
    F, prm, o, kg, ctx, _ = env
    N = prm.N
    rng = xrng(50 + level)
    z = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    pe = F.to_host(ctx.encode_ext(z, 2.0 ** 40, level))
    assert pe.shape == (level + prm.K, N)
    assert np.array_equal(pe[:level], F.to_host(ctx.encode(z, 2.0 ** 40, level)))
    q0 = prm.q[0]
    c0 = o.ntt(pe[:1], [0], inverse=True)[0].astype(object)
    signed = [int(v) - q0 if int(v) > q0 // 2 else int(v) for v in c0]
    for k in range(prm.K):
        pk = prm.p[k]
        ck = o.ntt(pe[level + k:level + k + 1], [prm.n_q + k], inverse=True)[0]
        assert all(int(a) == s % pk for a, s in zip(ck, signed)), f"special limb {k}"


@pytest.mark.gpu
@pytest.mark.parametrize("level", [8, 5, 1])
def test_rotate_hoisted_ext_and_dot_equal_oracle(env, level):
    F, prm, o, kg, ctx, _ = env
    rots = [1, 3, -2]
    hk, dk = keys_for(env, rots)
    rng = xrng(60 + level)
    a = [uniform_limbs(rng, prm.q[:level], prm.N) for _ in range(2)]
    ct = F.Ciphertext(F.to_device(a[0]), F.to_device(a[1]))
    outs = ctx.rotate_hoisted_ext(ct, [dk[r] for r in rots], rots)
    want = [rot_ext(o, times_p(o, prm, a[0]), a[1], hk[r], r) for r in rots]
    for got, (w0, w1) in zip(outs, want):
        assert np.array_equal(F.to_host(got.c0), w0) and np.array_equal(F.to_host(got.c1), w1)
    # ModDown of each gives the Q-basis hoisted rotation
    plain = ctx.rotate_hoisted(ct, [dk[r] for r in rots], rots)
    for g, p in zip(outs, plain):
        assert np.array_equal(F.to_host(ctx.moddown(g.c0)), F.to_host(p.c0))
        assert np.array_equal(F.to_host(ctx.moddown(g.c1)), F.to_host(p.c1))
    # an extended c0 added as it is
    e0 = uniform_limbs(rng, [prm.q[i] for i in range(level)] + prm.p, prm.N)
    out = ctx.rotate_hoisted_ext(ct, [dk[3]], [3], c0_ext=F.to_device(e0))[0]
    w0, w1 = rot_ext(o, e0, a[1], hk[3], 3)
    assert np.array_equal(F.to_host(out.c0), w0) and np.array_equal(F.to_host(out.c1), w1)
    # inner product and sum over Q.P
    ext_primes = [prm.q[i] for i in range(level)] + prm.p
    pts = [uniform_limbs(rng, ext_primes, prm.N) for _ in range(3)]
    d = ctx.dot_plain_ext(outs, [F.to_device(p) for p in pts], level)
    w0, w1 = dot_ext(o, want, pts, level)
    assert np.array_equal(F.to_host(d.c0), w0) and np.array_equal(F.to_host(d.c1), w1)
    s = ctx.add_ext(d.c0, outs[0].c0, level)
    assert np.array_equal(F.to_host(s), o.add(w0, want[0][0], o.ext_ids(level)))


@pytest.mark.gpu
@pytest.mark.parametrize("ext", [False, True])
def test_dot_plain_bsgs_equals_oracle(env, ext):
    """All giant steps' inner products in one launch (fides_dot_plain_bsgs): each output is the
    oracle's sum over the giant step's non-null diagonals; a giant step without terms is zero."""
    F, prm, o, kg, ctx, _ = env
    level, nb, ng = 6, 5, 4
    primes = prm.q[:level] + (prm.p if ext else [])
    ids = o.ext_ids(level) if ext else o.ids(level)
    rng = xrng(80 + ext)
    xs = [[uniform_limbs(rng, primes, prm.N) for _ in range(2)] for _ in range(nb)]
    pts = [[uniform_limbs(rng, primes, prm.N) if (i * nb + k) % 7 != 3 else None for k in range(nb)]
           for i in range(ng - 1)] + [[None] * nb]
    babies = [F.Ciphertext(F.to_device(a), F.to_device(b)) for a, b in xs]
    got = ctx.dot_plain_bsgs(babies, [[None if p is None else F.to_device(p) for p in row] for row in pts], level,
                             ext=ext)
    for i in range(ng):
        w0 = np.zeros((len(primes), prm.N), dtype=np.uint64)
        w1 = np.zeros_like(w0)
        for k in range(nb):
            if pts[i][k] is not None:
                w0 = o.add(w0, o.mul(xs[k][0], pts[i][k], ids), ids)
                w1 = o.add(w1, o.mul(xs[k][1], pts[i][k], ids), ids)
        assert np.array_equal(F.to_host(got[i].c0), w0) and np.array_equal(F.to_host(got[i].c1), w1), f"giant {i}"


@pytest.mark.gpu
@pytest.mark.parametrize("row_size,b_step,stride,offset",
                         [(14, 4, 1, 3), (8, 8, 2, 0), (5, 2, 3, -2), (4, 2, 1024, 0), (3, 4, 1, 1),
                          (38, 18, 1, 0)])
def test_cpp_facade_linear_transform_ext(env, row_size, b_step, stride, offset):
    """The facade's LinearTransform / LinearTransformMany on extended diagonals equal the
    restatement above residue for residue (after the facade's Rescale, applied to the
    restatement too), decrypt to the FP64 transform, and the batched form's first set equals
    the single transform.  Cases: several giant steps with and without offset, one giant step
    (bStep > rowSize), giant-step rotations by N/2 slots (the identity, skipped), and more than
    16 baby steps (one inner-product launch per giant step)."""
    F, prm, o, kg, ctx, _ = env
    from test_bootstrap import _facade_lib
    N, l = prm.N, prm.n_q
    rots = sorted(set([i * stride for i in range(1, b_step + 1)] + ([offset] if offset else [])))
    hk, dk = keys_for(env, rots)
    top = 2.0 ** 45
    S = [0.0] * (l + 1)
    S[l] = top
    for k in range(l, 1, -1):
        S[k - 1] = S[k] * S[k] / prm.q[k - 1]
    x, pre, want = problem(N, row_size, b_step, stride, offset, 70 + row_size)
    dz = np.stack([np.stack([p_.real, p_.imag], axis=1) for p_ in pre]).reshape(-1).copy()
    c0, c1 = kg.encrypt(encode(x, N, S[l]).astype(np.int64), l)
    lib = _facade_lib()
    u64p, dp = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
    lib.facade_linear_transform.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, C.c_int,
                                            C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_int, u64p, u64p, C.c_int,
                                            C.c_int, C.c_int, C.c_int, dp, C.c_int, C.c_int, u64p, dp, C.c_char_p,
                                            C.c_int]
    lo = l - 1
    out = np.zeros(3 * 2 * lo * N, dtype=np.uint64)
    sc = C.c_double()
    err = C.create_string_buffer(512)
    u64 = lambda a: np.ascontiguousarray(a, dtype=np.uint64).ctypes.data_as(u64p)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    rc = lib.facade_linear_transform(prm.logN, l, prm.K, prm.dnum, u64(primes), top, len(rots),
                                     (C.c_int * len(rots))(*rots),
                                     (C.c_void_p * len(rots))(*[dk[r].data_ptr() for r in rots]), l, u64(c0), u64(c1),
                                     row_size, b_step, stride, offset, dz.ctypes.data_as(dp), N // 2, 1, u64(out),
                                     C.byref(sc), err, 512)
    assert rc == 0, err.value.decode()
    res = [out[i * 2 * lo * N:(i + 1) * 2 * lo * N].reshape(2, lo, N) for i in range(3)]
    pts = [F.to_host(ctx.encode_ext(p, S[l], l)) for p in pre]  # the facade's own encoding
    w0, w1 = lt_ext_oracle(o, prm, c0, c1, pts, row_size, b_step, stride, offset, hk)
    assert np.array_equal(res[0][0], o.rescale(w0)) and np.array_equal(res[0][1], o.rescale(w1))
    got = decode(kg.decrypt_limb0(res[0][0], res[0][1]), N, sc.value)
    assert np.abs(got - want).max() < 1e-6
    assert np.array_equal(res[1], res[0])
    got_neg = decode(kg.decrypt_limb0(res[2][0], res[2][1]), N, sc.value)
    assert np.abs(got_neg + want).max() < 1e-6
