"""Bootstrapping: the special-FFT factorisation (CPU) and a full GPU bootstrap whose
decrypted output matches the FP64 plaintext (precision in bits, as the reference's
BootstrapPrecisionTests measure it, test/BootstrapPrecisionTests.cu:141-259)."""
import math

import numpy as np
import pytest

import oracle as O
from ckks_host import KeyGen, decode, encode, small_to_limbs, uniform_limbs, xrng


def _u0(n):
    N = 2 * n
    zeta = np.exp(1j * np.pi / N)
    e = [pow(5, j, 2 * N) for j in range(n)]
    return np.array([[zeta ** (e[j] * k) for k in range(n)] for j in range(n)])


@pytest.mark.parametrize("logn,levels", [(4, 2), (6, 3), (7, 3)])
def test_special_fft_factorisation(logn, levels):
    from fides_b200 import bootstrap as B
    n = 1 << logn
    U = _u0(n)
    w = xrng(logn).normal(size=n) + 1j * xrng(logn + 1).normal(size=n)
    P = B.bit_reverse_perm(n)
    v = w[P]
    for M in B.fft_levels(n, levels, inverse=False):
        v = B.apply_diags(M, v)
    assert np.abs(v - U @ w).max() < 1e-9 * n
    u = U @ w
    for M in B.fft_levels(n, levels, inverse=True):
        u = B.apply_diags(M, u)
    assert np.abs(u - w[P]).max() < 1e-9 * n
    assert np.abs(U.conj().T @ U - n * np.eye(n)).max() < 1e-9 * n


def test_slot_encoding_matches_client_encoder():
    from fides_b200 import bootstrap as B
    N = 64
    z = xrng(3).uniform(-1, 1, N // 2) + 1j * xrng(4).uniform(-1, 1, N // 2)
    assert np.array_equal(B.encode_coeffs(z, N, 2.0 ** 30), encode(z, N, 2.0 ** 30).astype(np.int64))
    assert np.abs(B.decode_coeffs(B.encode_coeffs(z, N, 2.0 ** 30), N, 2.0 ** 30) - z).max() < 1e-8


def make_boot(F, logN, n_q=20, dnum=4, hw=32, K=12):
    from fides_b200 import params as P
    from fides_b200 import bootstrap as B
    prm = P.chain(logN, 60, 50, n_q, dnum, name=f"boot N=2^{logN}")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=61, hamming_weight=hw)
    rk = F.to_device(kg.relin_key())
    conj = F.to_device(kg.auto_key(2 * prm.N - 1))
    probe = B.Bootstrapper.__new__(B.Bootstrapper)
    ev = B.Evaluator(F, ctx, rk, {}, conj, top_scale=2.0 ** 50)
    bs = B.Bootstrapper(ev, K=K)
    ev.rot_keys = {r: F.to_device(kg.rotation_key(r)) for r in bs.needed_rotations()}
    return prm, o, kg, ctx, ev, bs


@pytest.mark.gpu
def test_bootstrap_precision_n4096(fides):
    from fides_b200 import bootstrap as B
    prm, o, kg, ctx, ev, bs = make_boot(fides, 12)
    N, n = prm.N, prm.N // 2
    delta = 2.0 ** 50
    bs.prepare(top_level=prm.n_q, msg_scale=delta)
    assert bs.out_level >= 2
    rng = xrng(62)
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c0, c1 = kg.encrypt(encode(z, N, delta).astype(np.int64), 1)
    ct = B.Ct(fides.to_device(c0), fides.to_device(c1), delta)
    out = bs.bootstrap(ct)
    got = decode(kg.decrypt_limb0(fides.to_host(out.c0), fides.to_host(out.c1)), N, out.scale)
    err = np.abs(got - z).max()
    bits = -math.log2(err)
    print(f"bootstrap N=2^12: out level {out.level}, max error {err:.3e} ({bits:.1f} bits)")
    assert bits > 12


@pytest.mark.gpu
def test_chebyshev_paterson_stockmeyer(fides):
    """The EvalMod series evaluated by Paterson-Stockmeyer over two lanes decrypts to the FP64
    Chebyshev sum of the slots, lands ceil(log2 d) + 1 levels down, and each lane equals the
    same series evaluated alone (lanes are independent)."""
    from fides_b200 import bootstrap as B
    prm, o, kg, ctx, ev, bs = make_boot(fides, 12)
    N, n, l = prm.N, prm.N // 2, prm.n_q
    zs, cts = [], []
    for i in range(2):
        z = xrng(70 + i).uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z.astype(np.complex128), N, ev.S[l]).astype(np.int64), l)
        zs.append(z)
        cts.append(B.Ct(fides.to_device(c0), fides.to_device(c1), ev.S[l]))
    outs = bs._chebyshev_many(cts)
    alone = bs._chebyshev(cts[1])
    assert outs[0].level == l - (math.ceil(math.log2(bs.degree)) + 1)
    for z, out in zip(zs, outs):
        got = decode(kg.decrypt_limb0(fides.to_host(out.c0), fides.to_host(out.c1)), N, out.scale)
        ref = np.polynomial.chebyshev.chebval(z, bs.cheb)
        assert -math.log2(np.abs(got - ref).max()) > 20
    assert np.array_equal(fides.to_host(alone.c0), fides.to_host(outs[1].c0))
    assert np.array_equal(fides.to_host(alone.c1), fides.to_host(outs[1].c1))


@pytest.mark.gpu
def test_bootstrap_graph_replay_is_bit_identical(fides):
    import torch
    from fides_b200 import bootstrap as B
    prm, o, kg, ctx, ev, bs = make_boot(fides, 12)
    bs.prescale = 1 << 4
    delta = 2.0 ** 50
    bs.prepare(top_level=prm.n_q, msg_scale=delta)
    rng = xrng(63)
    n = prm.N // 2
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
    ct = B.Ct(fides.to_device(c0), fides.to_device(c1), delta)
    direct = bs.bootstrap(ct)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        gout = bs.bootstrap(ct)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(direct.c0, gout.c0) and torch.equal(direct.c1, gout.c1)
    got = decode(kg.decrypt_limb0(fides.to_host(gout.c0), fides.to_host(gout.c1)), prm.N, gout.scale)
    assert -math.log2(np.abs(got - z).max()) > 14


@pytest.mark.gpu
def test_concurrent_batch_equals_sequential(fides):
    """A batch bootstrapped on parallel streams (and as one graph with parallel branches)
    gives exactly the ciphertexts of one-at-a-time bootstraps."""
    import torch
    from fides_b200 import bootstrap as B
    prm, o, kg, ctx, ev, bs = make_boot(fides, 12)
    delta = 2.0 ** 50
    bs.prepare(top_level=prm.n_q, msg_scale=delta)
    rng = xrng(64)
    n = prm.N // 2
    cts = []
    for _ in range(3):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        cts.append(B.Ct(fides.to_device(c0), fides.to_device(c1), delta))
    seq = [bs.bootstrap(c) for c in cts]
    par = B.bootstrap_concurrent(bs, cts)
    torch.cuda.synchronize()
    for a, b in zip(seq, par):
        assert torch.equal(a.c0, b.c0) and torch.equal(a.c1, b.c1)
    g = torch.cuda.CUDAGraph()
    streams = [torch.cuda.Stream() for _ in cts]
    with torch.cuda.graph(g):
        gout = B.bootstrap_concurrent(bs, cts, streams)
    g.replay()
    torch.cuda.synchronize()
    for a, b in zip(seq, gout):
        assert torch.equal(a.c0, b.c0) and torch.equal(a.c1, b.c1)


@pytest.mark.gpu
@pytest.mark.parametrize("driver", ["python", "native"])
def test_served_bootstraps_in_a_mix(fides, driver):
    """Bootstrap requests through the request loop (two engines and a batch engine; graphs of
    the Python driver or of the C++ bootstrapper) mixed with HMult / HRotate requests submitted
    from several threads: every bootstrap equals the direct bootstrap of its input and every
    HMult / HRotate equals the same request run alone."""
    import random
    import threading
    import torch
    from fides_b200 import bootstrap as B
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    delta = 2.0 ** 50
    bs.prepare(top_level=prm.n_q, msg_scale=delta)
    nb = None
    if driver == "native":
        nb = native_for(F, prm, ev, bs)
        nb.prepare()
        engines = [B.make_native_engine(nb, 1) for _ in range(2)]
        batch_engine = B.make_native_engine(nb, 3)  # one graph: three ciphertexts in one launch sequence
        direct = lambda ct: nb.bootstrap(ct)
    else:
        engines = [B.make_engine(bs, delta) for _ in range(2)]
        batch_engine = B.make_batch_engine(bs, delta, 3)  # one graph, three ciphertexts per launch
        direct = lambda ct: bs.bootstrap(B.Ct(ct.c0, ct.c1, delta))
    rng = xrng(65)
    n = prm.N // 2
    boot_in, boot_ref = [], []
    for _ in range(6):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        ct = F.Ciphertext(F.to_device(c0[:1]), F.to_device(c1[:1]))
        boot_in.append(ct)
        r = direct(ct)
        boot_ref.append((r.c0.clone(), r.c1.clone()))
    torch.cuda.synchronize()
    rot_key = F.to_device(kg.rotation_key(1))
    reqs = []
    rnd = random.Random(7)
    for i in range(12):
        l = rnd.choice([4, 8, 12])
        a = F.Ciphertext(F.to_device(uniform_limbs(rng, prm.q[:l], prm.N)), F.to_device(uniform_limbs(rng, prm.q[:l], prm.N)))
        if i % 2:
            b = F.Ciphertext(F.to_device(uniform_limbs(rng, prm.q[:l], prm.N)), F.to_device(uniform_limbs(rng, prm.q[:l], prm.N)))
            reqs.append((F.OP_HMULT, a, b, l - 1))
        else:
            reqs.append((F.OP_ROTATE, a, None, l))
    alone = []
    for op, a, b, lo in reqs:
        alone.append(ctx.mult(a, b, ev.rk, rescale=True) if op == F.OP_HMULT else ctx.rotate(a, rot_key, 1))
    srv = F.Server(ctx, n_streams=2, max_batch=4)
    try:
        srv.set_relin_key(ev.rk)
        srv.add_rotation_key(1, rot_key)
        srv.set_max_inflight(1)
        for g, sin, sout in engines:
            srv.add_bootstrap(g, sin, sout)
        srv.add_bootstrap_batch(*batch_engine)
        out_lvl = engines[0][2].level
        jobs = [("b", i) for i in range(len(boot_in))] + [("o", i) for i in range(len(reqs))]
        random.Random(8).shuffle(jobs)
        outs = {}
        tickets = {}

        def worker(part):
            for kind, i in part:
                if kind == "b":
                    out = F.Ciphertext(ctx.empty(out_lvl), ctx.empty(out_lvl))
                    outs[("b", i)] = out
                    tickets[("b", i)] = srv.submit(F.OP_BOOTSTRAP, boot_in[i], out)
                else:
                    op, a, b, lo = reqs[i]
                    out = F.Ciphertext(ctx.empty(lo), ctx.empty(lo))
                    outs[("o", i)] = out
                    tickets[("o", i)] = srv.submit(op, a, out, b, 1)

        ts = [threading.Thread(target=worker, args=(jobs[k::3],)) for k in range(3)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for key, t in tickets.items():
            st, _ = srv.wait(t)
            assert st == 0, key
    finally:
        srv.close()
    for i, (r0, r1) in enumerate(boot_ref):
        assert torch.equal(outs[("b", i)].c0, r0) and torch.equal(outs[("b", i)].c1, r1), f"bootstrap {i}"
    if nb is not None:
        del engines, batch_engine
        nb.close()
    for i, x in enumerate(alone):
        assert torch.equal(outs[("o", i)].c0, x.c0) and torch.equal(outs[("o", i)].c1, x.c1), f"request {i}"


@pytest.mark.gpu
def test_bootstrap_sparse_secret_encapsulation(fides):
    """Dense (uniform ternary) secret with sparse-secret encapsulation: the level-1 input is
    switched to a HW-32 secret for ModRaise and back to the dense secret right after it, so
    every other key is the dense secret's.  The result decrypts under the dense secret."""
    from fides_b200 import params as P
    from fides_b200 import bootstrap as B
    F = fides
    prm = P.chain(12, 60, 50, 20, 4, name="boot N=2^12 dense")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
    dense = KeyGen(o, seed_stream=81)
    sparse = KeyGen(o, seed_stream=82, hamming_weight=32)
    assert np.count_nonzero(dense.s_coeff) > 1000
    to_sparse = F.to_device(dense.switching_key(sparse.s_eval, dense.s_eval))
    to_dense = F.to_device(dense.switching_key(dense.s_eval, sparse.s_eval))
    ev = B.Evaluator(F, ctx, F.to_device(dense.relin_key()), {}, F.to_device(dense.auto_key(2 * prm.N - 1)),
                     top_scale=2.0 ** 50)
    bs = B.Bootstrapper(ev, K=12, encapsulation=(to_sparse, to_dense))
    ev.rot_keys = {r: F.to_device(dense.rotation_key(r)) for r in bs.needed_rotations()}
    delta = 2.0 ** 50
    bs.prepare(top_level=prm.n_q, msg_scale=delta)
    rng = xrng(66)
    n = prm.N // 2
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c0, c1 = dense.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
    out = bs.bootstrap(B.Ct(F.to_device(c0), F.to_device(c1), delta))
    got = decode(dense.decrypt_limb0(F.to_host(out.c0), F.to_host(out.c1)), prm.N, out.scale)
    bits = -math.log2(np.abs(got - z).max())
    print(f"bootstrap with encapsulation N=2^12: {bits:.1f} bits, out level {out.level}")
    assert bits > 12


def make_config_d(F, seed=21):
    """Config D: N = 2^16, L+1 = 24 (60-bit q_0, 50-bit scaling primes), dnum 3, dense uniform
    ternary secret with HW-32 sparse-secret encapsulation, CtS / StC level budget {3, 3},
    input scale 2^50 pre-scaled by 2^5 (the bench's bootstrap)."""
    from fides_b200 import params as P
    from fides_b200 import bootstrap as B
    prm = P.chain(16, 60, 50, 24, 3, name="D")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=seed)
    sparse = KeyGen(o, seed_stream=seed + 1000, hamming_weight=32)
    ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
    encaps = (F.to_device(kg.switching_key(sparse.s_eval, kg.s_eval)),
              F.to_device(kg.switching_key(kg.s_eval, sparse.s_eval)))
    ev = B.Evaluator(F, ctx, F.to_device(kg.relin_key()), {}, F.to_device(kg.auto_key(2 * prm.N - 1)),
                     top_scale=2.0 ** 50)
    bs = B.Bootstrapper(ev, K=12, prescale_bits=5, encapsulation=encaps)
    assert bs.cts_levels == 3
    ev.rot_keys = {r: F.to_device(kg.rotation_key(r)) for r in bs.needed_rotations()}
    bs.prepare(top_level=prm.n_q, msg_scale=2.0 ** 50)
    return prm, o, kg, ctx, ev, bs


@pytest.fixture(scope="module")
def config_d(fides):
    return make_config_d(fides)


@pytest.mark.gpu
def test_bootstrap_config_d_n65536_batch8(fides, config_d):
    """Config D at full size: 2^15 slots uniform in [-1, 1]; every ciphertext of a batch of 8
    decrypts within 2^-15 of the FP64 plaintext (reference measure:
    test/BootstrapPrecisionTests.cu:141-259), and the batch bootstrapped on 8 parallel streams
    equals the one-at-a-time bootstraps bit for bit."""
    import torch
    from fides_b200 import bootstrap as B
    F = fides
    prm, o, kg, ctx, ev, bs = config_d
    delta = 2.0 ** 50
    n = prm.N // 2
    assert n == 1 << 15
    rng = xrng(22)
    zs, cts = [], []
    for _ in range(8):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        zs.append(z)
        cts.append(B.Ct(F.to_device(c0), F.to_device(c1), delta))
    seq = [bs.bootstrap(c) for c in cts]
    par = B.bootstrap_concurrent(bs, cts, [torch.cuda.Stream() for _ in cts])
    torch.cuda.synchronize()
    bits = []
    for i, (a, b, z) in enumerate(zip(seq, par, zs)):
        assert torch.equal(a.c0, b.c0) and torch.equal(a.c1, b.c1), f"ciphertext {i}: batch != single"
        got = decode(kg.decrypt_limb0(F.to_host(a.c0), F.to_host(a.c1)), prm.N, a.scale)
        bits.append(-math.log2(np.abs(got - z).max()))
    print(f"config D bootstrap: out level {seq[0].level}, precision {min(bits):.2f}..{max(bits):.2f} bits")
    assert seq[0].level >= 8
    assert min(bits) >= 15.0


# ---------------------------------------------------------------- the library's C++ bootstrapper
def native_for(F, prm, ev, bs, encaps=None):
    """A NativeBootstrapper with the Python driver's parameters and keys."""
    nb = F.NativeBootstrapper(ev.ctx, top_level=prm.n_q, top_scale=ev.S[prm.n_q], msg_scale=2.0 ** 50,
                              budget=(bs.cts_levels, bs.stc_levels), K=bs.K, r=bs.r, degree=bs.degree, baby=bs.baby,
                              prescale_bits=bs.prescale.bit_length() - 1, encapsulation=encaps is not None,
                              double_hoist=False)  # the Python driver's single-hoisted form
    nb.set_keys(ev.rk, ev.conj_key, *(encaps or (None, None)))
    for r in nb.rotations():
        nb.set_rotation_key(r, ev.rot_keys[r])
    return nb


def python_with_native_tables(bs, nb):
    """The Python driver re-prepared on the C++ driver's tables (special-FFT diagonals and
    Chebyshev coefficients), so that the two drivers can be compared residue for residue."""
    bs.cts, bs.stc, bs.cheb = nb.matrices("cts"), nb.matrices("stc"), nb.chebyshev()
    bs.prepare(top_level=bs.top, msg_scale=2.0 ** 50)
    return bs


@pytest.mark.gpu
def test_native_tables_match_numpy(fides):
    """The C++ driver's derived tables equal the Python driver's numpy ones to rounding: the
    composed special-FFT diagonals (same offsets), the Chebyshev coefficients and the rotation
    list."""
    from fides_b200 import bootstrap as B
    prm, o, kg, ctx, ev, bs = make_boot(fides, 12)
    nb = native_for(fides, prm, ev, bs)
    assert nb.rotations() == bs.needed_rotations()
    assert np.abs(nb.chebyshev() - np.asarray(bs.cheb)).max() < 1e-13
    for which, ref in (("cts", bs.cts), ("stc", bs.stc)):
        mats = nb.matrices(which)
        assert len(mats) == len(ref)
        for M, R in zip(mats, ref):
            assert sorted(M) == sorted(R)
            for k in M:
                assert np.abs(M[k] - R[k]).max() <= 1e-12 * max(1.0, np.abs(R[k]).max())


@pytest.mark.gpu
def test_native_bootstrap_equals_python_driver_n4096(fides):
    """N = 2^12: the C++ bootstrapper's output equals the Python driver's on the same tables
    bit for bit, decrypts to the FP64 plaintext (> 12 bits), and a batch through
    fides_bootstrap_batch equals the single bootstraps."""
    import torch
    from fides_b200 import bootstrap as B
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    nb = native_for(F, prm, ev, bs)
    nb.prepare()
    bs.top = prm.n_q
    python_with_native_tables(bs, nb)
    assert nb.out_level == bs.out_level
    delta = 2.0 ** 50
    rng = xrng(67)
    n = prm.N // 2
    zs, cts = [], []
    for _ in range(3):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        zs.append(z)
        cts.append(F.Ciphertext(F.to_device(c0), F.to_device(c1)))
    # same encoded diagonals
    for which, plans in (("cts", bs.cts_pts), ("stc", bs.stc_pts)):
        for m, P in enumerate(plans):
            for (i, j), pt in P["pts"].items():
                assert torch.equal(nb.plaintext(which, m, i, j, P["level"]), pt), f"{which} {m} ({i}, {j})"
    py = bs.bootstrap(B.Ct(cts[0].c0, cts[0].c1, delta))
    nat = nb.bootstrap(cts[0])
    batch = nb.bootstrap_batch(cts)
    torch.cuda.synchronize()
    bits_py = -math.log2(np.abs(decode(kg.decrypt_limb0(F.to_host(py.c0), F.to_host(py.c1)), prm.N, py.scale)
                                - zs[0]).max())
    bits_nat = -math.log2(np.abs(decode(kg.decrypt_limb0(F.to_host(nat.c0), F.to_host(nat.c1)), prm.N, nb.out_scale)
                                 - zs[0]).max())
    print(f"N=2^12 bootstrap: Python driver {bits_py:.2f} bits, C++ driver {bits_nat:.2f} bits")
    assert torch.equal(py.c0, nat.c0) and torch.equal(py.c1, nat.c1)
    for i, (ct, out) in enumerate(zip(cts, batch)):
        single = nat if i == 0 else nb.bootstrap(ct)
        torch.cuda.synchronize()
        assert torch.equal(single.c0, out.c0) and torch.equal(single.c1, out.c1), f"batch item {i}"
        got = decode(kg.decrypt_limb0(F.to_host(out.c0), F.to_host(out.c1)), prm.N, nb.out_scale)
        assert -math.log2(np.abs(got - zs[i]).max()) > 12
    nb.close()


@pytest.mark.gpu
def test_native_bootstrap_config_d_n65536(fides, config_d):
    """Config D through the C++ bootstrapper: encapsulation, prescale 2^5, budget {3, 3};
    >= 15 bits for a batch of 8 (fides_bootstrap_batch), batch = single bit for bit, and the
    single equals the Python driver's on the same tables; the double-hoisted form likewise
    >= 15 bits with batch = single."""
    import torch
    from fides_b200 import bootstrap as B
    F = fides
    prm, o, kg, ctx, ev, bs = config_d
    nb = native_for(F, prm, ev, bs, encaps=bs.encapsulation)
    nb.prepare()
    delta = 2.0 ** 50
    rng = xrng(23)
    n = prm.N // 2
    zs, cts = [], []
    for _ in range(8):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        zs.append(z)
        cts.append(F.Ciphertext(F.to_device(c0), F.to_device(c1)))
    batch = nb.bootstrap_batch(cts)
    single = nb.bootstrap(cts[0])
    torch.cuda.synchronize()
    assert torch.equal(single.c0, batch[0].c0) and torch.equal(single.c1, batch[0].c1)
    bits = []
    for out, z in zip(batch, zs):
        got = decode(kg.decrypt_limb0(F.to_host(out.c0), F.to_host(out.c1)), prm.N, nb.out_scale)
        bits.append(-math.log2(np.abs(got - z).max()))
    print(f"config D, C++ bootstrapper: out level {nb.out_level}, precision {min(bits):.2f}..{max(bits):.2f} bits")
    assert min(bits) >= 15.0
    python_with_native_tables(bs, nb)
    py = bs.bootstrap(B.Ct(cts[0].c0, cts[0].c1, delta))
    torch.cuda.synchronize()
    assert torch.equal(py.c0, single.c0) and torch.equal(py.c1, single.c1)
    # the C++ facade (EvalBootstrap, single and vector forms) on two of the inputs
    host = [(F.to_host(c.c0), F.to_host(c.c1)) for c in cts[:2]]
    fs, fb, L, _ = facade_bootstrap(F, prm, ev, bs, host, encaps=bs.encapsulation)
    assert L == nb.out_level
    for i in range(2):
        for got in (fs[i], fb[i]):
            assert np.array_equal(got[0], F.to_host(batch[i].c0)) and np.array_equal(got[1], F.to_host(batch[i].c1))
    nb.close()
    # the double-hoisted form (the library's default) on the same inputs and keys
    nd = F.NativeBootstrapper(ctx, top_level=prm.n_q, top_scale=ev.S[prm.n_q], msg_scale=delta,
                              budget=(bs.cts_levels, bs.stc_levels), K=bs.K, r=bs.r, degree=bs.degree, baby=bs.baby,
                              prescale_bits=bs.prescale.bit_length() - 1, encapsulation=True, double_hoist=True)
    nd.set_keys(ev.rk, ev.conj_key, *bs.encapsulation)
    for r in nd.rotations():
        nd.set_rotation_key(r, ev.rot_keys[r])
    nd.prepare()
    dbatch = nd.bootstrap_batch(cts)
    dsingle = nd.bootstrap(cts[3])
    torch.cuda.synchronize()
    assert torch.equal(dsingle.c0, dbatch[3].c0) and torch.equal(dsingle.c1, dbatch[3].c1)
    dbits = [-math.log2(np.abs(decode(kg.decrypt_limb0(F.to_host(x.c0), F.to_host(x.c1)), prm.N, nd.out_scale)
                                - z).max()) for x, z in zip(dbatch, zs)]
    print(f"config D, double-hoisted: precision {min(dbits):.2f}..{max(dbits):.2f} bits")
    assert min(dbits) >= 15.0
    nd.close()


# ---------------------------------------------------------------- the C++ evaluation facade
def _facade_lib():
    import ctypes as C
    import os
    from conftest import ROOT
    lib = C.CDLL(os.path.join(ROOT, "fideslib-fork_b200", "libfacade_test.so"))
    vp, u64p, dp, ip = C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_double), C.POINTER(C.c_int)
    vpp = C.POINTER(vp)
    lib.facade_bootstrap.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, vp, vp, C.c_int, ip, vpp,
                                     vp, vp, C.c_double, C.c_int, C.c_int, C.c_int, vpp, vpp, vpp, vpp, vpp, vpp, ip,
                                     dp, C.c_char_p, C.c_int]
    lib.facade_arith.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, vp, C.c_int, vp, C.c_int,
                                 u64p, u64p, u64p, u64p, u64p, u64p, C.c_char_p, C.c_int]
    lib.facade_plain.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, C.c_int, u64p, u64p, dp,
                                 C.c_int, u64p, C.c_char_p, C.c_int]
    lib.facade_more.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, vp, C.c_int, vp, C.c_int,
                                u64p, u64p, u64p, u64p, u64p, C.c_char_p, C.c_int]
    return lib


def facade_bootstrap(F, prm, ev, bs, cts_host, encaps=None, double_hoist=False):
    """Runs the facade's EvalBootstrap (single and batch) on host level-1 ciphertexts; returns
    (singles, batch, out_level, out_scale) as host arrays."""
    import ctypes as C
    lib = _facade_lib()
    vp = C.c_void_p
    rots = sorted(ev.rot_keys)
    N, nb_ = prm.N, len(cts_host)
    # the facade reports its output level after the first bootstrap; the output arrays are sized
    # for the top level and trimmed afterwards
    outs = [[np.zeros((prm.n_q, N), dtype=np.uint64) for _ in range(2)] for _ in range(2 * nb_)]
    ins = [np.ascontiguousarray(c, dtype=np.uint64) for ct in cts_host for c in ct]
    arr = lambda xs: (vp * len(xs))(*[x.ctypes.data for x in xs])
    lvl, sc = C.c_int(), C.c_double()
    err = C.create_string_buffer(512)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    rc = lib.facade_bootstrap(prm.logN, prm.n_q, prm.K, prm.dnum, primes.ctypes.data_as(C.POINTER(C.c_uint64)),
                              ev.S[prm.n_q], ev.rk.data_ptr(), ev.conj_key.data_ptr(), len(rots),
                              (C.c_int * len(rots))(*rots), (vp * len(rots))(*[ev.rot_keys[r].data_ptr() for r in rots]),
                              encaps[0].data_ptr() if encaps else None, encaps[1].data_ptr() if encaps else None,
                              2.0 ** 50, bs.prescale.bit_length() - 1, 1 if double_hoist else 0, nb_,
                              arr(ins[0::2]), arr(ins[1::2]),
                              arr([o[0] for o in outs[:nb_]]), arr([o[1] for o in outs[:nb_]]),
                              arr([o[0] for o in outs[nb_:]]), arr([o[1] for o in outs[nb_:]]), C.byref(lvl),
                              C.byref(sc), err, 512)
    assert rc == 0, err.value.decode()
    L = lvl.value
    singles = [(o[0][:L], o[1][:L]) for o in outs[:nb_]]
    batch = [(o[0][:L], o[1][:L]) for o in outs[nb_:]]
    return singles, batch, L, sc.value


@pytest.mark.gpu
def test_cpp_facade_bootstrap_n4096(fides):
    """The C++ facade (CryptoContextImpl::EvalBootstrapSetup / EvalBootstrap, single and vector
    forms) at N = 2^12, through a compiled driver: bit-identical to the ABI bootstrapper and to
    the Python driver on the same tables, > 12 bits against the FP64 plaintext."""
    import torch
    from fides_b200 import bootstrap as B
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    delta = 2.0 ** 50
    rng = xrng(68)
    n = prm.N // 2
    zs, cts = [], []
    for _ in range(2):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        zs.append(z)
        cts.append(kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1))
    singles, batch, L, scale = facade_bootstrap(F, prm, ev, bs, cts)
    nb = native_for(F, prm, ev, bs)
    nb.prepare()
    bs.top = prm.n_q
    python_with_native_tables(bs, nb)
    assert L == nb.out_level
    for i, (c, z) in enumerate(zip(cts, zs)):
        ct = F.Ciphertext(F.to_device(c[0]), F.to_device(c[1]))
        nat = nb.bootstrap(ct)
        py = bs.bootstrap(B.Ct(ct.c0, ct.c1, delta))
        torch.cuda.synchronize()
        for got in (singles[i], batch[i]):
            assert np.array_equal(got[0], F.to_host(nat.c0)) and np.array_equal(got[1], F.to_host(nat.c1))
            assert np.array_equal(got[0], F.to_host(py.c0)) and np.array_equal(got[1], F.to_host(py.c1))
        bits = -math.log2(np.abs(decode(kg.decrypt_limb0(*singles[i]), prm.N, scale) - z).max())
        assert bits > 12
    nb.close()


@pytest.mark.gpu
def test_cpp_facade_arithmetic(fides):
    """The C++ facade's EvalMult / EvalSquare / EvalRotate / EvalFastRotation(Precompute) /
    EvalAdd / EvalSub and constant forms under FLEXIBLEAUTO (operands adjusted to a common level
    at its canonical scale S_l, S_(l-1) = S_l^2 / q_(l-1)), and EvalMult + Rescale under
    FIXEDMANUAL, residue for residue against the oracle."""
    import ctypes as C
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 50, 8, 2, name="facade")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=69)
    rk, rot = kg.relin_key(), 5
    kr = kg.rotation_key(rot)
    rk_d, kr_d = F.to_device(rk), F.to_device(kr)
    N, l, q = prm.N, prm.n_q, prm.q
    S = [0.0] * (l + 1)
    S[l] = 2.0 ** 45
    for k in range(l, 1, -1):
        S[k - 1] = S[k] * S[k] / q[k - 1]
    rng = xrng(70)
    a = [uniform_limbs(rng, q, N) for _ in range(2)]
    b = [uniform_limbs(rng, q, N) for _ in range(2)]
    sizes = [l - 1, l, l, l, l, l, l - 1, l - 1, l - 2]
    out = np.zeros(2 * sum(sizes) * N, dtype=np.uint64)
    out_m = np.zeros(2 * (2 * l - 1) * N, dtype=np.uint64)
    err = C.create_string_buffer(512)
    u64 = lambda x: np.ascontiguousarray(x, dtype=np.uint64).ctypes.data_as(C.POINTER(C.c_uint64))
    primes = np.array(q + prm.p, dtype=np.uint64)
    rc = _facade_lib().facade_arith(prm.logN, l, prm.K, prm.dnum, u64(primes), S[l], rk_d.data_ptr(), rot,
                                    kr_d.data_ptr(), l, u64(a[0]), u64(a[1]), u64(b[0]), u64(b[1]), u64(out),
                                    u64(out_m), err, 512)
    assert rc == 0, err.value.decode()
    got, pos = [], 0
    for s_ in sizes:
        c0 = out[pos:pos + s_ * N].reshape(s_, N)
        c1 = out[pos + s_ * N:pos + 2 * s_ * N].reshape(s_, N)
        got.append((c0, c1))
        pos += 2 * s_ * N
    ids = lambda k: list(range(k))
    const = lambda v, k: np.array([[int(v) % q[i]] * N for i in range(k)], dtype=np.uint64)
    mult = o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True)
    kh = round(0.5 * S[l - 1] * q[l - 1] / S[l])
    kadj = round(S[l - 1] * q[l - 1] / S[l])
    adj = [o.rescale(o.mul(a[i], const(kadj, l), ids(l))) for i in range(2)]
    want = [mult,
            o.rotate(a[0], a[1], kr, rot),
            o.rotate(a[0], a[1], kr, rot),
            (o.add(a[0], b[0], ids(l)), o.add(a[1], b[1], ids(l))),
            (o.sub(a[0], b[0], ids(l)), o.sub(a[1], b[1], ids(l))),
            (o.add(a[0], const(round(0.25 * S[l]), l), ids(l)), a[1]),
            tuple(o.rescale(o.mul(a[i], const(kh, l), ids(l))) for i in range(2)),
            o.hmult(a[0], a[1], a[0], a[1], rk, rescale=True),
            o.hmult(mult[0], mult[1], adj[0], adj[1], rk, rescale=True)]
    names = ["EvalMult", "EvalRotate", "EvalFastRotation", "EvalAdd", "EvalSub", "EvalAdd(const)",
             "EvalMult(const)", "EvalSquare", "EvalMult(level-adjusted)"]
    for name, (g0, g1), (w0, w1) in zip(names, got, want):
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), name
    m0 = out_m[:l * N].reshape(l, N)
    m1 = out_m[l * N:2 * l * N].reshape(l, N)
    r0 = out_m[2 * l * N:(3 * l - 1) * N].reshape(l - 1, N)
    r1 = out_m[(3 * l - 1) * N:].reshape(l - 1, N)
    w0, w1 = o.hmult(a[0], a[1], b[0], b[1], rk, rescale=False)
    assert np.array_equal(m0, w0) and np.array_equal(m1, w1), "FIXEDMANUAL EvalMult"
    assert np.array_equal(r0, o.rescale(w0)) and np.array_equal(r1, o.rescale(w1)), "FIXEDMANUAL Rescale"


@pytest.mark.gpu
def test_native_bootstrap_59bit_chain_correction(fides):
    """The reference example's modulus sizes (60-bit q_0, 59-bit scaling primes) at N = 2^12:
    the level-2 input, at a scale close to q_0, is scaled down by 2^9 before ModRaise
    (correction_bits, OpenFHE's correction factor) and decrypts within 2^-12 after bootstrapping."""
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 59, 20, 4, name="boot59 N=2^12")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    ctx = F.Context(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=61, hamming_weight=32)
    S = [0.0] * (prm.n_q + 1)
    S[prm.n_q] = 2.0 ** 59
    for l in range(prm.n_q, 1, -1):
        S[l - 1] = S[l] * S[l] / prm.q[l - 1]
    nb = F.NativeBootstrapper(ctx, top_level=prm.n_q, top_scale=S[prm.n_q], msg_scale=S[2], correction_bits=9)
    keys = [F.to_device(kg.relin_key()), F.to_device(kg.auto_key(2 * prm.N - 1))]
    nb.set_keys(*keys)
    rk = {r: F.to_device(kg.rotation_key(r)) for r in nb.rotations()}
    for r, k in rk.items():
        nb.set_rotation_key(r, k)
    nb.prepare()
    rng = xrng(69)
    n = prm.N // 2
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    c0, c1 = kg.encrypt(encode(z, prm.N, S[2]).astype(np.int64), 2)
    out = nb.bootstrap(F.Ciphertext(F.to_device(c0), F.to_device(c1)))
    got = decode(kg.decrypt_limb0(F.to_host(out.c0), F.to_host(out.c1)), prm.N, nb.out_scale)
    bits = -math.log2(np.abs(got - z).max())
    print(f"59-bit chain bootstrap N=2^12: {bits:.1f} bits, out level {nb.out_level}")
    assert bits > 12
    nb.close()


@pytest.mark.gpu
@pytest.mark.parametrize("baby", [8, 16])
def test_native_double_hoisted_n4096(fides, baby):
    """N = 2^12, the C++ bootstrapper with double-hoisted linear transforms (baby steps and
    giant-step outputs in the extended basis, one ModDown + rescale per transform): the
    precision stays within half a bit of the single-hoisted form's on the same inputs, and a
    batch through fides_bootstrap_batch equals the single bootstraps bit for bit."""
    import torch
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    delta = 2.0 ** 50
    rng = xrng(71)
    n = prm.N // 2
    zs, cts = [], []
    for _ in range(3):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        zs.append(z)
        cts.append(F.Ciphertext(F.to_device(c0), F.to_device(c1)))
    bits = {}
    for dh in (False, True):
        nb = F.NativeBootstrapper(ctx, top_level=prm.n_q, top_scale=ev.S[prm.n_q], msg_scale=delta, K=bs.K, r=bs.r,
                                  degree=bs.degree, baby=baby, prescale_bits=bs.prescale.bit_length() - 1,
                                  double_hoist=dh)
        nb.set_keys(ev.rk, ev.conj_key)
        for r in nb.rotations():
            if r not in ev.rot_keys:
                ev.rot_keys[r] = F.to_device(kg.rotation_key(r))
            nb.set_rotation_key(r, ev.rot_keys[r])
        nb.prepare()
        batch = nb.bootstrap_batch(cts)
        single = nb.bootstrap(cts[1])
        torch.cuda.synchronize()
        assert torch.equal(single.c0, batch[1].c0) and torch.equal(single.c1, batch[1].c1)
        errs = [np.abs(decode(kg.decrypt_limb0(F.to_host(x.c0), F.to_host(x.c1)), prm.N, nb.out_scale) - z).max()
                for x, z in zip(batch, zs)]
        bits[dh] = -math.log2(max(errs))
        if dh and baby == 8:  # the C++ facade's EvalBootstrap in the same form
            host = [(F.to_host(c.c0), F.to_host(c.c1)) for c in cts[:2]]
            fs, fb, L, _ = facade_bootstrap(F, prm, ev, bs, host, double_hoist=True)
            assert L == nb.out_level
            for i in range(2):
                for got in (fs[i], fb[i]):
                    assert np.array_equal(got[0], F.to_host(batch[i].c0)) and np.array_equal(got[1], F.to_host(batch[i].c1))
        nb.close()
    print(f"N=2^12 baby {baby}: single-hoisted {bits[False]:.2f} bits, double-hoisted {bits[True]:.2f} bits")
    assert bits[True] > 12 and bits[True] >= bits[False] - 0.5


@pytest.mark.gpu
def test_native_bootstrap_reduced_noise_n4096(fides):
    """N = 2^12, the C++ bootstrapper on a context with the reduced-noise conversions (the
    reference's Parameters::reducedNoise): every key switch of the bootstrap uses the lifted
    ModUp / ModDown, the result differs from the plain context's and keeps its precision
    (within half a bit, above 12 bits)."""
    import torch
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    delta = 2.0 ** 50
    rng = xrng(73)
    n = prm.N // 2
    zs, cts = [], []
    for _ in range(2):
        z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
        c0, c1 = kg.encrypt(encode(z, prm.N, delta).astype(np.int64), 1)
        zs.append(z)
        cts.append(F.Ciphertext(F.to_device(c0), F.to_device(c1)))
    bits, outs = {}, {}
    for rn in (False, True):
        ctx.set_reduced_noise(rn)
        nb = F.NativeBootstrapper(ctx, top_level=prm.n_q, top_scale=ev.S[prm.n_q], msg_scale=delta, K=bs.K, r=bs.r,
                                  degree=bs.degree, prescale_bits=bs.prescale.bit_length() - 1)
        nb.set_keys(ev.rk, ev.conj_key)
        for r in nb.rotations():
            if r not in ev.rot_keys:
                ev.rot_keys[r] = F.to_device(kg.rotation_key(r))
            nb.set_rotation_key(r, ev.rot_keys[r])
        nb.prepare()
        batch = nb.bootstrap_batch(cts)
        torch.cuda.synchronize()
        outs[rn] = [(F.to_host(x.c0), F.to_host(x.c1)) for x in batch]
        errs = [np.abs(decode(kg.decrypt_limb0(*h), prm.N, nb.out_scale) - z).max() for h, z in zip(outs[rn], zs)]
        bits[rn] = -math.log2(max(errs))
        nb.close()
    ctx.set_reduced_noise(False)
    print(f"N=2^12 bootstrap: plain {bits[False]:.2f} bits, reduced noise {bits[True]:.2f} bits")
    assert not np.array_equal(outs[True][0][0], outs[False][0][0])
    assert bits[True] > 12 and bits[True] >= bits[False] - 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("n_slots", [2048, 100])
def test_cpp_facade_plaintexts(fides, n_slots):
    """The C++ facade's MakeCKKSPackedPlaintext (device encode at the level's canonical scale;
    fewer slots than N/2 are zero-padded to a power of two) and EvalMult / EvalAdd / EvalSub
    with that plaintext under FLEXIBLEAUTO (product rescaled to S_(l-1)) and FIXEDMANUAL (degree
    2, not rescaled): the plaintext's coefficients are within 1 of the host encoder's, its
    limbs are one integer polynomial, and every ciphertext result equals the oracle's
    operations on those limbs residue for residue; a plaintext at another scale is refused."""
    import ctypes as C
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 50, 8, 2, name="facade")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    N, L, q = prm.N, prm.n_q, prm.q
    l = L - 1
    S = [0.0] * (L + 1)
    S[L] = 2.0 ** 45
    for k in range(L, 1, -1):
        S[k - 1] = S[k] * S[k] / q[k - 1]
    rng = xrng(80 + n_slots)
    a = [uniform_limbs(rng, q[:l], N) for _ in range(2)]
    z = rng.uniform(-1, 1, n_slots) + 1j * rng.uniform(-1, 1, n_slots)
    zz = np.stack([z.real, z.imag], axis=1).reshape(-1).copy()
    sizes = [l, l - 1, l, l, l]  # plaintext limbs, then 4 ciphertexts
    out = np.zeros((sizes[0] + 2 * sum(sizes[1:])) * N, dtype=np.uint64)
    err = C.create_string_buffer(512)
    u64 = lambda x: np.ascontiguousarray(x, dtype=np.uint64).ctypes.data_as(C.POINTER(C.c_uint64))
    primes = np.array(q + prm.p, dtype=np.uint64)
    rc = _facade_lib().facade_plain(prm.logN, L, prm.K, prm.dnum, u64(primes), S[L], l, u64(a[0]), u64(a[1]),
                                    zz.ctypes.data_as(C.POINTER(C.c_double)), n_slots, u64(out), err, 512)
    assert rc == 0, err.value.decode()
    ids = list(range(l))
    pt = out[:l * N].reshape(l, N)
    # the encoded polynomial: n_slots zero-padded to n (a power of two), the 2n-ring encoding's
    # coefficients spread with gap N / 2n
    n = 1 << (n_slots - 1).bit_length()
    zp = np.zeros(n, dtype=np.complex128)
    zp[:n_slots] = z
    ref = np.zeros(N)
    ref[::N // (2 * n)] = encode(zp, 2 * n, S[l])
    m = o.ntt(pt, ids, inverse=True)[0].astype(object)
    m = np.array([int(v) - q[0] if int(v) > q[0] // 2 else int(v) for v in m], dtype=np.int64)
    diff = np.abs(m - ref.astype(np.int64))
    assert diff.max() <= 1 and np.count_nonzero(diff) <= max(1, N // 1000)
    assert np.array_equal(pt, o.ntt(small_to_limbs(m, q[:l]), ids))
    pos, got = l * N, []
    for s_ in sizes[1:]:
        got.append((out[pos:pos + s_ * N].reshape(s_, N), out[pos + s_ * N:pos + 2 * s_ * N].reshape(s_, N)))
        pos += 2 * s_ * N
    prod = [o.mul(a[i], pt, ids) for i in range(2)]
    want = [(o.rescale(prod[0]), o.rescale(prod[1])),
            (o.add(a[0], pt, ids), a[1]),
            (o.sub(a[0], pt, ids), a[1]),
            (prod[0], prod[1])]
    for name, (g0, g1), (w0, w1) in zip(["EvalMult(pt)", "EvalAdd(pt)", "EvalSub(pt)", "FIXEDMANUAL EvalMult(pt)"],
                                        got, want):
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), name


@pytest.mark.gpu
def test_cpp_facade_norelin_and_many(fides):
    """The C++ facade's EvalMultNoRelin + Relinearize (three-component ciphertexts; a lazily
    relinearised sum of two products), EvalNegate, EvalAddMany, EvalRotateMany (one batched
    launch sequence) and MultByMonomial against the oracle residue for residue, and the
    FLEXIBLEAUTO Rescale(Relinearize(EvalMultNoRelin)) against the fused product."""
    import ctypes as C
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 50, 8, 2, name="facade")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=69)
    rk, rot = kg.relin_key(), 3
    kr = kg.rotation_key(rot)
    rk_d, kr_d = F.to_device(rk), F.to_device(kr)
    N, l, q = prm.N, prm.n_q, prm.q
    rng = xrng(90)
    a = [uniform_limbs(rng, q, N) for _ in range(2)]
    b = [uniform_limbs(rng, q, N) for _ in range(2)]
    sizes = [l, l, l - 1, l, l, l, l, l]
    out = np.zeros(2 * sum(sizes) * N, dtype=np.uint64)
    err = C.create_string_buffer(512)
    u64 = lambda x: np.ascontiguousarray(x, dtype=np.uint64).ctypes.data_as(C.POINTER(C.c_uint64))
    primes = np.array(q + prm.p, dtype=np.uint64)
    rc = _facade_lib().facade_more(prm.logN, l, prm.K, prm.dnum, u64(primes), 2.0 ** 45, rk_d.data_ptr(), rot,
                                   kr_d.data_ptr(), l, u64(a[0]), u64(a[1]), u64(b[0]), u64(b[1]), u64(out), err, 512)
    assert rc == 0, err.value.decode()
    got, pos = [], 0
    for s_ in sizes:
        got.append((out[pos:pos + s_ * N].reshape(s_, N), out[pos + s_ * N:pos + 2 * s_ * N].reshape(s_, N)))
        pos += 2 * s_ * N
    ids = list(range(l))
    x0, x1, x2 = o.tensor(a[0], a[1], b[0], b[1])
    y0, y1, y2 = o.tensor(a[0], a[1], a[0], a[1])
    s0, s1, s2 = o.add(x0, y0, ids), o.add(x1, y1, ids), o.add(x2, y2, ids)
    f0, f1 = o.keyswitch(s2, rk)
    neg = [o.sub(np.zeros_like(a[i]), a[i], ids) for i in range(2)]
    # X^(N + 5) = -X^5: its limbs in EVALUATION form (the oracle's NTT of the coefficient vector)
    mono = np.zeros((l, N), dtype=np.uint64)
    for i in range(l):
        mono[i, 5] = q[i] - 1
    mono = o.ntt(mono, ids)
    want = [o.hmult(a[0], a[1], b[0], b[1], rk, rescale=False),
            (o.add(s0, f0, ids), o.add(s1, f1, ids)),
            o.hmult(a[0], a[1], b[0], b[1], rk, rescale=True),
            (neg[0], neg[1]),
            (o.add(o.add(a[0], b[0], ids), a[0], ids), o.add(o.add(a[1], b[1], ids), a[1], ids)),
            o.rotate(a[0], a[1], kr, rot),
            o.rotate(b[0], b[1], kr, rot),
            (o.mul(a[0], mono, ids), o.mul(a[1], mono, ids))]
    names = ["Relinearize(EvalMultNoRelin)", "lazy relinearisation of a sum", "FLEXIBLEAUTO NoRelin+Relinearize+Rescale",
             "EvalNegate", "EvalAddMany", "EvalRotateMany[0]", "EvalRotateMany[1]", "MultByMonomial"]
    for name, (g0, g1), (w0, w1) in zip(names, got, want):
        assert np.array_equal(g0, w0) and np.array_equal(g1, w1), name


@pytest.mark.gpu
def test_cpp_facade_bootstrap_to_level_n4096(fides):
    """The facade's EvalBootstrapToLevel at N = 2^12: a request for no more consumed levels than
    EvalBootstrap's gives its result bit for bit; three more consumed levels run the circuit on a
    chain cut short by three limbs at the top (ModRaise to fewer limbs), land exactly three limbs
    lower at that level's canonical scale and keep the precision (> 12 bits, within half a bit)."""
    import ctypes as C
    F = fides
    prm, o, kg, ctx, ev, bs = make_boot(F, 12)
    N, L = prm.N, prm.n_q
    delta = 2.0 ** 50
    rng = xrng(88)
    z = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    c0, c1 = kg.encrypt(encode(z, N, delta).astype(np.int64), 1)
    lib = _facade_lib()
    vp, u64p = C.c_void_p, C.POINTER(C.c_uint64)
    lib.facade_bootstrap_to_level.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, C.c_double, vp, vp, C.c_int,
                                              C.POINTER(C.c_int), C.POINTER(vp), C.c_double, C.c_int, C.c_int, u64p,
                                              u64p, u64p, u64p, u64p, u64p, u64p, u64p, C.POINTER(C.c_int),
                                              C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_char_p, C.c_int]
    rots = sorted(ev.rot_keys)
    outs = [np.zeros((L, N), dtype=np.uint64) for _ in range(6)]
    u64 = lambda x: np.ascontiguousarray(x, dtype=np.uint64).ctypes.data_as(u64p)
    lvl_d, lvl_t, sc_t = C.c_int(), C.c_int(), C.c_double()
    err = C.create_string_buffer(512)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    rc = lib.facade_bootstrap_to_level(prm.logN, L, prm.K, prm.dnum, u64(primes), ev.S[L], ev.rk.data_ptr(),
                                       ev.conj_key.data_ptr(), len(rots), (C.c_int * len(rots))(*rots),
                                       (vp * len(rots))(*[ev.rot_keys[r].data_ptr() for r in rots]), delta,
                                       bs.prescale.bit_length() - 1, 3, u64(c0), u64(c1), *[u64(x) for x in outs],
                                       C.byref(lvl_d), C.byref(lvl_t), C.byref(sc_t), err, 512)
    assert rc == 0, err.value.decode()
    ld, lt = lvl_d.value, lvl_t.value
    assert lt == ld - 3
    assert np.array_equal(outs[0][:ld], outs[2][:ld]) and np.array_equal(outs[1][:ld], outs[3][:ld])
    S = [0.0] * (L + 1)
    S[L] = ev.S[L]
    for k in range(L, 1, -1):
        S[k - 1] = S[k] * S[k] / prm.q[k - 1]
    assert abs(sc_t.value / S[lt] - 1) < 1e-12
    bits = lambda x0, x1, l, sc: -math.log2(np.abs(decode(kg.decrypt_limb0(x0[:l], x1[:l]), N, sc) - z).max())
    b_d = bits(outs[0], outs[1], ld, S[ld])
    b_t = bits(outs[4], outs[5], lt, sc_t.value)
    print(f"N=2^12 bootstrap: {ld} limbs {b_d:.2f} bits; to level (3 deeper): {lt} limbs {b_t:.2f} bits")
    assert b_t > 12 and b_t >= b_d - 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("row_size,b_step,stride,offset", [(14, 4, 1, 3), (8, 8, 2, 0), (5, 2, 3, -2), (38, 18, 1, 0)])
def test_cpp_facade_linear_transform(fides, row_size, b_step, stride, offset):
    """The facade's LinearTransform / LinearTransformMany (the reference's BSGS contract:
    pre-rotated diagonals r_k = -bStep (k / bStep) stride - offset, hoisted baby steps, giant
    steps folded from the top, the offset rotation last) decrypt, after Rescale, to the FP64
    y[i] = sum_k x[i + k stride + offset] D_k[i]; the batched form's first set equals the single
    transform bit for bit and its second (negated diagonals) gives -y."""
    import ctypes as C
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 50, 8, 2, name="facade")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    kg = KeyGen(o, seed_stream=91)
    N, l = prm.N, prm.n_q
    n = N // 2
    rots = sorted(set([i * stride for i in range(1, b_step + 1)] + ([offset] if offset else [])))
    keys = {r: F.to_device(kg.rotation_key(r)) for r in rots}
    top = 2.0 ** 45
    S = [0.0] * (l + 1)
    S[l] = top
    for k in range(l, 1, -1):
        S[k - 1] = S[k] * S[k] / prm.q[k - 1]
    rng = xrng(92 + row_size)
    x = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    D = rng.uniform(-1, 1, (row_size, n)) + 1j * rng.uniform(-1, 1, (row_size, n))
    # diagonals[k] = Rot(D_k, r_k): slot i holds D_k[i + r_k]
    pre = [np.roll(D[k], b_step * (k // b_step) * stride + offset) for k in range(row_size)]
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
                                     (C.c_int * len(rots))(*rots), (C.c_void_p * len(rots))(*[keys[r].data_ptr() for r in rots]),
                                     l, u64(c0), u64(c1), row_size, b_step, stride, offset, dz.ctypes.data_as(dp), n,
                                     0, u64(out), C.byref(sc), err, 512)
    assert rc == 0, err.value.decode()
    res = [out[i * 2 * lo * N:(i + 1) * 2 * lo * N].reshape(2, lo, N) for i in range(3)]
    want = sum(np.roll(x, -(k * stride + offset)) * D[k] for k in range(row_size))
    got = decode(kg.decrypt_limb0(res[0][0], res[0][1]), N, sc.value)
    assert np.abs(got - want).max() < 1e-6
    assert np.array_equal(res[1], res[0])
    got_neg = decode(kg.decrypt_limb0(res[2][0], res[2][1]), N, sc.value)
    assert np.abs(got_neg + want).max() < 1e-6


@pytest.mark.gpu
def test_cpp_facade_raw_plaintext_and_params(fides):
    """The reference's raw exchange formats in the C++ layer: a context built from RawParams
    (Parameters::adaptTo), a device-encoded plaintext exported as RawPlainText in EVALUATION,
    COEFFICIENT and natural-order EVALUATION form and loaded back unchanged; the COEFFICIENT
    export is the encoder's integer polynomial (within 1 of the host encoder's coefficients) and
    the EVALUATION export its NTT (the oracle's), the natural-order one the same residues permuted."""
    import ctypes as C
    from fides_b200 import params as P
    F = fides
    prm = P.chain(12, 60, 50, 6, 2, name="raw")
    o = O.Oracle(prm.logN, prm.q, prm.p, prm.dnum)
    N, L = prm.N, prm.n_q
    rng = xrng(95)
    z = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    zz = np.stack([z.real, z.imag], axis=1).reshape(-1).copy()
    outs = [np.zeros((L, N), dtype=np.uint64) for _ in range(3)]
    lib = _facade_lib()
    u64p, dp = C.POINTER(C.c_uint64), C.POINTER(C.c_double)
    lib.facade_raw_plaintext.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_double, dp, C.c_int,
                                         u64p, u64p, u64p, C.c_char_p, C.c_int]
    u64 = lambda a: np.ascontiguousarray(a, dtype=np.uint64).ctypes.data_as(u64p)
    err = C.create_string_buffer(512)
    primes = np.array(prm.q + prm.p, dtype=np.uint64)
    psi = np.array(o.psi, dtype=np.uint64)
    top = 2.0 ** 45
    rc = lib.facade_raw_plaintext(prm.logN, L, prm.K, prm.dnum, u64(primes), u64(psi), top, zz.ctypes.data_as(dp),
                                  N // 2, *[u64(x) for x in outs], err, 512)
    assert rc == 0, err.value.decode()
    ev_, co_, na_ = outs
    ids = list(range(L))
    assert np.array_equal(o.ntt(co_, ids), ev_)
    m = np.array([int(v) - prm.q[0] if int(v) > prm.q[0] // 2 else int(v) for v in co_[0]], dtype=np.int64)
    ref = encode(z, N, top).astype(np.int64)
    diff = np.abs(m - ref)
    assert diff.max() <= 1 and np.count_nonzero(diff) <= max(1, N // 1000)
    for j in range(L):
        assert np.array_equal(np.sort(na_[j]), np.sort(ev_[j]))
