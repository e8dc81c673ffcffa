"""Device slot encode / decode (fides_encode / fides_decode) against the host encoder.

The encoder is floating point followed by a rounding, so its parity bar is: every integer
coefficient within 1 of the host encoder's (FP64 numpy FFT of the same canonical embedding)
and at most 1 in 10^3 coefficients off at all (values within ~2^-10 of a rounding tie at
scale 2^45, where the two FFTs' last-bit differences decide; 7 of 65536 measured); every limb of the output
is then bit-exact with the oracle's NTT of those coefficients (the modular half is integer
work).  Decode: slots within 1e-9 of the host decoder's at scale 2^40.  The reference's
device encode documents the same contract: "numerically the same plaintext, not a guaranteed
byte-identical one" (src/CKKS/DeviceEncodeBatch.cu, ifft tables comment)."""
import numpy as np
import pytest

import oracle as O
from ckks_host import decode, encode, small_to_limbs, xrng

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def C(fides):
    from fides_b200 import params as P
    prm = P.config_c(4)
    return prm, O.Oracle(prm.logN, prm.q, prm.p, prm.dnum), fides.Context(prm.logN, prm.q, prm.p, prm.dnum)


def device_coeffs(fides, ctx, pt, q):
    """Centred integer coefficients of every limb of a device plaintext (INTT on the GPU)."""
    import torch
    x = pt.clone()
    ctx.intt(x)
    h = fides.to_host(x).astype(object)
    rows = [np.array([int(v) - q[j] if int(v) > q[j] // 2 else int(v) for v in h[j]], dtype=np.int64)
            for j in range(h.shape[0])]
    return rows


def check_encoded(fides, o, ctx, pt, ref_coeff, q, level):
    rows = device_coeffs(fides, ctx, pt[:1], q)
    m = rows[0]
    diff = np.abs(m - ref_coeff.astype(np.int64))
    assert diff.max() <= 1 and np.count_nonzero(diff) <= max(1, len(m) // 1000)
    ids = list(range(level))
    exp = o.ntt(small_to_limbs(m, q[:level]), ids)
    assert np.array_equal(fides.to_host(pt), exp)


@pytest.mark.parametrize("level", [30, 1])
def test_encode_full_slots(fides, C, level):
    import torch
    prm, o, ctx = C
    N = prm.N
    rng = xrng(2000 + level)
    z = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    pt = ctx.encode(torch.from_numpy(z), 2.0 ** 45, level)
    assert pt.shape == (level, N)
    check_encoded(fides, o, ctx, pt, encode(z, N, 2.0 ** 45), prm.q, level)


@pytest.mark.parametrize("n", [1, 8, 1024, 8192])
def test_encode_sparse_slots(fides, C, n):
    """n < N/2 slots: the coefficients of the 2n-ring encoding spread with gap N / 2n."""
    import torch
    prm, o, ctx = C
    N = prm.N
    rng = xrng(2100 + n)
    z = rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)
    pt = ctx.encode(torch.from_numpy(z), 2.0 ** 40, 6)
    small = encode(z, 2 * n, 2.0 ** 40)
    ref = np.zeros(N)
    ref[::N // (2 * n)] = small
    check_encoded(fides, o, ctx, pt, ref, prm.q, 6)
    back = ctx.decode(pt, 2.0 ** 40, n_slots=n).cpu().numpy()
    assert np.abs(back - z).max() < 1e-9


def test_decode_matches_host_decoder(fides, C):
    import torch
    prm, o, ctx = C
    N = prm.N
    rng = xrng(2200)
    m = np.round(rng.normal(0, 2.0 ** 40, N)).astype(np.int64)
    limbs = o.ntt(small_to_limbs(m, prm.q[:3]), [0, 1, 2])
    got = ctx.decode(fides.to_device(limbs), 2.0 ** 40).cpu().numpy()
    assert np.abs(got - decode(m, N, 2.0 ** 40)).max() < 1e-9


def test_encode_batch_equals_singles_and_roundtrip(fides, C):
    import torch
    prm, o, ctx = C
    N = prm.N
    rng = xrng(2300)
    zs = rng.uniform(-1, 1, (5, N // 2)) + 1j * rng.uniform(-1, 1, (5, N // 2))
    pts = ctx.encode(torch.from_numpy(zs), 2.0 ** 40, 12)
    assert pts.shape == (5, 12, N)
    for i in range(5):
        assert torch.equal(pts[i], ctx.encode(torch.from_numpy(zs[i]), 2.0 ** 40, 12))
    back = ctx.decode(pts, 2.0 ** 40).cpu().numpy()
    assert np.abs(back - zs).max() < 1e-9


def test_encode_overflow_sets_status_and_bad_sizes_raise(fides, C):
    import torch
    prm, o, ctx = C
    N = prm.N
    ctx.device_status(clear=True)
    z = np.full(N // 2, 1.0 + 0j)
    ctx.encode(torch.from_numpy(z), 2.0 ** 66, 2)  # coefficients ~2^66 beyond the 2^62 limit
    assert ctx.device_status(clear=True) & 2
    ctx.encode(torch.from_numpy(z), 2.0 ** 40, 2)
    assert ctx.device_status(clear=True) == 0
    with pytest.raises(fides.FidesError):
        ctx.encode(torch.from_numpy(np.ones(3, dtype=np.complex128)), 2.0 ** 40, 2)
    with pytest.raises(fides.FidesError):
        ctx.encode(torch.from_numpy(np.ones(N, dtype=np.complex128)), 2.0 ** 40, 2)
