"""The walk's random draws, pinned on the CPU.

The fused and plain walks draw their steps from Philox4x32-10 (Salmon,
Moraes, Dror & Shaw, SC'11) through a Box-Muller transform written with IEEE
single operations only.  The GPU draws equal the oracle's bit for bit (the
Philox walks of tests/test_gpu_parity.py match the oracle exactly), so pinning
the oracle's generator pins the product's:

* the block function against the known-answer vectors published with the
  Random123 library (the SC'11 authors' reference implementation), and
  against a big-integer restatement here on random counters and keys;
* the counter layout (walker, step, draw, stream) and the transform against
  float64 Box-Muller of the same words: the series logarithm and the
  quadrant sine/cosine stay within a few float32 rounding errors;
* the normals' distribution (moments, Kolmogorov-Smirnov, no correlation
  between the normals of one block).

The reference draws with cuRAND XORWOW (sim3d_kernel.cu:61-70, :403-405),
which is not reproduced; walks with these draws agree with the reference's
statistically (tests/test_reference_gpu.py)."""
import numpy as np
import pytest

from oracle import oracle as oz

M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF

# Philox4x32-10 known answers: (counter, key) -> output, from Random123's
# published test vectors.
KAT = [
    ((0x00000000, 0x00000000, 0x00000000, 0x00000000), (0x00000000, 0x00000000),
     (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF),
     (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox_py(c, k):
    """Philox4x32-10 with Python integers: ten rounds of two 32x32->64
    multiplies, the key bumped by the Weyl constants between rounds."""
    c0, c1, c2, c3 = c
    k0, k1 = k
    for r in range(10):
        if r:
            k0, k1 = (k0 + W0) & MASK, (k1 + W1) & MASK
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = (p1 >> 32) ^ c1 ^ k0, p1 & MASK, (p0 >> 32) ^ c3 ^ k1, p0 & MASK
    return c0, c1, c2, c3


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert tuple(int(v) for v in oz.philox_block(ctr, *key)) == want
    assert philox_py(ctr, key) == want


def test_philox_block_matches_restatement():
    rng = np.random.default_rng(8)
    for _ in range(500):
        c = tuple(int(v) for v in rng.integers(0, 2**32, 4, dtype=np.uint64))
        k = tuple(int(v) for v in rng.integers(0, 2**32, 2, dtype=np.uint64))
        assert tuple(int(v) for v in oz.philox_block(c, *k)) == philox_py(c, k)


def _box_muller64(ua, ub):
    """Float64 Box-Muller of the oracle's word mapping: u = ua 2^-32 + 2^-33
    in (0, 1]; angle (q + t) pi/2 with q = ub >> 30 and t = (ub mod 2^30)
    2^-30 - 1/2.  u and t are first rounded as the oracle forms them (the word
    to float32, then one fused multiply-add), so what remains is the error of
    the transform itself, not the 24-bit resolution of its inputs."""
    f32 = lambda v: v.astype(np.float32).astype(np.float64)  # noqa: E731
    u = f32(f32(ua) * 2.0**-32 + 2.0**-33)
    rad = np.sqrt(-2.0 * np.log(u))
    q = (ub >> 30).astype(np.float64)
    t = f32(f32(ub & 0x3FFFFFFF) * 2.0**-30 - 0.5)
    ang = (q + t) * (np.pi / 2)
    return rad * np.cos(ang), rad * np.sin(ang)


def test_normals_layout_and_accuracy():
    """Normals of walkers 0..N-1, draws 0..3 at one step: counter (walker,
    step, draw, stream); words (0, 1) give normals 0 and 1, words (2, 3) give
    normal 2.  Each within 8 float32 rounding errors (relative to
    max(1, |n|)) of float64 Box-Muller of the same rounded inputs."""
    k0, k1, stream, step, N, nd = 0x1234567, 0x89ABCDEF, 3, 4321, 4000, 4
    got = oz.philox_normals(k0, k1, stream, N, step, nd).astype(np.float64)
    w, d = np.meshgrid(np.arange(N), np.arange(nd), indexing="ij")
    words = np.array([philox_py((int(a), step, int(b), stream), (k0, k1))
                      for a, b in zip(w.ravel(), d.ravel())], dtype=np.uint64).reshape(N, nd, 4)
    n0, n1 = _box_muller64(words[..., 0], words[..., 1])
    n2, _ = _box_muller64(words[..., 2], words[..., 3])
    want = np.stack([n0, n1, n2], axis=-1)
    err = np.abs(got - want) / np.maximum(1.0, np.abs(want))
    assert err.max() <= 8 * 2.0**-24, err.max()


def test_box_muller_extremes_and_quadrants():
    """The word range's ends and every quadrant boundary: finite normals,
    within the same bound.  ua = 0 gives the largest radius,
    sqrt(2 * 33 ln 2) = 6.76; ua = 2^32 - 1 rounds u to 1 and the radius to 0."""
    edges = np.array([0, 1, 2**23, 2**24 - 1, 2**31, 2**32 - 2**8, 2**32 - 1], np.uint64)
    quads = np.array([q << 30 | m for q in range(4) for m in (0, 1, 2**29, 2**30 - 1)], np.uint64)
    ua, ub = (g.ravel() for g in np.meshgrid(edges, quads, indexing="ij"))
    got = oz.box_muller_pairs(ua, ub).astype(np.float64)
    assert np.isfinite(got).all()
    want = np.stack(_box_muller64(ua, ub), axis=-1)
    err = np.abs(got - want) / np.maximum(1.0, np.abs(want))
    assert err.max() <= 8 * 2.0**-24, err.max()
    r = np.hypot(got[:, 0], got[:, 1])
    assert abs(r[ua == 0].max() - np.sqrt(66 * np.log(2))) < 1e-5
    assert r[ua == 2**32 - 1].max() == 0.0


def test_normals_distribution():
    from scipy import stats
    x = oz.philox_normals(7, 11, 0, 200_000, 17, 1).reshape(-1, 3).astype(np.float64)
    n = x.shape[0]
    for j in range(3):
        assert abs(x[:, j].mean()) < 5 / np.sqrt(n)
        assert abs(x[:, j].var() - 1) < 5 * np.sqrt(2 / n)
        assert stats.kstest(x[:, j], "norm").pvalue > 1e-4
    c = np.corrcoef(x.T)
    assert np.abs(c[np.triu_indices(3, 1)]).max() < 5 / np.sqrt(n)
    # consecutive steps of one walker are independent too
    y = oz.philox_normals(7, 11, 0, 200_000, 18, 1).reshape(-1, 3).astype(np.float64)
    assert abs(np.corrcoef(x[:, 0], y[:, 0])[0, 1]) < 5 / np.sqrt(n)
