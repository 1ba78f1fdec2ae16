"""Substrate ingestion on the GPU (nz_ingest_split / plan / write) against
the reference's own code and the host restatement.

* bit for bit against tests/golden/ingestion.npz, made by running the
  reference's split_matrix_to_list and createBoundaryZ (utils/common_utils.py:
  41-55, utils/adjust_geometry.py:3-36) on a matrix whose fibres continue
  through the z face as another fibre, as themselves, or not at all;
* bit for bit against the host restatement (split_fibers + bound_z) on a
  seeded matrix of about 1e5 spheres with the same three kinds of fibre, a
  partner claimed by two fibres, end keys repeated (the last fibre with a
  key wins) and rows after the last fibre (dropped); the two timings are
  printed;
* fibres too short for the pad are refused, as the reference's create_pad
  fails on them.
"""
import time

import numpy as np
import pytest

from nozomi_b200 import substrates as sb

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def synthetic_matrix(n_fibres=1000, n_per=100, L=100.0, seed=3):
    """Fibres along z in a cubic box of edge L, each ending exactly at
    z = L/2: a third straight (their own partner), a third starting where
    the straight fibre before them ends (whose end two fibres then claim),
    a third tilted (no partner); then a few stray rows after the last
    fibre."""
    rng = np.random.default_rng(seed)
    z = np.linspace(-L / 2, L / 2, n_per + 1)[1:]
    assert z[-1] == L / 2
    rows = []
    xy = rng.uniform(-L / 2, L / 2, (n_fibres, 2))
    for k in range(n_fibres):
        kind = k % 3
        x0, y0 = xy[k]
        if kind == 0:
            x1, y1 = x0, y0
        elif kind == 1:
            # start where the straight fibre k-1 ends
            x0, y0, x1, y1 = xy[k - 1][0], xy[k - 1][1], xy[k][0], xy[k][1]
        else:
            x1, y1 = x0 + 0.5, y0 - 0.25
        t = np.linspace(0.0, 1.0, n_per)
        f = np.stack([x0 + (x1 - x0) * t, y0 + (y1 - y0) * t, z, rng.uniform(0.4, 1.2, n_per),
                      np.full(n_per, k + 0.7)], axis=1)
        rows.append(f)
    tail = np.stack([rng.uniform(-L / 2, L / 2, 7), rng.uniform(-L / 2, L / 2, 7), np.linspace(-10, 10, 7),
                     np.full(7, 0.5), np.full(7, 1e6)], axis=1)
    return np.concatenate(rows + [tail]), L


def test_ingestion_on_device_matches_reference_golden():
    from tests._fixtures import GOLDEN
    z = np.load(GOLDEN / "ingestion.npz")
    A, L = z["matrix"], float(z["L"])
    rows, spheres, lengths = sb.ingest_on_device(A, L)
    np.testing.assert_array_equal(lengths, z["lengths"])
    np.testing.assert_array_equal(rows.cpu().numpy(), z["fibres"])
    sph = spheres.cpu().numpy()
    np.testing.assert_array_equal(sph[:4], z["fibres"][:, :4].T)
    np.testing.assert_array_equal(sph[4], np.repeat(np.arange(len(lengths)), lengths).astype(np.float64))


def test_ingestion_on_device_matches_host_on_1e5_spheres():
    A, L = synthetic_matrix()
    # a partner claimed twice and a repeated end key: fibre 3's start is
    # fibre 0's end too, and fibre 6 ends where fibre 0 ends (the later wins)
    A[3 * 100, :2] = A[0 * 100 + 99, :2]
    A[6 * 100 + 99, :2] = A[0 * 100 + 99, :2]
    t0 = time.perf_counter()
    host = sb.bound_z(sb.split_fibers(A.copy(), L), L)
    t_host = time.perf_counter() - t0
    Ad = torch.from_numpy(A).cuda()
    sb.ingest_on_device(Ad, L)  # warm: library load and allocations
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rows, spheres, lengths = sb.ingest_on_device(Ad, L)
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    ref = np.concatenate(host)
    assert rows.shape[0] == ref.shape[0] > 1e5
    np.testing.assert_array_equal(lengths, [f.shape[0] for f in host])
    np.testing.assert_array_equal(rows.cpu().numpy(), ref)
    print(f"ingestion of {A.shape[0]} rows -> {ref.shape[0]} spheres: host {t_host * 1e3:.1f} ms, "
          f"device {t_dev * 1e3:.2f} ms (incl. two size reads)")


def test_short_fibres_refused():
    from nozomi_b200._lib import NozomiError
    A, L = synthetic_matrix(n_fibres=6, n_per=20)  # 20 rows < 25: a padded fibre cannot be built
    with pytest.raises(NozomiError, match="fewer than 25"):
        sb.ingest_on_device(A, L)
    rows, spheres, lengths = sb.ingest_on_device(A[:0], L)
    assert rows.shape == (0, 5) and spheres.shape == (5, 0) and lengths.size == 0
