"""Collision detection of the substrate generator (collide_spheres_gpu,
substrate_generator/helper/CollisionDetection.py:10-62).

* CPU: the oracle's numpy restatement (oracle/collide_oracle.py) equals the
  reference function's own output (tests/golden/collision.npz, made by
  make_golden.py from a seeded, jittered 500-axon bundle; buff 0 and 0.05 um)
  pair for pair.  The fixture's closest call lies 1.4e-5 um from the
  threshold, far above float32 rounding, so summation order cannot flip it.
* GPU: nz_collide_cells / nz_collide_pairs / nz_pairs_sort give the same
  pairs, in the same order; and equal the oracle on a seeded substrate of
  60,000 random spheres of 300 fibres, some outside the grid (which take
  part in no pair in either).
"""
import numpy as np
import pytest

from oracle.collide_oracle import collide


def _fixture():
    from tests._fixtures import GOLDEN
    return np.load(GOLDEN / "collision.npz")


def test_oracle_matches_reference_collision_pairs():
    z = _fixture()
    for i in (0, 1):
        pairs = collide(z["pos"], z["radii"], z["fiber_id"], *z["L"], buff=float(z[f"buff{i}"]))
        np.testing.assert_array_equal(pairs, z[f"pairs{i}"].astype(np.int64))
        assert z[f"margin{i}"] > 1e-5


def _random_spheres(S=60_000, nfib=300, L=(60.0, 60.0, 40.0), seed=13):
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.uniform(-L[k] / 2 - 3.0, L[k] / 2 + 3.0, S) for k in range(3)], axis=1).astype(np.float32)
    r = rng.uniform(0.3, 1.2, S).astype(np.float32)
    fid = rng.integers(0, nfib, S).astype(np.float32)
    return pos, r, fid, L


@pytest.mark.gpu
def test_device_collision_matches_reference_fixture():
    torch = pytest.importorskip("torch")
    from nozomi_b200.collide import detect_collision
    z = _fixture()
    for i in (0, 1):
        pairs = detect_collision(torch.from_numpy(z["pos"]), z["radii"], z["fiber_id"], *z["L"],
                                 buff=float(z[f"buff{i}"]))
        np.testing.assert_array_equal(pairs.cpu().numpy(), z[f"pairs{i}"].astype(np.int64))


@pytest.mark.gpu
def test_device_collision_matches_oracle_on_random_spheres():
    import time
    torch = pytest.importorskip("torch")
    from nozomi_b200.collide import detect_collision
    pos, r, fid, L = _random_spheres()
    t0 = time.perf_counter()
    ref = collide(pos, r, fid, *L, buff=0.02)
    t_cpu = time.perf_counter() - t0
    detect_collision(pos, r, fid, *L, buff=0.02)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    got = detect_collision(pos, r, fid, *L, buff=0.02)
    torch.cuda.synchronize()
    t_gpu = time.perf_counter() - t0
    assert ref.shape[0] > 10_000
    np.testing.assert_array_equal(got.cpu().numpy(), ref)
    print(f"{len(pos)} spheres, {ref.shape[0]} pairs: oracle {t_cpu * 1e3:.0f} ms, device {t_gpu * 1e3:.1f} ms")


def test_block_grid_is_the_reference_grid():
    """The product's grid (float32: blocks of Lx/10, ceil(L/block) per axis,
    edges L/n) equals the oracle's, including boxes where float32 rounding
    of L/(L/10) decides between 10 and 11 blocks."""
    from nozomi_b200.collide import block_grid
    from oracle.collide_oracle import block_grid as oracle_grid
    for L in ((60.0, 60.0, 40.0), (69.53915176460134, 69.53915176460134, 40.0), (9.734261, 9.734261, 40.0),
              (33.3, 33.3, 100.1)):
        g = block_grid(*L)
        n, d, _ = oracle_grid(*L)
        assert (g.nx, g.ny, g.nz) == tuple(int(v) for v in n)
        assert np.array([g.dLx, g.dLy, g.dLz], np.float32).tobytes() == d.tobytes()
