"""Collision detection of the substrate generator, restated in numpy — TEST
INFRASTRUCTURE ONLY (tests/ import it; the product never does).

Restates collide_spheres_gpu (simulation_toolkit/substrate_generator/helper/
CollisionDetection.py:10-50) with intersect_block (:52-63) and set_segments
(:65-115): blocks of edge Lx/10 (float32), ceil(L/block) per axis; a sphere
belongs to a block when all six boundary distances, evaluated in float32 in
the reference's operation order (:76-86), are below jump_tol = 1; a pair of
spheres of different fibres collides when (r_a + r_b + buff) - |x_a - x_b| > 0
in float32, and is found when the two spheres share a block.  Result: the
(a < b) rows, unique, in lexicographic order.  Candidate pairs come from a
k-d tree over the centres (within the largest possible collision distance),
then every candidate is tested exactly as above.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def block_grid(Lx, Ly, Lz):
    """(n [3] int, d [3] float32 block edges, h [3] float32 half box) in float32."""
    Lf = np.array([Lx, Ly, Lz], f32)
    block = f32(Lf[0] / f32(10))
    n = np.ceil(Lf / block).astype(np.int64)
    d = (Lf / n.astype(f32)).astype(f32)
    return n, d, (Lf / f32(2)).astype(f32)


def block_ranges(pos, r, Lx, Ly, Lz, jump_tol=1.0):
    """[S, 3, 2] first and last block per axis a sphere belongs to (lo > hi:
    none).  The two distances per axis, n*dL - r - x - L/2 and
    x - ((n+1)*dL + r - L/2), are evaluated for every block index."""
    n, d, h = block_grid(Lx, Ly, Lz)
    pos = np.asarray(pos, f32)
    r = np.asarray(r, f32)
    out = np.zeros((pos.shape[0], 3, 2), np.int64)
    for ax in range(3):
        idx = np.arange(n[ax])
        t0 = ((idx[None, :].astype(f32) * d[ax] - r[:, None]) - pos[:, ax:ax + 1]) - h[ax]
        t1 = pos[:, ax:ax + 1] - ((((idx + 1)[None, :].astype(f32) * d[ax]) + r[:, None]) - h[ax])
        ok = (t0 < f32(jump_tol)) & (t1 < f32(jump_tol))
        anyok = ok.any(axis=1)
        lo = np.where(anyok, ok.argmax(axis=1), 1)
        hi = np.where(anyok, n[ax] - 1 - ok[:, ::-1].argmax(axis=1), 0)
        out[:, ax, 0], out[:, ax, 1] = lo, hi
    return out


def collide(pos, r, fid, Lx, Ly, Lz, buff=0.0):
    """(M, 2) int64 colliding pairs, as the reference returns them."""
    from scipy.spatial import cKDTree
    pos = np.asarray(pos, f32)
    r = np.asarray(r, f32)
    fid = np.asarray(fid, f32)
    if pos.shape[0] < 2:
        return np.zeros((0, 2), np.int64)
    rng = block_ranges(pos, r, Lx, Ly, Lz)
    reach = 2.0 * float(r.max()) + abs(float(buff)) + 1e-3
    cand = cKDTree(pos.astype(np.float64)).query_pairs(reach, output_type="ndarray")
    if cand.size == 0:
        return np.zeros((0, 2), np.int64)
    a, b = cand[:, 0], cand[:, 1]
    dx, dy, dz = (pos[a, k] - pos[b, k] for k in range(3))
    dm = np.sqrt((dx * dx + dy * dy) + dz * dz)
    hit = ((r[a] + r[b]) + f32(buff)) - dm > f32(0)
    hit &= fid[a] != fid[b]
    share = np.ones(a.size, bool)
    for ax in range(3):
        share &= np.maximum(rng[a, ax, 0], rng[b, ax, 0]) <= np.minimum(rng[a, ax, 1], rng[b, ax, 1])
    pairs = np.sort(cand[hit & share], axis=1)
    return np.unique(pairs, axis=0).astype(np.int64)


def margin(pos, r, fid, buff=0.0):
    """Smallest |(r_a + r_b + buff) - |x_a - x_b|| over pairs of different
    fibres within reach, in float64: how far the closest call is from the
    threshold (a fixture whose margin is far above float32 rounding gives the
    same pairs whatever order the distance is summed in)."""
    from scipy.spatial import cKDTree
    pos = np.asarray(pos, np.float64)
    r = np.asarray(r, np.float64)
    cand = cKDTree(pos).query_pairs(2.0 * r.max() + abs(buff) + 1e-3, output_type="ndarray")
    a, b = cand[:, 0], cand[:, 1]
    keep = np.asarray(fid)[a] != np.asarray(fid)[b]
    v = (r[a] + r[b] + buff) - np.linalg.norm(pos[a] - pos[b], axis=1)
    return float(np.abs(v[keep]).min())
