"""Cell-list oracle — TEST INFRASTRUCTURE ONLY (numpy).

Restates ``DiffSim3d.set_segments`` (simulation_toolkit/simulation_engine/
diffsim3d.py:107-174): a sphere belongs to cell (n, m, p) when, on every axis,
neither boundary distance of its bounding box to the cell reaches ``jump_tol``
(``in_segment < jump_tol``, :128-141); K is the largest member count (:144);
each cell's list holds the K spheres of smallest ``in_segment``, sorted by
index (:167), at offset K*(p*nx*ny + m*nx + n) (:166).  The reference sorts with
numpy's default (unstable) argsort, which leaves the order of equal
``in_segment`` values unspecified; here ties are broken by lower sphere index
(a stable sort), which decides only which non-member pads a cell when two pads
tie at the K-th place.

All arithmetic is float64 in the reference's operation order.
"""
from __future__ import annotations

import numpy as np


def in_segment(spheres: np.ndarray, L, nseg, cell) -> np.ndarray:
    """``in_segment`` of every sphere for one cell (diffsim3d.py:128-139)."""
    Lx, Ly, Lz = (float(v) for v in L)
    nx, ny, nz = nseg
    n, m, p = cell
    dLx, dLy, dLz = Lx / nx, Ly / ny, Lz / nz
    sx, sy, sz, sr = spheres[0], spheres[1], spheres[2], spheres[3]
    inx_min = n * dLx - sr - sx - Lx / 2
    inx_max = sx - ((n + 1) * dLx + sr - Lx / 2)
    iny_min = m * dLy - sr - sy - Ly / 2
    iny_max = sy - ((m + 1) * dLy + sr - Ly / 2)
    inz_min = p * dLz - sr - sz - Lz / 2
    inz_max = sz - ((p + 1) * dLz + sr - Lz / 2)
    v = np.maximum(inx_min, inx_max)
    v = np.maximum(v, iny_min)
    v = np.maximum(v, iny_max)
    v = np.maximum(v, inz_min)
    v = np.maximum(v, inz_max)
    return v


def segments_reference(spheres: np.ndarray, L, nseg, jump_tol: float = 1.0):
    """(K, segments int32 [ncell*K]) as ``set_segments`` builds them."""
    spheres = np.asarray(spheres, dtype=np.float64)
    nx, ny, nz = nseg
    vals = {}
    K = 0
    for n in range(nx):
        for m in range(ny):
            for p in range(nz):
                v = in_segment(spheres, L, nseg, (n, m, p))
                vals[(n, m, p)] = v
                K = max(K, int(np.count_nonzero(v < jump_tol)))
    seg = np.zeros(nx * ny * nz * K, dtype=np.int32)
    for (n, m, p), v in vals.items():
        off = K * (p * nx * ny + m * nx + n)
        seg[off:off + K] = np.sort(np.argsort(v, kind="stable")[:K])
    return K, seg


def cells_members(spheres: np.ndarray, L, nseg, jump_tol: float = 1.0):
    """Compact lists of members only: (start, count, items), cells in the
    reference's order, items ascending within a cell."""
    spheres = np.asarray(spheres, dtype=np.float64)
    nx, ny, nz = nseg
    ncell = nx * ny * nz
    lists = [None] * ncell
    for n in range(nx):
        for m in range(ny):
            for p in range(nz):
                v = in_segment(spheres, L, nseg, (n, m, p))
                lists[p * nx * ny + m * nx + n] = np.nonzero(v < jump_tol)[0].astype(np.int32)
    count = np.array([len(x) for x in lists], dtype=np.int32)
    start = np.zeros(ncell, dtype=np.int32)
    if ncell > 1:
        start[1:] = np.cumsum(count)[:-1]
    items = np.concatenate(lists).astype(np.int32) if ncell else np.zeros(0, np.int32)
    return start, count, items


def padded_as_lists(K: int, segments: np.ndarray, ncell: int):
    """The padded table seen as (start, count, items)."""
    start = (np.arange(ncell, dtype=np.int32) * K).astype(np.int32)
    count = np.full(ncell, K, dtype=np.int32)
    return start, count, np.ascontiguousarray(segments, dtype=np.int32)


def cells_round(spheres: np.ndarray, L, nseg, margin: float):
    """The fused walk's rounded near lists (nz_cells_count_round): the
    members by the box test with jump_tol = margin, keeping only cells whose
    box lies within r + margin + 1e-4 of the sphere's centre (Euclidean,
    float64).  (start, count, items), items ascending within a cell."""
    spheres = np.asarray(spheres, dtype=np.float64)
    Lx, Ly, Lz = (float(v) for v in L)
    nx, ny, nz = nseg
    st, ct, it = cells_members(spheres, L, nseg, margin)
    dL = (Lx / nx, Ly / ny, Lz / nz)
    keep = []
    for c in range(nx * ny * nz):
        n, m, p = c % nx, (c // nx) % ny, c // (nx * ny)
        s = it[st[c]:st[c] + ct[c]]
        lo = np.array([n * dL[0] - Lx / 2, m * dL[1] - Ly / 2, p * dL[2] - Lz / 2])
        hi = lo + np.array(dL)
        e = np.maximum(np.maximum(lo[:, None] - spheres[:3, s], 0.0), spheres[:3, s] - hi[:, None])
        R = spheres[3, s] + margin + 1e-4
        keep.append(s[(e * e).sum(axis=0) <= R * R])
    count = np.array([len(x) for x in keep], dtype=np.int32)
    start = np.zeros(nx * ny * nz, dtype=np.int32)
    start[1:] = np.cumsum(count)[:-1]
    return start, count, np.concatenate(keep).astype(np.int32)
