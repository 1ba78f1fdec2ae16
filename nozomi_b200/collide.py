"""Collision detection of the substrate generator on the GPU.

``detect_collision(positions, radii, fiber_id, Lx, Ly, Lz, buff)`` has the
reference's signature and result (substrate_generator/helper/
CollisionDetection.py:7-8, collide_spheres_gpu :10-50): the (M, 2) int64
indices (a < b) of every pair of spheres of different fibres with
(r_a + r_b + buff) - |x_a - x_b| > 0, in lexicographic order.  The reference
tests the pairs of each block of a grid of edge Lx/10 with a dense matrix
per block; here the blocks are cell lists built on the device
(nz_collide_cells), every pair of a block's members is tested once and
emitted by the first block the two spheres share (nz_collide_pairs), and the
rows are put in order on the device (nz_pairs_sort).  Spheres that belong to
no block (more than 1 um outside the grid) take part in no pair; the
reference may still test some of them as padding entries of a block,
depending on its sort's tie order.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L
from .engine import require_cuda


def block_grid(Lx, Ly, Lz) -> L.Grid:
    """The reference's grid in float32: blocks of edge Lx/10, ceil(L/block)
    blocks per axis, block edges L/n (:26-27, :69-71)."""
    Lf = np.array([Lx, Ly, Lz], np.float32)
    block = np.float32(Lf[0] / np.float32(10))
    n = np.ceil(Lf / block).astype(np.int64)
    d = (Lf / n.astype(np.float32)).astype(np.float32)
    return L.Grid(float(Lf[0]), float(Lf[1]), float(Lf[2]), float(d[0]), float(d[1]), float(d[2]),
                  int(n[0]), int(n[1]), int(n[2]))


def detect_collision(positions, radii, fiber_id, Lx, Ly, Lz, buff=0.0, sort: bool = True) -> torch.Tensor:
    """(M, 2) int64 indices of colliding sphere pairs of different fibres
    (see the module docstring); positions [S, 3], radii and fiber_id [S],
    any device or host arrays, computed in float32 on the current GPU."""
    require_cuda()
    lib = L.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    f32 = lambda a: torch.as_tensor(a, dtype=torch.float32).to(dev).contiguous()  # noqa: E731
    pos, r, fid = f32(positions).reshape(-1, 3), f32(radii).reshape(-1), f32(fiber_id).reshape(-1)
    S = int(pos.shape[0])
    if r.numel() != S or fid.numel() != S:
        raise L.NozomiError("positions, radii and fiber_id need one row per sphere")
    if S and not (torch.isfinite(pos).all() and torch.isfinite(r).all()):
        raise L.NozomiError("sphere positions and radii must be finite")
    g = block_grid(float(Lx), float(Ly), float(Lz))
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    scratch = torch.empty(max(1, int(lib.nz_collide_scratch_bytes(S, ctypes.byref(g)))), dtype=torch.uint8,
                          device=dev)
    counts = torch.zeros(2, dtype=torch.int32, device=dev)
    L.check(lib.nz_collide_cells(p(pos), p(r), S, ctypes.byref(g), p(counts), p(scratch), scratch.numel(), stream),
            "nz_collide_cells")
    members = int(counts[0].item())
    items = torch.empty(max(members, 1), dtype=torch.int32, device=dev)
    cap = max(1024, 4 * S)
    for _ in range(2):  # a second pass only when the first buffer was too small
        pairs = torch.empty((cap, 2), dtype=torch.int32, device=dev)
        L.check(lib.nz_collide_pairs(p(pos), p(r), p(fid), S, ctypes.byref(g), float(np.float32(buff)), p(items),
                                     members, p(pairs), cap, ctypes.c_void_p(counts.data_ptr() + 4), p(scratch),
                                     scratch.numel(), stream), "nz_collide_pairs")
        n = int(counts[1].item())
        if n <= cap:
            break
        cap = n
    pairs = pairs[:n]
    if sort and n:
        out = torch.empty_like(pairs)
        ss = torch.empty(max(1, int(lib.nz_pairs_sort_scratch_bytes(S))), dtype=torch.uint8, device=dev)
        L.check(lib.nz_pairs_sort(p(pairs), n, S, p(out), p(ss), ss.numel(), stream), "nz_pairs_sort")
        pairs = out
    return pairs.to(torch.int64)
