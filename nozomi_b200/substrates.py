"""Substrates: the reference's pickle format and the synthetic workloads.

Format (simulation_toolkit/utils/common_utils.py:17-25, written by
substrate_generator at cli/substrate_main.py:110): a pickle of
``[Tensor(N, 5) x, y, z, r, fiber_id, float L]``; fibres are split where a
sphere sits at z == L/2 (common_utils.py:41-55); z-periodic continuation pads
25 spheres at each end from the partner fibre shifted by -/+L
(utils/adjust_geometry.py:3-36).  The cubic box L is all the format holds; an
optional third element ``(Lx, Ly, Lz)`` extends it to non-cubic boxes (the
reference's loader ignores extra elements only if it unpacks two, so files with
the extension are written only on request).

Synthetic workloads (seeded, numpy.random.default_rng):
  * ``beaded_axon``: one axon of n spheres on the z axis at 1 um spacing, radii
    U[0.5, 1.5], z-periodic images by the reference's pad rule;
  * ``packed_axons``: n beaded axons in a periodic box, base radius lognormal,
    Gaussian bead bulges r(z) = r0 (1 + a exp(-(z - z_b)^2 / (2 * 1.5^2))) every
    ``bead_spacing`` um at a random phase, a ~ U[0.2, 0.5], centres packed
    without overlap between axons by pairwise relaxation, images across every
    face the axon comes within 2 um of.
"""
from __future__ import annotations

import pickle
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Substrate:
    """Spheres grouped into structures (axons) in a box centred on the origin."""
    fibers: list          # list of [n_i, 4] arrays (x, y, z, r); fibre k is structure k
    L: tuple              # (Lx, Ly, Lz)
    meta: dict = field(default_factory=dict)

    @property
    def nstructures(self) -> int:
        return len(self.fibers)

    def spheres(self) -> np.ndarray:
        """[5, S] float64: cx, cy, cz, r, structure id (geometry.py:58-64 layout)."""
        cols = []
        for k, f in enumerate(self.fibers):
            f = np.asarray(f, np.float64)
            cols.append(np.vstack([f[:, 0], f[:, 1], f[:, 2], f[:, 3], np.full(f.shape[0], float(k))]))
        if not cols:
            return np.zeros((5, 0))
        return np.concatenate(cols, axis=1)

    @property
    def S(self) -> int:
        return int(sum(np.asarray(f).shape[0] for f in self.fibers))

    def geometry(self, D=2.0, T2=100.0, rho=1.0, D_box=None):
        """The reference-style SimGeometry3D of this substrate."""
        from .geometry import SimGeometry3D, Structure3D
        g = SimGeometry3D(*self.L, D if D_box is None else D_box, T2, rho)
        for f in self.fibers:
            f = np.asarray(f, np.float64)
            g.add_structure(Structure3D(f[:, 0], f[:, 1], f[:, 2], f[:, 3], D, T2, rho))
        return g


# ---------------------------------------------------------------------------
# the reference's file format
# ---------------------------------------------------------------------------
def load_pickle(path):
    """(array [N,5], L) from a substrate pickle (common_utils.py:17-19);
    torch tensors are converted on the CPU."""
    with open(path, "rb") as f:
        data = pickle.load(f)
    arr, L = data[0], data[1]
    if hasattr(arr, "cpu"):
        arr = arr.cpu().numpy()
    box = tuple(float(v) for v in data[2]) if len(data) > 2 else (float(L),) * 3
    return np.asarray(arr, np.float64), float(L), box


def save_pickle(path, arr, L, box=None):
    """Write [array, L] (or [array, L, box] when box is given)."""
    import torch
    t = torch.as_tensor(np.asarray(arr, np.float64))
    payload = [t, L] if box is None else [t, L, tuple(box)]
    with open(path, "wb") as f:
        pickle.dump(payload, f, protocol=pickle.HIGHEST_PROTOCOL)


def split_fibers(arr: np.ndarray, box_length: float) -> list:
    """Fibres end at a sphere with z == L/2 exactly (common_utils.py:41-55)."""
    out, start = [], 0
    for i in range(len(arr)):
        if arr[i, 2] == box_length / 2:
            out.append(np.array(arr[start:i + 1]))
            start = i + 1
    return out


def pad_z(end_fiber: np.ndarray, start_fiber: np.ndarray, Lz: float, pad: int = 50) -> np.ndarray:
    """z-periodic continuation (adjust_geometry.py:22-36): the last pad/2
    spheres of the partner shifted by -Lz before, its first pad/2 shifted by +Lz
    after; the fibre-id column follows the fibre's own ids."""
    h = pad // 2
    s, w = np.asarray(start_fiber, np.float64), np.asarray(end_fiber, np.float64)
    cols = [np.concatenate((w[-h:, c], s[:, c], w[:h, c])) for c in range(2)]
    z = np.concatenate((w[-h:, 2] - Lz, s[:, 2], w[:h, 2] + Lz))
    r = np.concatenate((w[-h:, 3], s[:, 3], w[:h, 3]))
    fid = np.concatenate((s[-h:, 4], s[:, 4], s[:h, 4]))
    return np.stack([cols[0], cols[1], z, r, fid], axis=1)


def bound_z(fibers: list, Lz: float) -> list:
    """createBoundaryZ (adjust_geometry.py:3-20): a fibre whose first sphere's
    (x, y) is the last sphere's (x, y) of some fibre gets that partner's pad."""
    for f in fibers:
        f[:, -1] = f[:, -1].astype(int)
    by_end = {}
    for f in fibers:
        by_end[(f[-1][0], f[-1][1])] = f
    out = []
    for f in fibers:
        key = (f[0][0], f[0][1])
        out.append(pad_z(by_end[key], f, Lz) if key in by_end else f)
    return out


def ingest_on_device(matrix, L: float, Lz: float | None = None, pad: int = 50):
    """split_fibers + bound_z on the GPU (nz_ingest_split / plan / write):
    the matrix [M, 5] (x, y, z, r, fibre id; numpy or a torch tensor) is
    split at z == L/2 and its fibres z-padded from their partners.  Returns
    (rows [S, 5] float64 as bound_z returns them, concatenated; spheres
    [5, S] float64 with the fibre index as structure id; fibre lengths
    [F] int64 on the host), the arrays on the device.  Lz defaults to L."""
    import ctypes
    import torch
    from . import _lib as lib_
    from .engine import _p, _stream, require_cuda
    require_cuda()
    lib = lib_.load()
    dev = torch.device("cuda", torch.cuda.current_device())
    A = torch.as_tensor(matrix, dtype=torch.float64).to(dev).contiguous()
    if A.ndim != 2 or A.shape[1] != 5:
        raise lib_.NozomiError(f"substrate matrix must be [M, 5], got {tuple(A.shape)}")
    M = int(A.shape[0])
    Lz = float(L) if Lz is None else float(Lz)
    scratch = torch.empty(max(1, int(lib.nz_ingest_scratch_bytes(M))), dtype=torch.uint8, device=dev)
    ends = torch.empty(max(M, 1), dtype=torch.int32, device=dev)
    counts = torch.zeros(3, dtype=torch.int32, device=dev)  # fibres, output rows, short padded fibres
    c = ctypes.c_void_p
    lib_.check(lib.nz_ingest_split(_p(A), M, float(L), _p(ends), c(counts.data_ptr()), _p(scratch), scratch.numel(),
                                   _stream()), "nz_ingest_split")
    F = int(counts[0].item())
    partner = torch.empty(max(F, 1), dtype=torch.int32, device=dev)
    offset = torch.empty(max(F, 1), dtype=torch.int32, device=dev)
    lib_.check(lib.nz_ingest_plan(_p(A), _p(ends), F, int(pad), _p(partner), _p(offset), c(counts.data_ptr() + 4),
                                  c(counts.data_ptr() + 8), _p(scratch), scratch.numel(), _stream()), "nz_ingest_plan")
    h = counts.cpu().numpy()
    if h[2]:
        raise lib_.NozomiError(f"{int(h[2])} fibre(s) continue through the z face with fewer than {pad // 2} "
                               "spheres in them or in their partner")
    S = int(h[1])
    rows = torch.empty((S, 5), dtype=torch.float64, device=dev)
    spheres = torch.empty((5, S), dtype=torch.float64, device=dev)
    lib_.check(lib.nz_ingest_write(_p(A), _p(ends), F, _p(partner), _p(offset), S, Lz, int(pad), _p(rows),
                                   _p(spheres), _stream()), "nz_ingest_write")
    off = offset[:F].cpu().numpy().astype(np.int64)
    lengths = np.diff(np.append(off, S))
    return rows, spheres, lengths


def from_pickle_device(path) -> Substrate:
    """from_pickle with the split and the z padding done on the GPU."""
    arr, L, box = load_pickle(path)
    rows, _, lengths = ingest_on_device(arr, L, box[2])
    r = rows.cpu().numpy()
    fibers = [f[:, :4] for f in np.split(r, np.cumsum(lengths)[:-1])] if len(lengths) else []
    return Substrate(fibers, box, {"source": str(path), "ingested": "device"})


def from_pickle(path) -> Substrate:
    """The simulation driver's ingestion (simulation_main.py:37-54)."""
    arr, L, box = load_pickle(path)
    fibers = bound_z(split_fibers(arr, L), box[2])
    return Substrate([f[:, :4] for f in fibers], box, {"source": str(path)})


# ---------------------------------------------------------------------------
# synthetic workloads
# ---------------------------------------------------------------------------
def beaded_axon(n: int = 40, Lz: float = 40.0, Lxy: float = 8.0, seed: int = 1) -> Substrate:
    """One axon of n spheres on the z axis (z_i = -Lz/2 + 0.5 + i), radii
    U[0.5, 1.5], with the reference's +/-25-sphere z-periodic images."""
    rng = np.random.default_rng(seed)
    z = -Lz / 2 + 0.5 + np.arange(n, dtype=np.float64)
    r = rng.uniform(0.5, 1.5, n)
    fib = np.zeros((n, 5))
    fib[:, 2], fib[:, 3] = z, r
    padded = pad_z(fib, fib, Lz)
    return Substrate([padded[:, :4]], (Lxy, Lxy, Lz), {"kind": "beaded_axon", "n": n, "seed": seed})


def _bead_profile(r0, amp, phase, z, spacing, width=1.5):
    zc = (z[None, :] - phase[:, None]) % spacing
    d = np.minimum(zc, spacing - zc)
    return r0[:, None] * (1.0 + amp[:, None] * np.exp(-d ** 2 / (2 * width ** 2)))


def _required_distances(R: np.ndarray, dz: float) -> np.ndarray:
    """[n, n]: the smallest centre distance at which no sphere of axon i
    overlaps one of axon j, for axons on the same z grid of step dz with
    radius profiles R [n, k] (z-periodic profiles are compared cyclically)."""
    n, k = R.shape
    req = np.zeros((n, n))
    rmax = R.max()
    max_shift = min(k - 1, int(np.ceil(2 * rmax / dz)))
    for m in range(0, max_shift + 1):
        Rj = np.roll(R, -m, axis=1)
        for a, b in ((R, Rj), (Rj, R)) if m else ((R, R),):
            # (r_i[z] + r_j[z + m dz])^2 - (m dz)^2, maximised over z, in row blocks
            for i0 in range(0, n, 64):
                s2 = (a[i0:i0 + 64, None, :] + b[None, :, :]) ** 2 - (m * dz) ** 2
                req[i0:i0 + 64] = np.maximum(req[i0:i0 + 64], np.sqrt(np.maximum(s2.max(-1), 0.0)))
    return req


def _pack_centres(req: np.ndarray, box, rng, max_iter: int):
    """Centres in a periodic 2-D box, pairwise distances >= req, by relaxing
    overlaps from random positions (minimum-image)."""
    n = req.shape[0]
    Lx, Ly = box
    # start from a jittered grid in random order: few overlaps to relax
    nx = max(1, int(np.ceil(np.sqrt(n * Lx / Ly))))
    ny = max(1, int(np.ceil(n / nx)))
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * Lx / nx - Lx / 2, (np.arange(ny) + 0.5) * Ly / ny - Ly / 2)
    cells = rng.permutation(nx * ny)[:n]
    P = np.stack([gx.ravel()[cells], gy.ravel()[cells]], axis=1)
    P += rng.uniform(-0.25, 0.25, P.shape) * np.array([Lx / nx, Ly / ny])
    b = np.array([Lx, Ly])
    req = req.copy()
    np.fill_diagonal(req, 0.0)
    worst = np.inf
    for it in range(max_iter):
        d = P[:, None, :] - P[None, :, :]
        d -= b * np.round(d / b)
        dist = np.sqrt((d ** 2).sum(-1)) + np.eye(n)
        ov = np.maximum(0.0, req - dist)
        np.fill_diagonal(ov, 0.0)
        worst = ov.max()
        if worst < 1e-9:
            return P, it
        P += ((ov / dist)[:, :, None] * d * 0.5).sum(1)
        P = (P + b / 2) % b - b / 2
    raise RuntimeError(f"packing did not converge (largest overlap {worst:.3g} um)")


def _pack_centres_near(req: np.ndarray, box, rng, max_iter: int):
    """_pack_centres with the overlaps of each relaxation step taken only over
    pairs closer than the largest required distance (a periodic k-d tree's
    pair query), O(n log n) per step instead of O(n^2): the same start, the
    same update rule, rounding aside."""
    from scipy.spatial import cKDTree
    n = req.shape[0]
    Lx, Ly = box
    nx = max(1, int(np.ceil(np.sqrt(n * Lx / Ly))))
    ny = max(1, int(np.ceil(n / nx)))
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * Lx / nx - Lx / 2, (np.arange(ny) + 0.5) * Ly / ny - Ly / 2)
    cells = rng.permutation(nx * ny)[:n]
    P = np.stack([gx.ravel()[cells], gy.ravel()[cells]], axis=1)
    P += rng.uniform(-0.25, 0.25, P.shape) * np.array([Lx / nx, Ly / ny])
    b = np.array([Lx, Ly])
    rc = float(req.max())
    worst = np.inf
    for it in range(max_iter):
        Q = np.mod(P + b / 2, b)
        Q[Q >= b] = 0.0
        pairs = cKDTree(Q, boxsize=b).query_pairs(rc, output_type="ndarray")
        if pairs.size == 0:
            return P, it
        i, j = pairs[:, 0], pairs[:, 1]
        d = P[i] - P[j]
        d -= b * np.round(d / b)
        dist = np.sqrt((d ** 2).sum(-1))
        ov = np.maximum(0.0, req[i, j] - dist)
        worst = ov.max()
        if worst < 1e-9:
            return P, it
        f = (ov / dist)[:, None] * d * 0.5
        disp = np.zeros_like(P)
        np.add.at(disp, i, f)
        np.add.at(disp, j, -f)
        P = P + disp
        P = (P + b / 2) % b - b / 2
    raise RuntimeError(f"packing did not converge (largest overlap {worst:.3g} um)")


def _axons_with_images(P, R, z, L, image_margin):
    Lx, Ly, Lz = L
    dz = z[1] - z[0]
    fibers = []
    rmax = R.max(1)
    for i in range(P.shape[0]):
        base = np.stack([np.full(z.size, P[i, 0]), np.full(z.size, P[i, 1]), z, R[i]], axis=1)
        nimg = int(np.ceil((rmax[i] + image_margin) / dz)) + 1
        zimg = np.concatenate([base[-nimg:] - [0, 0, Lz, 0], base, base[:nimg] + [0, 0, Lz, 0]])
        parts = [zimg]
        reach = rmax[i] + image_margin
        sx = [0.0] + ([Lx] if P[i, 0] - reach < -Lx / 2 else []) + ([-Lx] if P[i, 0] + reach > Lx / 2 else [])
        sy = [0.0] + ([Ly] if P[i, 1] - reach < -Ly / 2 else []) + ([-Ly] if P[i, 1] + reach > Ly / 2 else [])
        for ox in sx:
            for oy in sy:
                if ox == 0.0 and oy == 0.0:
                    continue
                parts.append(zimg + [ox, oy, 0.0, 0.0])
        fibers.append(np.concatenate(parts))
    return fibers


def packed_axons(n_axons: int = 200, L=(40.0, 40.0, 80.0), spheres_per_axon: int = 100, r_mean: float = 1.0,
                 r_sd: float = 0.3, bead_amp=(0.2, 0.5), bead_spacing: float = 8.0, r_min: float = 0.45,
                 gap: float = 0.05, seed: int = 2, image_margin: float = 2.0, max_iter: int = 4000) -> Substrate:
    rng = np.random.default_rng(seed)
    Lx, Ly, Lz = (float(v) for v in L)
    dz = Lz / spheres_per_axon
    z = -Lz / 2 + dz / 2 + dz * np.arange(spheres_per_axon)
    sigma = np.sqrt(np.log(1 + (r_sd / r_mean) ** 2))
    mu = np.log(r_mean) - sigma ** 2 / 2
    r0 = np.maximum(rng.lognormal(mu, sigma, n_axons), r_min)
    amp = rng.uniform(bead_amp[0], bead_amp[1], n_axons)
    phase = rng.uniform(0, bead_spacing, n_axons)
    R = _bead_profile(r0, amp, phase, z, bead_spacing)               # [n, k]
    req = _required_distances(R, dz) + gap
    P, it = _pack_centres(req, (Lx, Ly), rng, max_iter)
    fibers = _axons_with_images(P, R, z, (Lx, Ly, Lz), image_margin)
    vf = float(np.mean([np.pi * (R[:, k] ** 2).sum() for k in range(z.size)]) / (Lx * Ly))
    return Substrate(fibers, (Lx, Ly, Lz), {"kind": "packed_axons", "n_axons": n_axons, "seed": seed,
                                             "centres": P, "r0": r0, "amp": amp, "bead_phase": phase,
                                             "volume_fraction": vf, "relax_iterations": it})


def axon_bundle(n_axons: int, seed: int, spheres_per_axon: int = 40, Lz: float = 40.0, r_range=(0.5, 1.5),
                area_fraction: float = 0.35, gap: float = 0.05, image_margin: float = 2.0) -> Substrate:
    """n beaded axons built like the single axon of ``beaded_axon`` (spheres at
    Lz / n spacing, radii uniform in r_range, z-periodic), packed without
    overlap in a square periodic box sized for the given mean cross-section
    area fraction."""
    rng = np.random.default_rng(seed)
    dz = Lz / spheres_per_axon
    z = -Lz / 2 + dz / 2 + dz * np.arange(spheres_per_axon)
    R = rng.uniform(r_range[0], r_range[1], (n_axons, spheres_per_axon))
    side = float(np.sqrt(np.pi * (R ** 2).mean(1).sum() / area_fraction))
    req = _required_distances(R, dz) + gap
    P, it = _pack_centres_near(req, (side, side), rng, 20000)
    fibers = _axons_with_images(P, R, z, (side, side, Lz), image_margin)
    return Substrate(fibers, (side, side, Lz), {"kind": "axon_bundle", "n_axons": n_axons, "seed": seed,
                                                 "relax_iterations": it})


def cell_grid(L, cell: float):
    """Cells per axis for a target cell edge (at least 1)."""
    return tuple(max(1, int(round(float(a) / cell))) for a in L)
