"""Device-side objects over the C ABI: substrates with their cell lists, walker
state, and the walk / seeding / reduction calls.

PyTorch provides device memory and the current stream; every computation is a
kernel of libnozomi_b200.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from ._lib import NozomiError


def require_cuda():
    if not torch.cuda.is_available():
        raise NozomiError("nozomi_b200 needs a CUDA device (sm_100a); there is no CPU path")
    L.load()


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def validate_substrate(sph64: np.ndarray, nstructures: int, L3, nseg, D, T2):
    """Host-side checks of a substrate before any device work (the reference
    checks none of these): finite centres, finite positive radii, structure
    ids that are integers in [0, nstructures), a positive box, at least one
    cell per axis, finite D >= 0 and T2 > 0 for every structure and the box.
    Raises NozomiError naming the first problem."""
    sph64 = np.asarray(sph64, dtype=np.float64)
    if sph64.ndim != 2 or sph64.shape[0] != 5:
        raise NozomiError(f"spheres must be [5, S] (cx, cy, cz, r, structure id), got {sph64.shape}")
    if sph64.size:
        bad = ~np.isfinite(sph64[:4]).all(axis=0)
        if bad.any():
            raise NozomiError(f"sphere {int(np.argmax(bad))} has a non-finite centre or radius")
        if (sph64[3] <= 0).any():
            raise NozomiError(f"sphere {int(np.argmax(sph64[3] <= 0))} has radius <= 0")
        sid = sph64[4]
        okid = np.isfinite(sid) & (sid == np.round(sid)) & (sid >= 0) & (sid < nstructures)
        if not okid.all():
            raise NozomiError(f"sphere {int(np.argmax(~okid))} has structure id {sid[np.argmax(~okid)]!r} "
                              f"outside [0, {nstructures})")
    Lv = np.asarray(L3, dtype=np.float64)
    if Lv.shape != (3,) or not (np.isfinite(Lv).all() and (Lv > 0).all()):
        raise NozomiError(f"box {tuple(L3)} must be three finite positive lengths")
    if len(tuple(nseg)) != 3 or min(int(v) for v in nseg) < 1:
        raise NozomiError(f"cell grid {tuple(nseg)} needs at least one cell per axis")
    Dv, Tv = np.asarray(D, np.float64).ravel(), np.asarray(T2, np.float64).ravel()
    if Dv.size != nstructures + 1 or Tv.size != nstructures + 1:
        raise NozomiError("D and T2 need one entry per structure plus the box")
    if not (np.isfinite(Dv).all() and (Dv >= 0).all()):
        raise NozomiError("D must be finite and >= 0")
    if not (np.isfinite(Tv).all() and (Tv > 0).all()):
        raise NozomiError("T2 must be finite and > 0")


def box_grid(L3, nseg) -> L.Grid:
    """The reference's float constants Lx.. and dLx = Lx / nseg (diffsim3d.py:115-120)."""
    Lx, Ly, Lz = (float(v) for v in L3)
    nx, ny, nz = (int(v) for v in nseg)
    return L.Grid(np.float32(Lx), np.float32(Ly), np.float32(Lz), np.float32(Lx / nx), np.float32(Ly / ny),
                  np.float32(Lz / nz), nx, ny, nz)


def record_order(sph64: np.ndarray, nstructures: int):
    """The index form's records of spheres [5, S]: the spheres sorted by
    structure id (stable); returns rec4 [max(S, 1), 4] float32 (x, y, z, r),
    rec_sid [max(S, 1)] int32, sid_start [nstructures + 2] int32 (the first
    record of each structure, S at the end) and perm [max(S, 1)] int32 (each
    sphere's record).  Arrays keep one row at least, so that an empty
    substrate still has device pointers."""
    S = sph64.shape[1]
    sid = sph64[4].astype(np.int64)
    order = np.argsort(sid, kind="stable")
    perm = np.zeros(max(S, 1), np.int32)
    perm[order] = np.arange(S, dtype=np.int32)
    rec_sid = np.zeros(max(S, 1), np.int32)
    rec_sid[:S] = sid[order]
    rec4 = np.zeros((max(S, 1), 4), np.float32)
    rec4[:S] = sph64[:4, order].T
    sid_start = np.searchsorted(rec_sid[:S], np.arange(nstructures + 2)).astype(np.int32)
    return rec4, rec_sid, sid_start, perm


class DeviceSubstrate:
    """Spheres [5,S] (cx, cy, cz, r, structure id), box, cell grid, compact cell
    lists built on the GPU (DiffSim3d.set_segments, diffsim3d.py:107-174), the
    fused walk's form of those lists, and D / T2 per structure.

    idx_bytes selects the fused walk's list form: 0, per-entry records (each
    entry carries its sphere's centre, radius and structure id); 2 or 4, index
    lists (each entry a 16- or 32-bit index into one record array of the
    substrate, the spheres sorted by structure id); None, index lists of 16
    bits when S <= 65536, else 32.  near_round: near lists by the Euclidean
    sphere-to-cell test (the default) or the reference's box test."""

    def __init__(self, spheres: np.ndarray, nstructures: int, L3, nseg, D, T2, jump_tol: float = 1.0,
                 cells: tuple | None = None, near_margin: float | None = None, idx_bytes: int | None = None,
                 near_round: bool = True):
        sph64 = np.ascontiguousarray(spheres, dtype=np.float64).reshape(5, -1)
        validate_substrate(sph64, int(nstructures), L3, nseg, D, T2)
        require_cuda()
        dev = _dev()
        self.S = sph64.shape[1]
        if idx_bytes is None:
            idx_bytes = 2 if self.S <= 65536 else 4
        if idx_bytes not in (0, 2, 4) or (idx_bytes == 2 and self.S > 65536):
            raise NozomiError(f"list form idx_bytes={idx_bytes} does not suit {self.S} spheres (0, 2 up to 65536, 4)")
        self.idx_bytes = int(idx_bytes)
        self.near_round = bool(near_round)
        self.nstructures = int(nstructures)
        self.L = tuple(float(v) for v in L3)
        self.nseg = tuple(int(v) for v in nseg)
        self.ncell = self.nseg[0] * self.nseg[1] * self.nseg[2]
        self.jump_tol = float(jump_tol)
        self.grid = box_grid(self.L, self.nseg)
        self.spheres64 = torch.from_numpy(sph64).to(dev)
        self.spheres = torch.from_numpy(sph64.astype(np.float32)).to(dev)
        self.D = torch.as_tensor(np.asarray(D, np.float32), device=dev)
        self.T2 = torch.as_tensor(np.asarray(T2, np.float32), device=dev)
        if cells is None:
            self._build_cells()
        else:
            st, ct, it = cells
            self.cell_start = torch.as_tensor(np.asarray(st, np.int32), device=dev)
            self.cell_count = torch.as_tensor(np.asarray(ct, np.int32), device=dev)
            self.cell_items = torch.as_tensor(np.asarray(it, np.int32), device=dev)
            self.n_items = int(self.cell_items.numel())
        if self.idx_bytes:
            self._records(sph64)
        self._gather()
        self.near_margin = None
        self.near = None
        if near_margin is not None:
            self.set_near_margin(near_margin)

    def _records(self, sph64: np.ndarray):
        """The index form's record array on the device (record_order)."""
        dev = _dev()
        rec4, rec_sid, sid_start, perm = record_order(sph64, self.nstructures)
        self.rec4 = torch.from_numpy(rec4).to(dev)
        self.rec_sid = torch.from_numpy(rec_sid).to(dev)
        self.sid_start = torch.from_numpy(sid_start).to(dev)
        self.perm = torch.from_numpy(perm).to(dev)

    def _index(self, start, count, items, n):
        """Index-form entries of member lists (start, count, items)."""
        dt = torch.int16 if self.idx_bytes == 2 else torch.int32
        idx = torch.empty(max(n, 1), dtype=dt, device=_dev())
        L.check(L.load().nz_cells_index(_p(items), n, _p(self.perm), self.S, _p(start), _p(count), self.ncell, _p(idx),
                                        self.idx_bytes, _stream()), "nz_cells_index")
        return idx

    def _build_cells(self, margin: float | None = None, store: bool = True, rounded: bool = False):
        """Member lists with the reference's box test (margin: jump_tol by
        default); rounded: the near lists' Euclidean test (nz_cells_*_round)."""
        dev = _dev()
        lib = L.load()
        Lx, Ly, Lz = self.L
        nx, ny, nz = self.nseg
        tol = self.jump_tol if margin is None else float(margin)
        count_fn = lib.nz_cells_count_round if rounded else lib.nz_cells_count
        fill_fn = lib.nz_cells_fill_round if rounded else lib.nz_cells_fill
        counts = torch.empty(self.ncell, dtype=torch.int32, device=dev)
        L.check(count_fn(_p(self.spheres64), self.S, Lx, Ly, Lz, nx, ny, nz, tol, _p(counts), _stream()),
                "nz_cells_count")
        offsets = torch.empty(self.ncell, dtype=torch.int32, device=dev)
        total = torch.zeros(1, dtype=torch.int32, device=dev)
        L.check(lib.nz_exclusive_scan_i32(_p(counts), _p(offsets), self.ncell, _p(total), _stream()),
                "nz_exclusive_scan_i32")
        n_items = int(total.item())  # one host sync: the list length sizes the item array
        items = torch.empty(max(n_items, 1), dtype=torch.int32, device=dev)
        cursor = torch.empty(self.ncell, dtype=torch.int32, device=dev)
        L.check(fill_fn(_p(self.spheres64), self.S, Lx, Ly, Lz, nx, ny, nz, tol, _p(offsets), _p(counts), _p(cursor),
                        _p(items), _stream()), "nz_cells_fill")
        if not store:
            return offsets, counts, items, n_items
        self.cell_start, self.cell_count, self.cell_items = offsets, counts, items
        self.n_items = n_items

    def set_near_margin(self, margin: float | None):
        """Build (or drop, with None) the near lists of the fused walk: the
        same grid with a smaller membership margin (0 < margin < jump_tol),
        by the Euclidean test when near_round (nz_cells_count_round), else by
        the reference's box test."""
        if margin is None:
            self.near_margin, self.near = None, None
            return
        margin = float(margin)
        if not 0.0 < margin < self.jump_tol:
            raise NozomiError(f"near margin {margin} must lie in (0, {self.jump_tol})")
        st, ct, it, n = self._build_cells(margin, store=False, rounded=self.near_round)
        dev = _dev()
        self.near_n = n
        if self.idx_bytes:
            self.near_margin = margin
            self.near = (st, ct, it, None, None, self._index(st, ct, it, n))
            return
        sph4 = torch.empty((max(n, 1), 4), dtype=torch.float32, device=dev)
        sid = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        L.check(L.load().nz_cells_gather(_p(self.spheres), self.S, _p(it), n, _p(st), _p(ct), self.ncell, _p(sph4),
                                         _p(sid), _stream()), "nz_cells_gather")
        self.near_margin = margin
        self.near = (st, ct, it, sph4, sid, None)

    def _gather(self):
        """The fused walk's form of the member lists: index entries, or
        per-entry records."""
        dev = _dev()
        n = int(self.n_items)
        if self.idx_bytes:
            self.cell_sph4 = self.cell_sid = None
            self.cell_idx = self._index(self.cell_start, self.cell_count, self.cell_items, n)
            return
        self.cell_idx = None
        self.cell_sph4 = torch.empty((max(n, 1), 4), dtype=torch.float32, device=dev)
        self.cell_sid = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        L.check(L.load().nz_cells_gather(_p(self.spheres), self.S, _p(self.cell_items), n, _p(self.cell_start),
                                         _p(self.cell_count), self.ncell, _p(self.cell_sph4), _p(self.cell_sid),
                                         _stream()), "nz_cells_gather")

    def max_count(self) -> int:
        return int(self.cell_count.max().item()) if self.ncell else 0

    def padded_segments(self, K: int | None = None) -> tuple[int, torch.Tensor]:
        """The reference's padded table (K, segments[ncell*K])."""
        K = self.max_count() if K is None else int(K)
        seg = torch.empty(self.ncell * K, dtype=torch.int32, device=_dev())
        Lx, Ly, Lz = self.L
        nx, ny, nz = self.nseg
        L.check(L.load().nz_segments_fill(_p(self.spheres64), self.S, Lx, Ly, Lz, nx, ny, nz, K, _p(seg), _stream()),
                "nz_segments_fill")
        return K, seg

    def with_padded_lists(self) -> "DeviceSubstrate":
        """A view whose cell lists are the reference's padded table."""
        K, seg = self.padded_segments()
        other = object.__new__(DeviceSubstrate)
        other.__dict__.update(self.__dict__)
        dev = _dev()
        other.cell_start = torch.arange(self.ncell, dtype=torch.int32, device=dev) * K
        other.cell_count = torch.full((self.ncell,), K, dtype=torch.int32, device=dev)
        other.cell_items = seg
        other.n_items = int(seg.numel())
        other._gather()  # in the index form the record array (and perm) is shared
        other.K = K
        other.near_margin, other.near = None, None
        return other

    def struct(self) -> L.Substrate:
        ptr = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        s = L.Substrate(self.grid, self.nstructures, self.S, self.spheres.data_ptr(), self.cell_start.data_ptr(),
                        self.cell_count.data_ptr(), self.cell_items.data_ptr(), ptr(self.cell_sph4),
                        ptr(self.cell_sid), self.D.data_ptr(), self.T2.data_ptr())
        s.n_items = int(self.n_items)
        if self.near is not None:
            st, ct, _, sph4, sid, nidx = self.near
            s.near_margin = self.near_margin
            s.near_start, s.near_count = st.data_ptr(), ct.data_ptr()
            s.near_sph4, s.near_sid, s.near_idx = ptr(sph4), ptr(sid), ptr(nidx)
            s.near_items = int(self.near_n)
        if self.idx_bytes:
            s.idx_bytes, s.cell_idx = self.idx_bytes, self.cell_idx.data_ptr()
            s.rec4, s.rec_sid, s.sid_start = self.rec4.data_ptr(), self.rec_sid.data_ptr(), self.sid_start.data_ptr()
        return s

    def nbytes(self) -> int:
        ts = [self.spheres64, self.spheres, self.D, self.T2, self.cell_start, self.cell_count, self.cell_items,
              self.cell_sph4, self.cell_sid, self.cell_idx] + (list(self.near) if self.near is not None else [])
        if self.idx_bytes:
            ts += [self.rec4, self.rec_sid, self.sid_start, self.perm]
        return sum(t.numel() * t.element_size() for t in ts if t is not None)


def philox_draws(key: int, stream_id: int = 0) -> L.Draws:
    key = int(key) & 0xFFFFFFFFFFFFFFFF
    return L.Draws(None, 0, 0, key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF, stream_id & 0xFFFFFFFF)


def injected_draws(table: torch.Tensor) -> L.Draws:
    """table: [N, nsteps, maxk] float32 on the device."""
    return L.Draws(table.data_ptr(), int(table.shape[1]), int(table.shape[2]), 0, 0, 0)


def seed(sub: DeviceSubstrate, targets, N: int, key: int, max_rounds: int = 100000, stream_id: int = 1,
         id0: int = 0):
    """Seed walkers [id0, id0 + N) uniformly into the target structures (the
    box is structure sub.nstructures).  Returns (spins [3,N] float32, label [N])."""
    dev = _dev()
    tgt = np.zeros(sub.nstructures + 1, np.uint8)
    tgt[np.asarray(list(targets), np.int64)] = 1
    tgt_d = torch.from_numpy(tgt).to(dev)
    spins = torch.empty((3, N), dtype=torch.float32, device=dev)
    label = torch.empty(N, dtype=torch.int32, device=dev)
    left = torch.zeros(1, dtype=torch.int32, device=dev)
    s = sub.struct()
    key = int(key) & 0xFFFFFFFFFFFFFFFF
    L.check(L.load().nz_seed_range(L.byref(s), _p(tgt_d), int(id0), N, key & 0xFFFFFFFF, key >> 32, stream_id,
                                   max_rounds, _p(spins), _p(label), _p(left), _stream()), "nz_seed_range")
    n_left = int(left.item())
    if n_left:
        raise NozomiError(f"seeding left {n_left} of {N} walkers unplaced after {max_rounds} rounds "
                          f"(target structures {sorted(set(int(t) for t in targets))} may have no volume)")
    return spins, label


@dataclass
class Walkers:
    """Walker arrays in the reference's layout (diffsim3d.py:42-45, :62)."""
    spins: torch.Tensor               # [3, N]
    spins0: torch.Tensor              # [3, N]
    phase: torch.Tensor | None = None     # [ndir, N]
    diffdir: torch.Tensor | None = None   # [3, ndir]
    sig: torch.Tensor | None = None       # [N]
    phi: torch.Tensor | None = None       # [6, N]
    label: torch.Tensor | None = None
    n_iter: torch.Tensor | None = None
    n_scatter: torch.Tensor | None = None
    flags: torch.Tensor | None = None

    @property
    def N(self) -> int:
        return int(self.spins.shape[1])

    def struct(self) -> L.Walkers:
        nd = 0 if self.diffdir is None else int(self.diffdir.shape[1])
        v = lambda t: None if t is None else t.data_ptr()  # noqa: E731
        return L.Walkers(self.N, v(self.spins), v(self.spins0), v(self.phase), v(self.diffdir), nd, v(self.sig),
                         v(self.phi), v(self.label), v(self.n_iter), v(self.n_scatter), v(self.flags))

    @staticmethod
    def with_counters(spins, spins0, **kw) -> "Walkers":
        N = spins.shape[1]
        dev = spins.device
        z = lambda: torch.zeros(N, dtype=torch.int32, device=dev)  # noqa: E731
        return Walkers(spins, spins0, label=z(), n_iter=z(), n_scatter=z(), flags=z(), **kw)


def walk_step(sub: DeviceSubstrate, wk: Walkers, mode: int, dt: float, G: float, Garea: float, step: int,
              draws: L.Draws):
    s = sub.struct()
    w = wk.struct()
    L.check(L.load().nz_walk_step(L.byref(s), L.byref(w), mode, np.float32(dt), np.float32(G), np.float32(Garea),
                                  int(step), L.byref(draws), _stream()), "nz_walk_step")


class FusedState:
    """Packed walkers of the fused walk: four float4 per walker."""

    def __init__(self, N: int):
        dev = _dev()
        self.N = N
        self.pos = torch.empty((N, 4), dtype=torch.float32, device=dev)
        self.org = torch.empty((N, 4), dtype=torch.float32, device=dev)
        self.phi = torch.empty((N, 4), dtype=torch.float32, device=dev)
        self.comp = torch.empty((N, 4), dtype=torch.float32, device=dev)

    def struct(self) -> L.State:
        return L.State(self.N, self.pos.data_ptr(), self.org.data_ptr(), self.phi.data_ptr(), self.comp.data_ptr())

    def nbytes(self) -> int:
        return 4 * 16 * self.N

    @staticmethod
    def from_walkers(wk: Walkers, ids: torch.Tensor | None = None) -> "FusedState":
        st = FusedState(wk.N)
        st.pack(wk, ids)
        return st

    def pack(self, wk: Walkers, ids: torch.Tensor | None = None):
        """Pack walkers (reference layout) into this state; walker ids are
        ids[w], or w."""
        s = self.struct()
        w = wk.struct()
        L.check(L.load().nz_state_pack(L.byref(w), _p(ids), L.byref(s), _stream()), "nz_state_pack")

    def to_walkers(self, wk: Walkers):
        s = self.struct()
        w = wk.struct()
        L.check(L.load().nz_state_unpack(L.byref(s), L.byref(w), _stream()), "nz_state_unpack")

    def to_walkers_by_id(self, wk: Walkers):
        """Unpack into walker-id order (undoes re-binning)."""
        s = self.struct()
        w = wk.struct()
        bad = torch.zeros(1, dtype=torch.int32, device=_dev())
        L.check(L.load().nz_state_unpack_by_id(L.byref(s), L.byref(w), _p(bad), _stream()), "nz_state_unpack_by_id")
        return bad

    def walker_ids(self) -> torch.Tensor:
        return self.org[:, 3].contiguous().view(torch.int32)

    @staticmethod
    def sort_bins(grid: L.Grid, coarsen: int, nlabels: int = 0) -> int:
        """Keys of a re-binning: coarsened cells, times labels when nlabels > 0."""
        return (-(-grid.nx // coarsen)) * (-(-grid.ny // coarsen)) * (-(-grid.nz // coarsen)) * max(nlabels, 1)

    def sort_kernels(self, grid: L.Grid, coarsen: int, nlabels: int = 0) -> int:
        """Library kernels one sort_into launches: bin count, the histogram
        scan (one kernel, or three above SCAN_SINGLE_KEYS bins), scatter."""
        if self.N == 0:
            return 0
        return 2 + (1 if self.sort_bins(grid, coarsen, nlabels) <= L.SCAN_SINGLE_KEYS else 3)

    def sort_into(self, other: "FusedState", grid: L.Grid, coarsen: int, scratch: torch.Tensor | None = None,
                  nlabels: int = 0):
        """Re-bin into `other` by cell (coarsened), or by (label, cell) when
        nlabels > 0.  Returns the scratch buffer for reuse."""
        nb = self.sort_bins(grid, coarsen, nlabels)
        need = int(L.load().nz_sort_scratch_bytes(self.N, nb))
        if scratch is None or scratch.numel() < need:
            scratch = torch.empty(need, dtype=torch.uint8, device=_dev())
        a, b = self.struct(), other.struct()
        L.check(L.load().nz_state_sort_keyed(L.byref(a), L.byref(grid), coarsen, int(nlabels), L.byref(b), _p(scratch),
                                             scratch.numel(), _stream()), "nz_state_sort_keyed")
        return scratch

    def signal(self, dirs: torch.Tensor, amps: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Sum over walkers of exp(i amp_b u_d . Phi): [2, ndir, nb] float64."""
        ndir, nb = int(dirs.shape[1]), int(amps.numel())
        if out is None:
            out = torch.zeros((2, ndir, nb), dtype=torch.float64, device=_dev())
        s = self.struct()
        L.check(L.load().nz_signal_phi(L.byref(s), _p(dirs), ndir, _p(amps), nb, _p(out), _stream()), "nz_signal_phi")
        return out

    def phase(self, dirs: torch.Tensor) -> torch.Tensor:
        ndir = int(dirs.shape[1])
        out = torch.empty((ndir, self.N), dtype=torch.float32, device=_dev())
        s = self.struct()
        L.check(L.load().nz_phase_from_phi(L.byref(s), _p(dirs), ndir, _p(out), _stream()), "nz_phase_from_phi")
        return out


def _check_tables(who: str, step1: int, mode: int, G=None, Garea=None, moments=None):
    """The kernels index the protocol tables and the moment rows by global
    step; the C ABI cannot see their lengths, so they are checked here."""
    if mode & L.MODE_PHI:
        for name, t in (("G", G), ("Garea", Garea)):
            if t is None or t.dtype != torch.float32 or t.numel() < step1:
                raise NozomiError(f"{who}: {name} must be float32 with at least {step1} entries (steps to {step1})")
    if moments is not None and (moments.dtype != torch.float64 or moments.numel() < 6 * step1):
        raise NozomiError(f"{who}: moments must be float64 with at least {step1} rows of 6")


def walk_fused(sub: DeviceSubstrate, st: FusedState, mode: int, dt: float, G: torch.Tensor | None,
               Garea: torch.Tensor | None, step0: int, step1: int, draws: L.Draws,
               moments: torch.Tensor | None = None):
    _check_tables("walk_fused", int(step1), mode, G, Garea, moments if mode & L.MODE_MOMENTS else None)
    s = sub.struct()
    a = st.struct()
    L.check(L.load().nz_walk_fused(L.byref(s), L.byref(a), mode, np.float32(dt), _p(G), _p(Garea), int(step0),
                                   int(step1), L.byref(draws), _p(moments), _stream()), "nz_walk_fused")


def walk_fused_moments(sub: DeviceSubstrate, st: FusedState, mode: int, dt: float, step0: int, step1: int,
                       draws: L.Draws, moments: torch.Tensor, scratch: torch.Tensor | None = None) -> torch.Tensor:
    """Steps [step0, step1) with the per-step displacement moments added to
    moments[step0:step1] ([nsteps, 6] float64).  Returns the scratch buffer
    (float32, grown as needed) for reuse."""
    _check_tables("walk_fused_moments", int(step1), 0, moments=moments)
    lib = L.load()
    need = int(lib.nz_walk_fused_moments_scratch_bytes(st.N, int(step1) - int(step0)))
    if scratch is None or scratch.numel() * 4 < need:
        scratch = torch.empty(max(need // 4, 1), dtype=torch.float32, device=_dev())
    s = sub.struct()
    a = st.struct()
    L.check(lib.nz_walk_fused_moments(L.byref(s), L.byref(a), mode, np.float32(dt), None, None, int(step0),
                                      int(step1), L.byref(draws), _p(scratch), scratch.numel() * 4, _p(moments),
                                      _stream()), "nz_walk_fused_moments")
    return scratch


def moments(spins: torch.Tensor, spins0: torch.Tensor, out: torch.Tensor):
    L.check(L.load().nz_moments(_p(spins), _p(spins0), int(spins.shape[1]), _p(out), _stream()), "nz_moments")
