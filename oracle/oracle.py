"""ctypes front end of the C oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs
import this module.  See walk_oracle.c for what each entry restates.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from oracle.build import build_oracle

MODE_SIG, MODE_PHASE, MODE_PHI, MODE_TANGENT64 = 1, 2, 4, 8
FLAG_DRAWS_EXHAUSTED, FLAG_ITER_CAP, FLAG_UNSEEDED = 1, 2, 4
RNG_INJECT, RNG_PHILOX = 0, 1

_P = ctypes.c_void_p


class _Geom(ctypes.Structure):
    _fields_ = [("S", ctypes.c_int), ("nstructures", ctypes.c_int),
                ("Lx", ctypes.c_float), ("Ly", ctypes.c_float), ("Lz", ctypes.c_float),
                ("dLx", ctypes.c_float), ("dLy", ctypes.c_float), ("dLz", ctypes.c_float),
                ("nLx", ctypes.c_float), ("nLy", ctypes.c_float), ("nLz", ctypes.c_float),
                ("spheres", _P), ("cell_start", _P), ("cell_count", _P), ("cell_items", _P),
                ("D", _P), ("T2", _P)]


class _Rng(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("normals", _P), ("nsteps", ctypes.c_int), ("maxk", ctypes.c_int),
                ("key0", ctypes.c_uint32), ("key1", ctypes.c_uint32), ("stream", ctypes.c_uint32),
                ("id0", ctypes.c_uint32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(build_oracle()))
        i, f, d, u = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_uint32
        _lib.oz_walk_f32.argtypes = [_P, _P, i, i, i, i, f, _P, _P, _P, _P, _P, _P, i, _P, _P, _P, _P, _P, _P, _P, i]
        _lib.oz_walk_f64.argtypes = [_P, _P, i, i, i, i, d, _P, _P, _P, _P, _P, _P, i, _P, _P, _P, _P, _P, _P, i]
        _lib.oz_seed.argtypes = [_P, _P, i, u, u, u, i, _P, _P, i]
        _lib.oz_seed_range.argtypes = [_P, _P, u, i, u, u, u, i, _P, _P, i]
        _lib.oz_segments.argtypes = [_P, i, d, d, d, i, i, i, i, _P, i]
        _lib.oz_segments.restype = ctypes.c_int
        _lib.oz_seed_accept.argtypes = [_P, _P, i, _P, _P]
        _lib.oz_philox_normals.argtypes = [u, u, u, i, i, i, _P]
        _lib.oz_philox_block.argtypes = [_P, u, u]
        _lib.oz_box_muller_pairs.argtypes = [_P, _P, i, _P]
        _lib.oz_moments.argtypes = [i, _P, _P, _P]
        _lib.oz_signal_phi.argtypes = [i, _P, _P, i, _P, i, _P, _P]
        _lib.oz_signal_phase.argtypes = [i, _P, i, _P, i, _P, _P]
        _lib.oz_cells.argtypes = [_P, i, d, d, d, i, i, i, d, _P, _P, _P]
        _lib.oz_cells.restype = ctypes.c_longlong
        _lib.oz_set_phase64.argtypes = [_P]
        _lib.oz_set_phase64.restype = None
        for fn in ("oz_walk_f32", "oz_walk_f64", "oz_seed", "oz_seed_range"):
            getattr(_lib, fn).restype = ctypes.c_int
        for fn in ("oz_seed_accept", "oz_philox_normals", "oz_philox_block", "oz_box_muller_pairs", "oz_moments",
                   "oz_signal_phi", "oz_signal_phase"):
            getattr(_lib, fn).restype = None
    return _lib


def cells(spheres64, L, nseg, jump_tol: float = 1.0):
    """Member cell lists (start, count, items) built on the host in C."""
    sph = np.ascontiguousarray(spheres64, np.float64)
    nx, ny, nz = (int(v) for v in nseg)
    ncell = nx * ny * nz
    count = np.zeros(ncell, np.int32)
    start = np.zeros(ncell, np.int32)
    Lx, Ly, Lz = (float(v) for v in L)
    total = lib().oz_cells(sph.ctypes.data, sph.shape[1], Lx, Ly, Lz, nx, ny, nz, jump_tol, count.ctypes.data,
                           start.ctypes.data, None)
    items = np.zeros(max(int(total), 1), np.int32)
    lib().oz_cells(sph.ctypes.data, sph.shape[1], Lx, Ly, Lz, nx, ny, nz, jump_tol, count.ctypes.data,
                   start.ctypes.data, items.ctypes.data)
    return start, count, items[:int(total)]


def segments(spheres64, L, nseg, K: int, nthreads: int = 0):
    """The reference's padded table [ncell*K] (oz_segments)."""
    sph = np.ascontiguousarray(spheres64, np.float64)
    nx, ny, nz = (int(v) for v in nseg)
    seg = np.zeros(nx * ny * nz * int(K), np.int32)
    rc = lib().oz_segments(sph.ctypes.data, sph.shape[1], *(float(v) for v in L), nx, ny, nz, int(K),
                           seg.ctypes.data, nthreads)
    if rc:
        raise RuntimeError(f"oz_segments failed ({rc})")
    return seg


def _ptr(a):
    return None if a is None else a.ctypes.data


@dataclass
class Geometry:
    """Spheres [5,S] float32 (cx, cy, cz, r, structure id), box, cell grid and
    cell lists (start, count, items)."""
    spheres: np.ndarray
    nstructures: int
    L: tuple
    nseg: tuple
    start: np.ndarray
    count: np.ndarray
    items: np.ndarray
    D: np.ndarray
    T2: np.ndarray
    dL: tuple = None
    _keep: list = field(default_factory=list)

    def struct(self) -> _Geom:
        sph = np.ascontiguousarray(self.spheres, dtype=np.float32)
        st = np.ascontiguousarray(self.start, dtype=np.int32)
        ct = np.ascontiguousarray(self.count, dtype=np.int32)
        it = np.ascontiguousarray(self.items, dtype=np.int32)
        if it.size == 0:
            it = np.zeros(1, np.int32)
        D = np.ascontiguousarray(self.D, dtype=np.float32)
        T2 = np.ascontiguousarray(self.T2, dtype=np.float32)
        self._keep = [sph, st, ct, it, D, T2]
        Lx, Ly, Lz = (np.float32(v) for v in self.L)
        nx, ny, nz = self.nseg
        if self.dL is not None:
            dLx, dLy, dLz = (np.float32(v) for v in self.dL)
        else:
            dLx, dLy, dLz = (np.float32(float(a) / n) for a, n in zip(self.L, self.nseg))
        return _Geom(sph.shape[1], self.nstructures, Lx, Ly, Lz, dLx, dLy, dLz,
                     float(nx), float(ny), float(nz),
                     sph.ctypes.data, st.ctypes.data, ct.ctypes.data, it.ctypes.data,
                     D.ctypes.data, T2.ctypes.data)


def injected(normals: np.ndarray):
    n = np.ascontiguousarray(normals, dtype=np.float32)
    r = _Rng(RNG_INJECT, n.ctypes.data, n.shape[1], n.shape[2], 0, 0, 0, 0)
    r._keep = n
    return r


def philox(key0: int, key1: int = 0, stream: int = 0, id0: int = 0):
    """Philox draws; walker w of the call draws as global walker id0 + w."""
    return _Rng(RNG_PHILOX, None, 0, 0, key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF, stream & 0xFFFFFFFF,
                id0 & 0xFFFFFFFF)


def walk_f32(geom: Geometry, rng, mode: int, spins, spins0, step0: int, nsteps: int, dt: float,
             G=None, Garea=None, phase=None, diffdir=None, sig=None, phi=None,
             counters: bool = True, work: bool = False, nthreads: int = 0, phase64=None):
    """Run steps [step0, step0+nsteps) in place on float32 arrays.  Returns a
    dict of per-walker label / n_iter / n_scatter / flags (and work sums).
    phase64: optional [ndir, N] float64 receiving the exact (FP64) phase of
    this single-precision trajectory along diffdir."""
    N = spins.shape[1]
    g = geom.struct()
    lab = np.zeros(N, np.int32) if counters else None
    nit = np.zeros(N, np.int32) if counters else None
    nsc = np.zeros(N, np.int32) if counters else None
    flg = np.zeros(N, np.int32) if counters else None
    wk = np.zeros(4, np.int64) if work else None
    G = None if G is None else np.ascontiguousarray(G, np.float32)
    Garea = None if Garea is None else np.ascontiguousarray(Garea, np.float32)
    dd = None if diffdir is None else np.ascontiguousarray(diffdir, np.float32)
    ndir = 0 if dd is None else dd.shape[1]
    lib().oz_set_phase64(_ptr(phase64))
    try:
        rc = lib().oz_walk_f32(ctypes.byref(g), ctypes.byref(rng), mode, N, step0, nsteps, float(dt),
                               _ptr(G), _ptr(Garea), _ptr(spins), _ptr(spins0), _ptr(phase), _ptr(dd), ndir,
                               _ptr(sig), _ptr(phi), _ptr(lab), _ptr(nit), _ptr(nsc), _ptr(flg), _ptr(wk),
                               nthreads)
    finally:
        lib().oz_set_phase64(None)
    if rc != 0:
        raise RuntimeError(f"oz_walk_f32 failed ({rc})")
    return {"label": lab, "n_iter": nit, "n_scatter": nsc, "flags": flg, "work": wk}


def walk_f64(geom: Geometry, rng, mode: int, spins, spins0, step0: int, nsteps: int, dt: float,
             G=None, Garea=None, phase=None, diffdir=None, sig=None, phi=None, nthreads: int = 0):
    N = spins.shape[1]
    g = geom.struct()
    lab = np.zeros(N, np.int32)
    nit = np.zeros(N, np.int32)
    nsc = np.zeros(N, np.int32)
    flg = np.zeros(N, np.int32)
    G = None if G is None else np.ascontiguousarray(G, np.float64)
    Garea = None if Garea is None else np.ascontiguousarray(Garea, np.float64)
    dd = None if diffdir is None else np.ascontiguousarray(diffdir, np.float64)
    ndir = 0 if dd is None else dd.shape[1]
    rc = lib().oz_walk_f64(ctypes.byref(g), ctypes.byref(rng), mode, N, step0, nsteps, float(dt),
                           _ptr(G), _ptr(Garea), _ptr(spins), _ptr(spins0), _ptr(phase), _ptr(dd), ndir,
                           _ptr(sig), _ptr(phi), _ptr(lab), _ptr(nit), _ptr(nsc), _ptr(flg), nthreads)
    if rc != 0:
        raise RuntimeError(f"oz_walk_f64 failed ({rc})")
    return {"label": lab, "n_iter": nit, "n_scatter": nsc, "flags": flg}


def seed(geom: Geometry, targets, N: int, key0: int, key1: int = 0, stream: int = 1,
         max_rounds: int = 10000, nthreads: int = 0, id0: int = 0):
    """Seed walkers [id0, id0 + N) (oz_seed_range); returns (spins, label, left)."""
    tgt = np.zeros(geom.nstructures + 1, np.uint8)
    tgt[np.asarray(list(targets), dtype=np.int64)] = 1
    spins = np.full((3, N), np.nan, np.float32)
    label = np.zeros(N, np.int32)
    g = geom.struct()
    left = lib().oz_seed_range(ctypes.byref(g), tgt.ctypes.data, id0 & 0xFFFFFFFF, N, key0 & 0xFFFFFFFF,
                               key1 & 0xFFFFFFFF, stream, max_rounds, spins.ctypes.data, label.ctypes.data,
                               nthreads)
    return spins, label, left


def seed_accept(geom: Geometry, targets, pos):
    tgt = np.zeros(geom.nstructures + 1, np.uint8)
    tgt[np.asarray(list(targets), dtype=np.int64)] = 1
    pos = np.ascontiguousarray(pos, np.float32)
    out = np.zeros(pos.shape[1], np.uint8)
    g = geom.struct()
    lib().oz_seed_accept(ctypes.byref(g), tgt.ctypes.data, pos.shape[1], pos.ctypes.data, out.ctypes.data)
    return out.astype(bool)


def philox_block(counter, key0: int, key1: int) -> np.ndarray:
    """One Philox4x32-10 block of the 4-word counter under key (key0, key1)."""
    c = np.ascontiguousarray(np.asarray(counter, dtype=np.uint64) & 0xFFFFFFFF, dtype=np.uint32).copy()
    lib().oz_philox_block(c.ctypes.data, key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF)
    return c


def box_muller_pairs(ua, ub) -> np.ndarray:
    """The oracle's Box-Muller transform of 32-bit word pairs: [n, 2] float32."""
    ua = np.ascontiguousarray(ua, np.uint32)
    ub = np.ascontiguousarray(ub, np.uint32)
    out = np.zeros((ua.size, 2), np.float32)
    lib().oz_box_muller_pairs(ua.ctypes.data, ub.ctypes.data, ua.size, out.ctypes.data)
    return out


def philox_normals(key0: int, key1: int, stream: int, N: int, step: int, ndraw: int):
    """Normals [N, ndraw, 3] of draws 0..ndraw-1 of walkers 0..N-1 at `step`:
    counter (walker, step, draw, stream); words 0, 1 and 2, 3 go through one
    Box-Muller each, the last normal of the second pair unused."""
    out = np.zeros((N, ndraw, 3), np.float32)
    lib().oz_philox_normals(key0 & 0xFFFFFFFF, key1 & 0xFFFFFFFF, stream, N, step, ndraw, out.ctypes.data)
    return out


def moments(spins, spins0):
    out = np.zeros(6, np.float64)
    s = np.ascontiguousarray(spins, np.float32)
    s0 = np.ascontiguousarray(spins0, np.float32)
    lib().oz_moments(s.shape[1], s.ctypes.data, s0.ctypes.data, out.ctypes.data)
    return out


def signal_phi(phi, dirs, amps):
    phi = np.ascontiguousarray(phi, np.float32)
    dirs = np.ascontiguousarray(dirs, np.float64)
    amps = np.ascontiguousarray(amps, np.float64)
    ndir, nb = dirs.shape[1], amps.size
    re = np.zeros(ndir * nb)
    im = np.zeros(ndir * nb)
    lib().oz_signal_phi(phi.shape[1], phi.ctypes.data, dirs.ctypes.data, ndir, amps.ctypes.data, nb,
                        re.ctypes.data, im.ctypes.data)
    return (re + 1j * im).reshape(ndir, nb)


def signal_phase(phase, amps):
    phase = np.ascontiguousarray(phase, np.float64)
    amps = np.ascontiguousarray(amps, np.float64)
    ndir, N = phase.shape
    nb = amps.size
    re = np.zeros(ndir * nb)
    im = np.zeros(ndir * nb)
    lib().oz_signal_phase(N, phase.ctypes.data, ndir, amps.ctypes.data, nb, re.ctypes.data, im.ctypes.data)
    return (re + 1j * im).reshape(ndir, nb)
