"""Diffusion simulation engine with the reference's object API.

``DiffSim3d`` / ``DwiSim3d`` keep the methods, attributes and call sequence of
simulation_toolkit/simulation_engine/diffsim3d.py:8-261 — set_segments, setup,
step, dwi_step, dwi_multidirections_step,
calculate_diffusion_coefficients_and_kurtoses, simulate,
simulate_multi_directions — and the GPUArray-like attributes the reference's
tests read (``spins_d``, ``spins0_d``, ``sig_d``, ``phase_d`` with ``.get()``,
slicing and arithmetic).  Every step runs in libnozomi_b200.so:

  * ``step`` / ``dwi_step`` / ``dwi_multidirections_step``: one launch of the
    plain walk kernel per call, like the reference;
  * ``DwiSim3d.simulate*``: by default the whole waveform in a few fused
    launches (walker state in registers, Kahan-compensated phase as the
    3-vector Phi, phase_d += u_d . Phi at the end).  Trajectories are identical
    to the per-step path (same draws, same arithmetic); phases differ from the
    per-step FP32 sums only by their rounding.  ``exact=True`` runs the
    per-step path, whose phase matches the reference's float sums bit for bit.

Differences that callers may notice: no nvcc JIT per geometry (the library is
prebuilt), any walker count (the reference needs a multiple of 1000), draws
from a counter-based generator keyed by ``initstates_int`` (reproducible), and
an error instead of an endless loop when seeding targets have no volume.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine
from . import _lib as L
from .waveforms import step_tables


class DeviceArray:
    """The part of pycuda's GPUArray the reference's callers use, over a torch
    tensor on the device."""

    def __init__(self, t: torch.Tensor):
        self.t = t

    def get(self) -> np.ndarray:
        return self.t.detach().cpu().numpy()

    def copy(self) -> "DeviceArray":
        return DeviceArray(self.t.clone())

    @property
    def shape(self):
        return tuple(self.t.shape)

    @property
    def dtype(self):
        return np.dtype(str(self.t.dtype).replace("torch.", ""))

    @property
    def size(self):
        return self.t.numel()

    @property
    def ndim(self):
        return self.t.dim()

    def __len__(self):
        return self.t.shape[0]

    def __getitem__(self, idx):
        return DeviceArray(self.t[idx])

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a if dtype is None else a.astype(dtype)

    @staticmethod
    def _o(o):
        return o.t if isinstance(o, DeviceArray) else o

    def __add__(self, o): return DeviceArray(self.t + self._o(o))
    def __radd__(self, o): return DeviceArray(self._o(o) + self.t)
    def __sub__(self, o): return DeviceArray(self.t - self._o(o))
    def __rsub__(self, o): return DeviceArray(self._o(o) - self.t)
    def __mul__(self, o): return DeviceArray(self.t * self._o(o))
    def __rmul__(self, o): return DeviceArray(self._o(o) * self.t)
    def __truediv__(self, o): return DeviceArray(self.t / self._o(o))
    def __pow__(self, p): return DeviceArray(self.t ** p)
    def __neg__(self): return DeviceArray(-self.t)

    def __repr__(self):
        return f"DeviceArray({self.get()!r})"


class DiffSim3d:
    """Simulates diffusion within a 3D geometry of structures (diffsim3d.py:8-226)."""

    def __init__(self, geom, nspins, diffdir=None):
        engine.require_cuda()
        self.pars = dict()
        self.set_spins(nspins)
        self.set_geometry(geom)
        self.set_diffusion_directions(diffdir)
        self.set_block_grid(nspins)
        self.issetup = False
        self._sub = None
        self._fsub = None
        self._step = 0
        self._key = None

    # -- configuration (diffsim3d.py:65-104, :176-178) -----------------------
    def set_diffusion_directions(self, diffdir=None):
        if diffdir is None:
            diffdir = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1]])
        if np.isscalar(diffdir):
            raise TypeError("diffdir cannot be a scalar (so far)")
        diffdir = np.asarray(diffdir)
        if (diffdir.shape[0] != 3) or (diffdir.ndim != 2):
            raise TypeError("diffdir must be a numpy array of size 3xN")
        self.ndiffdir = diffdir.shape[1]
        self.pars['ndiffdir'] = self.ndiffdir
        self.diffdir = DeviceArray(torch.as_tensor(diffdir.astype(np.float32), device="cuda").contiguous())
        self.issetup = False

    def set_spins(self, nspins):
        self.nspins = int(nspins)
        self.pars['nspins'] = self.nspins
        self.issetup = False

    def set_geometry(self, geom):
        self.geom = geom
        self.pars['nspheres'] = geom.nsphere
        self.pars['nstructures'] = geom.nstructures
        self.pars['Lx'] = geom.Lx
        self.pars['Ly'] = geom.Ly
        self.pars['Lz'] = geom.Lz
        self.pars['D'] = ','.join(map(str, [s.D for s in geom.structures]))
        self.pars['T2'] = ','.join(map(str, [s.T2 for s in geom.structures]))
        self._sub = None
        self._fsub = None
        self.issetup = False

    def set_block_grid(self, nspins):
        """Kept for call compatibility; launch shapes are chosen by the library."""
        self.nblock = 256
        self.ngrid = (int(nspins) + 255) // 256

    def set_segments(self, nsegx=1, nsegy=1, nsegz=1, near_margin=None):
        """Cell lists on the GPU (diffsim3d.py:107-174): the member lists the
        kernels use and the reference's padded table in ``self.segments``."""
        self.nsegx, self.nsegy, self.nsegz = int(nsegx), int(nsegy), int(nsegz)
        self.pars['dLx'] = self.pars['Lx'] / self.nsegx
        self.pars['dLy'] = self.pars['Ly'] / self.nsegy
        self.pars['dLz'] = self.pars['Lz'] / self.nsegz
        self.pars['nLx'], self.pars['nLy'], self.pars['nLz'] = self.nsegx, self.nsegy, self.nsegz
        self._sub = self.geom.device_substrate(nseg=(self.nsegx, self.nsegy, self.nsegz), near_margin=near_margin)
        if self.geom.nsphere > 0:
            K, seg = self._sub.padded_segments()
            self.spheres_per_segment = K
            self.segments = seg.cpu().numpy()
            self.segments_d = DeviceArray(seg)
        else:
            self.spheres_per_segment = 0
            self.segments = np.zeros(0, np.intc)
        self.pars['nspheres_per_seg'] = self.spheres_per_segment
        self.issetup = False

    # The fused walk's own lists: 0.667 um cells (coarser for boxes that
    # would need more than about 4M cells) and a near margin of 3.9 step
    # lengths sqrt(2 D dt), clamped to [0.3, 0.9] um.  On packed beaded-axon
    # substrates this is within 2 % of the fastest shape measured both for
    # narrow-pulse runs (dt = 2 us) and for DWI (dt = 5 us).
    FUSED_CELL = 0.667
    FUSED_MARGIN_STEPS = 3.9
    FUSED_MAX_CELLS = 4_000_000
    DISP_BUDGET = 1 << 30  # bytes of per-step displacements one moments launch may store

    def _fused_substrate(self, dt: float):
        """Cell lists of the fused walk for time step dt, built once per
        geometry and margin.  They do not depend on set_segments: nseg sets
        the reference's padded table and the per-step path, while the fused
        walk scans its own finer grid.  The grid and margin change which
        spheres a walker scans, never a trajectory (every list holds every
        sphere within the 1 um margin the reference's lists hold)."""
        dmax = max(float(st.D) for st in self.geom.structures)
        margin = min(0.9, max(0.3, round(self.FUSED_MARGIN_STEPS * float(np.sqrt(2 * dmax * dt)), 2)))
        if self._fsub is None or self._fsub[0] != margin:
            vol = float(self.geom.Lx) * float(self.geom.Ly) * float(self.geom.Lz)
            cell = max(self.FUSED_CELL, (vol / self.FUSED_MAX_CELLS) ** (1.0 / 3.0))
            self._fsub = (margin, self.geom.device_substrate(cell=cell, near_margin=margin))
        return self._fsub[1]

    # -- set-up (diffsim3d.py:35-63) ----------------------------------------
    def setup(self, structures=None, initstates_int=None):
        if self._sub is None:
            self.set_segments()
        if initstates_int is None:
            initstates_int = int(np.random.randint(np.iinfo(np.int32).max))
        self._key = int(initstates_int)
        targets = list(range(self.geom.nstructures + 1)) if structures is None else [int(s) for s in structures]
        spins, label = engine.seed(self._sub, targets, self.nspins, key=self._key ^ 0x5EED)
        self.spins = spins.cpu().numpy()
        self.spins_d = DeviceArray(spins)
        self.spins0_d = self.spins_d.copy()
        self.phase_d = DeviceArray(torch.zeros(self.ndiffdir * self.nspins, dtype=torch.float32, device="cuda"))
        self.spheres_d = DeviceArray(self._sub.spheres)
        self.sig_d = DeviceArray(torch.ones((1, self.nspins), dtype=torch.float32, device="cuda"))
        self._label = label
        self._draws = engine.philox_draws(self._key, 0)
        self._step = 0
        self.issetup = True

    def _walkers(self, phase=None, diffdir=None) -> engine.Walkers:
        return engine.Walkers(self.spins_d.t, self.spins0_d.t, phase=phase, diffdir=diffdir,
                              sig=self.sig_d.t.view(-1))

    # -- one step per call (diffsim3d.py:199-226) -----------------------------
    def step(self, dt):
        if not self.issetup:
            self.setup()
        engine.walk_step(self._sub, self._walkers(), L.MODE_SIG, dt, 0.0, 0.0, self._step, self._draws)
        self._step += 1

    def dwi_step(self, gwave_dt, G, G_area_at_each_time_step):
        """randomWalk3d_phase: phase along x, y, z into rows 0..2 of phase_d."""
        if not self.issetup:
            self.setup()
        if self.ndiffdir < 3:
            raise ValueError("dwi_step writes three phase rows: construct with 3 or more directions")
        eye = getattr(self, "_eye", None)
        if eye is None:
            eye = self._eye = torch.eye(3, dtype=torch.float32, device="cuda").contiguous()
        phase = self.phase_d.t.view(self.ndiffdir, self.nspins)[:3]
        engine.walk_step(self._sub, self._walkers(phase=phase, diffdir=eye), L.MODE_PHASE, gwave_dt, G,
                         G_area_at_each_time_step, self._step, self._draws)
        self._step += 1

    def dwi_multidirections_step(self, gwave_dt, G, G_area_at_each_time_step):
        if not self.issetup:
            self.setup()
        phase = self.phase_d.t.view(self.ndiffdir, self.nspins)
        engine.walk_step(self._sub, self._walkers(phase=phase, diffdir=self.diffdir.t), L.MODE_PHASE, gwave_dt, G,
                         G_area_at_each_time_step, self._step, self._draws)
        self._step += 1

    # -- narrow-pulse moments (diffsim3d.py:180-197) --------------------------
    def calculate_diffusion_coefficients_and_kurtoses(self, step_idx, current_time, dx_array, dy_array, dz_array,
                                                     Kx2_array, Ky2_array, Kz2_array, Kx4_array, Ky4_array,
                                                     Kz4_array):
        """Adds, at index step_idx: sum dx^2 / (2 t N) to the D arrays and
        sum dx^2 / N, sum dx^4 / N to the second / fourth moment arrays."""
        m = torch.zeros(6, dtype=torch.float64, device="cuda")
        engine.moments(self.spins_d.t, self.spins0_d.t, m)
        n = float(self.nspins)
        t = float(current_time)
        for arr, v in ((dx_array, m[0] / (2 * t * n)), (dy_array, m[1] / (2 * t * n)), (dz_array, m[2] / (2 * t * n)),
                       (Kx2_array, m[0] / n), (Ky2_array, m[1] / n), (Kz2_array, m[2] / n),
                       (Kx4_array, m[3] / n), (Ky4_array, m[4] / n), (Kz4_array, m[5] / n)):
            tgt = arr.t if isinstance(arr, DeviceArray) else arr
            tgt[step_idx] += v.to(tgt.dtype)

    # -- fused: many steps per launch -------------------------------------------
    def run_fused(self, G, Garea, dt, mode, steps_per_launch=2000, coarsen=None, phi=None, moments=None):
        """All steps of the G / Garea tables through the fused walk, on the
        walkers of this object (positions, spins0, sig and Phi updated).
        Walkers are re-binned between launches by (label, bin) with bins of
        about 4 um (``coarsen`` cells per axis)."""
        if not self.issetup:
            self.setup()
        fsub = self._fused_substrate(dt)
        if coarsen is None:
            coarsen = max(1, int(round(4.0 / (float(self.geom.Lx) / fsub.nseg[0]))))
        G = torch.as_tensor(np.asarray(G, np.float32), device="cuda")
        Garea = torch.as_tensor(np.asarray(Garea, np.float32), device="cuda")
        n = int(G.numel())
        if phi is None:
            phi = torch.zeros((6, self.nspins), dtype=torch.float32, device="cuda")
        wk = engine.Walkers(self.spins_d.t, self.spins0_d.t, phi=phi, sig=self.sig_d.t.view(-1),
                            label=self._label)
        st = engine.FusedState.from_walkers(wk)
        spare = engine.FusedState(self.nspins)
        scratch = None
        s0 = 0
        # moments without phase: the walk stores per-step displacements (at
        # most about 1 GiB of them per launch) and one reduction forms the sums
        disp = bool(mode & L.MODE_MOMENTS) and not (mode & (L.MODE_PHI | L.MODE_PHASE))
        dscratch = None
        if disp:
            per = max(1, min(steps_per_launch, self.DISP_BUDGET // (12 * max(self.nspins, 1))))
        else:
            per = steps_per_launch if not (mode & L.MODE_MOMENTS) else min(steps_per_launch, L.MOMENT_STEPS)
        Gs = torch.zeros(self._step + n, dtype=torch.float32, device="cuda")
        Gas = torch.zeros_like(Gs)
        Gs[self._step:] = G
        Gas[self._step:] = Garea
        while s0 < n:
            s1 = min(n, s0 + per)
            scratch = st.sort_into(spare, fsub.grid, coarsen, scratch, nlabels=fsub.nstructures + 1)
            st, spare = spare, st
            if disp:
                dscratch = engine.walk_fused_moments(fsub, st, mode & L.MODE_SIG, dt, self._step + s0,
                                                     self._step + s1, self._draws, moments, dscratch)
            else:
                engine.walk_fused(fsub, st, mode, dt, Gs, Gas, self._step + s0, self._step + s1, self._draws,
                                  moments=moments)
            s0 = s1
        st.to_walkers_by_id(wk)  # back to walker-id order, the reference's layout
        self._label = wk.label
        self._step += n
        return phi


class DwiSim3d(DiffSim3d):
    """DWI phase over a gradient waveform (diffsim3d.py:228-261)."""

    def _protocol(self, gwave):
        return step_tables(gwave)

    def simulate(self, gwave, structures=None, initstates=None, exact=False):
        """Phase along x, y, z: [ndiffdir, nspins] (rows 0..2 written)."""
        if not self.issetup:
            self.setup(structures=structures, initstates_int=initstates)
        G, Ga = self._protocol(gwave)
        if exact:
            for n in range(G.size):
                self.dwi_step(gwave.dt, float(G[n]), float(Ga[n]))
        else:
            phi = self.run_fused(G, Ga, gwave.dt, L.MODE_PHI | L.MODE_SIG)
            eye = torch.eye(3, dtype=torch.float32, device="cuda").contiguous()
            self._add_phase(phi, eye, rows=3)
        return self.phase_d.get().reshape(self.ndiffdir, self.nspins)

    def simulate_multi_directions(self, gwave, structures=None, initstates=None, exact=False):
        """Phase along every direction of diffdir: [ndiffdir, nspins]."""
        if not self.issetup:
            self.setup(structures=structures, initstates_int=initstates)
        G, Ga = self._protocol(gwave)
        if exact:
            for n in range(G.size):
                self.dwi_multidirections_step(gwave.dt, float(G[n]), float(Ga[n]))
        else:
            phi = self.run_fused(G, Ga, gwave.dt, L.MODE_PHI | L.MODE_SIG)
            self._add_phase(phi, self.diffdir.t, rows=self.ndiffdir)
        return self.phase_d.get().reshape(self.ndiffdir, self.nspins)

    def _add_phase(self, phi, dirs, rows):
        wk = engine.Walkers(self.spins_d.t, self.spins0_d.t, phi=phi)
        st = engine.FusedState.from_walkers(wk)
        ph = st.phase(dirs)
        self.phase_d.t.view(self.ndiffdir, self.nspins)[:rows] += ph

    def signal(self, gwave, bvalues=None, amplitudes=None, structures=None, initstates=None):
        """Normalised signal S[d][b] = mean_w exp(i a_b phi_w,d) of a fresh run
        of the waveform (amplitudes in units of 100 mT/m, or b in ms/um^2)."""
        if amplitudes is None:
            amplitudes = gwave.amplitude_for_b(bvalues)
        if not self.issetup:
            self.setup(structures=structures, initstates_int=initstates)
        G, Ga = self._protocol(gwave)
        phi = self.run_fused(G, Ga, gwave.dt, L.MODE_PHI | L.MODE_SIG)
        st = engine.FusedState.from_walkers(engine.Walkers(self.spins_d.t, self.spins0_d.t, phi=phi))
        amps = torch.as_tensor(np.asarray(amplitudes, np.float32).ravel(), device="cuda")
        s = st.signal(self.diffdir.t, amps).cpu().numpy()
        return (s[0] + 1j * s[1]) / self.nspins
