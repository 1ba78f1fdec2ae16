"""The fused production path of one substrate: seed, walk every step of a
protocol in a few launches with walkers re-binned by cell between them, and
reduce the signal on the device.

This is the work of DwiSim3d.simulate_multi_directions
(simulation_toolkit/simulation_engine/diffsim3d.py:246-261, one kernel launch
per waveform sample) plus the signal reduction the reference leaves to the
caller, and of the narrow-pulse loop of cli/simulation_main.py:91-118 (walk
plus one moment kernel per step).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import engine
from . import _lib as L
from .substrates import Substrate, cell_grid
from .waveforms import step_tables


@dataclass
class Tuning:
    """Launch shape of the fused walk (chosen by nozomi_b200.autotune)."""
    cell: float = 1.0             # cell edge, um
    steps_per_launch: int = 500   # steps between walker re-binnings
    coarsen: int = 4              # re-binning bins = cells coarsened by this factor per axis
    by_label: bool = True         # re-bin by (label, bin): a warp's walkers share a structure
    near_margin: float | None = 0.5  # margin of the near lists (None: full lists only)
    lists: str = "index"          # the fused walk's list form: "index" (16/32-bit) or "records"
    near_shape: str = "round"     # near lists by the Euclidean sphere-to-cell test ("round") or the box test
    stage: int = 0                # batched walk: records a CTA stages in shared memory (0: none)


def idx_bytes_for(lists: str):
    """DeviceSubstrate's idx_bytes for a Tuning.lists value."""
    if lists == "records":
        return 0
    if lists == "index":
        return None
    raise ValueError(f"list form {lists!r} is not 'index' or 'records'")


def device_substrate(sub: Substrate, D=2.0, T2=100.0, cell: float = 1.0, nseg=None, D_box=None,
                     jump_tol: float = 1.0, near_margin: float | None = None,
                     lists: str = "index", near_shape: str = "round") -> engine.DeviceSubstrate:
    nseg = cell_grid(sub.L, cell) if nseg is None else nseg
    ns = sub.nstructures
    Dv = np.full(ns + 1, D, np.float32)
    if D_box is not None:
        Dv[ns] = D_box
    T2v = np.full(ns + 1, T2, np.float32)
    if near_shape not in ("round", "box"):
        raise ValueError(f"near-list shape {near_shape!r} is not 'round' or 'box'")
    return engine.DeviceSubstrate(sub.spheres(), ns, sub.L, nseg, Dv, T2v, jump_tol=jump_tol, near_margin=near_margin,
                                  idx_bytes=idx_bytes_for(lists), near_round=near_shape == "round")


class DwiRun:
    """Walkers of one substrate under one gradient waveform; signal for every
    (direction, amplitude) pair of the unit-amplitude waveform (phase is linear
    in the gradient: phi(a) = a * phi(1))."""

    def __init__(self, dsub: engine.DeviceSubstrate, gwave, dirs: np.ndarray, amplitudes, N: int, seed: int = 0,
                 targets=None, tuning: Tuning | None = None, positions: torch.Tensor | None = None, id0: int = 0):
        self.sub = dsub
        self.id0 = int(id0)  # global id of walker 0: a shard walks walkers [id0, id0 + N) of a larger run
        self.tuning = tuning or Tuning()
        self.dt = float(gwave.dt)
        G, Ga = step_tables(gwave)
        self.nsteps = G.size
        dev = torch.device("cuda", torch.cuda.current_device())
        self.G = torch.from_numpy(G).to(dev)
        self.Garea = torch.from_numpy(Ga).to(dev)
        d = np.asarray(dirs, np.float64)
        if d.ndim != 2 or d.shape[0] != 3:
            raise TypeError("dirs must be a 3 x ndir array")
        self.dirs = torch.from_numpy(d.astype(np.float32)).to(dev)
        self.amps = torch.as_tensor(np.asarray(amplitudes, np.float32).ravel(), device=dev)
        self.N = int(N)
        self.seed = int(seed)
        self.targets = list(range(dsub.nstructures + 1)) if targets is None else list(targets)
        self.draws = engine.philox_draws(self.seed, 0)
        self.positions = positions
        self._scratch = None
        self.launches = 0

    def initial_positions(self):
        """(positions [3,N], labels [N]) — given, or seeded on the device."""
        if self.positions is not None:
            return self.positions, None
        return engine.seed(self.sub, self.targets, self.N, key=self.seed ^ 0x5EED, id0=self.id0)

    def prepare(self, positions=None, labels=None):
        """Walker state from positions [3, N] and labels [N] (seeded on the
        device when None).  Host arrays (numpy or CPU tensors) are copied to
        the current GPU on the current stream, asynchronously when they are
        pinned; the caller keeps them unchanged until the stream has passed
        the copy."""
        if positions is None:
            positions, labels = self.initial_positions()
        dev = torch.device("cuda", torch.cuda.current_device())
        x = torch.as_tensor(positions)
        if x.device != dev or x.dtype != torch.float32:
            x = x.to(dev, torch.float32, non_blocking=True)
        if x.dim() != 2 or x.shape[0] != 3:
            raise TypeError("positions must be a 3 x N array")
        N = x.shape[1]
        if labels is None:
            lab = torch.full((N,), -1, dtype=torch.int32, device=dev)
        else:
            lab = torch.as_tensor(labels)
            if lab.device != dev or lab.dtype != torch.int32:
                lab = lab.to(dev, torch.int32, non_blocking=True)
            if lab.numel() != N:
                raise TypeError("labels need one entry per walker")
        wk = engine.Walkers(x.contiguous(), x.clone(), phi=torch.zeros((6, N), device=dev), label=lab.contiguous())
        ids = None
        if self.id0:
            ids = torch.arange(self.id0, self.id0 + N, dtype=torch.int64, device=dev).to(torch.int32)
        self.state = engine.FusedState.from_walkers(wk, ids)
        self.spare = engine.FusedState(N)
        self.launches = 1 if N else 0  # library kernels since prepare: the pack
        return self

    def walk(self, events: list | None = None):
        """All steps: re-bin, then one fused launch per steps_per_launch steps.
        events: if a list, (start, end) CUDA events of each fused launch are
        appended to it."""
        t = self.tuning
        nl = self.sub.nstructures + 1 if t.by_label else 0
        stream = torch.cuda.current_stream()
        for s0 in range(0, self.nsteps, t.steps_per_launch):
            self.launches += self.state.sort_kernels(self.sub.grid, t.coarsen, nl) + (1 if self.state.N else 0)
            self._scratch = self.state.sort_into(self.spare, self.sub.grid, t.coarsen, self._scratch, nlabels=nl)
            self.state, self.spare = self.spare, self.state
            if events is not None:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            engine.walk_fused(self.sub, self.state, L.MODE_PHI, self.dt, self.G, self.Garea, s0,
                              min(self.nsteps, s0 + t.steps_per_launch), self.draws)
            if events is not None:
                e1.record(stream)
                events.append((e0, e1))
        return self

    def signal_sums(self) -> torch.Tensor:
        """[2, ndir, nb] float64 sums over walkers of cos / sin."""
        out = self.state.signal(self.dirs, self.amps)
        self.launches += 1 if self.state.N else 0
        return out

    def signal(self) -> np.ndarray:
        s = self.signal_sums().cpu().numpy()
        return (s[0] + 1j * s[1]) / self.state.N

    def walkers(self) -> engine.Walkers:
        """The walkers in walker-id order, reference layout (positions, spins0,
        Phi [6,N], label, flags)."""
        N = self.state.N
        dev = self.state.pos.device

        def fresh():
            return engine.Walkers(torch.empty((3, N), device=dev), torch.empty((3, N), device=dev),
                                  phi=torch.empty((6, N), device=dev),
                                  label=torch.empty(N, dtype=torch.int32, device=dev),
                                  flags=torch.empty(N, dtype=torch.int32, device=dev))
        wk = fresh()
        if not self.id0:
            self.state.to_walkers_by_id(wk)
            return wk
        # a shard: state order, then scattered to slot (walker id - id0)
        self.state.to_walkers(wk)
        slot = self.state.walker_ids().to(torch.int64) - self.id0
        out = fresh()
        for name in ("spins", "spins0", "phi"):
            getattr(out, name)[:, slot] = getattr(wk, name)
        for name in ("label", "flags"):
            getattr(out, name)[slot] = getattr(wk, name)
        return out

    def phase(self) -> torch.Tensor:
        """Per-walker phase [ndir, N] of the unit waveform, walker-id order."""
        wk = self.walkers()
        st = engine.FusedState.from_walkers(wk)
        return st.phase(self.dirs)


def simulate_dwi(sub: Substrate, gwave, dirs, bvalues=None, amplitudes=None, N: int = 100000, D=2.0, T2=100.0,
                 seed: int = 0, targets=None, tuning: Tuning | None = None) -> np.ndarray:
    """Signal S[d][b] of a substrate under gwave, along dirs, for b-values
    (ms/um^2) or wave amplitudes (units of 100 mT/m)."""
    engine.require_cuda()
    if amplitudes is None:
        amplitudes = gwave.amplitude_for_b(bvalues)
    tuning = tuning or Tuning()
    dsub = device_substrate(sub, D=D, T2=T2, cell=tuning.cell, near_margin=tuning.near_margin, lists=tuning.lists,
                            near_shape=tuning.near_shape)
    run = DwiRun(dsub, gwave, dirs, amplitudes, N, seed=seed, targets=targets, tuning=tuning).prepare()
    return run.walk().signal()
