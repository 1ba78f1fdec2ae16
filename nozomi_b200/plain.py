"""The plain per-substrate path: one substrate at a time, one launch of the
plain walk kernel per waveform sample with the reference's per-direction
phase array [ndir, N] in HBM (the data flow of
DwiSim3d.simulate_multi_directions, diffsim3d.py:246-261), then the signal.
It is the baseline the batched and served paths are measured against.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine
from . import _lib as L
from .waveforms import step_tables


def run_plain(dsub: engine.DeviceSubstrate, spec, positions: torch.Tensor) -> torch.Tensor:
    """Walk `positions` [3,N] through spec's waveform; returns the signal sums
    [2, ndir, nb] (float64, device)."""
    G, Ga = step_tables(spec.gwave)
    N = positions.shape[1]
    dirs = torch.as_tensor(np.asarray(spec.dirs, np.float32), device="cuda").contiguous()
    amps = torch.as_tensor(np.asarray(spec.amplitudes, np.float32).ravel(), device="cuda")
    nd = dirs.shape[1]
    wk = engine.Walkers(positions.clone(), positions.clone(), phase=torch.zeros((nd, N), device="cuda"), diffdir=dirs)
    draws = engine.philox_draws(spec.seed, 0)
    dt = float(spec.gwave.dt)
    s, w = dsub.struct(), wk.struct()
    lib = L.load()
    stream = torch.cuda.current_stream().cuda_stream
    for n in range(G.size):
        rc = lib.nz_walk_step(L.byref(s), L.byref(w), L.MODE_PHASE, np.float32(dt), np.float32(G[n]),
                              np.float32(Ga[n]), n, L.byref(draws), stream)
        if rc:
            L.check(rc, "nz_walk_step")
    out = torch.zeros((2, nd, amps.numel()), dtype=torch.float64, device="cuda")
    L.check(lib.nz_signal_phase(wk.phase.data_ptr(), nd, N, amps.data_ptr(), amps.numel(), out.data_ptr(), stream),
            "nz_signal_phase")
    return out
