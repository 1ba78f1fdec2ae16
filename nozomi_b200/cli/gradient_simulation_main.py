"""Gradient (PGSE / OGSE) driver of one substrate file.

The reference's CLI dispatches ``gradient_simulation`` to a module that is
not in its tree (cli/main.py:17, .gitignore:25); this driver builds the same
walk from the engine API it calls (DwiSim3d.simulate_multi_directions,
diffsim3d.py:246-261) and the JSON keys of
experiment/setup/simulation/{pgse,ogse}_sim_params.json: ``gradient.type``
PGSE (big_delta, little_delta) or OGSE (num_oscil, duration), gradient
``direction`` (one [x, y, z] or a list of them), optional ``bvalues``
(ms/um^2).  Writes the per-walker phase [ndir, N] of the unit waveform and the
signal per (direction, b) to ``<substrate dir>/../sim/DWIdata/``, with a JSON
record of the run's timings and sizes beside them.
"""
from __future__ import annotations

import os
import pickle
import time

import numpy as np

from ..diffsim3d import DwiSim3d
from ..waveforms import ApodizedCosineOGSEWaveform, PGDiffWaveform
from .simulation_main import build_geometry, write_run_record


def waveform(params):
    g = params['gradient']
    dt = float(params['time_step'])
    te = float(params['sim_time'])
    kind = g['type'].upper()
    if kind == 'PGSE':
        return PGDiffWaveform(float(g['big_delta']), float(g['little_delta']), te, time_step=dt)
    if kind == 'OGSE':
        return ApodizedCosineOGSEWaveform(int(g['num_oscil']), float(g['duration']), te=te, time_step=dt)
    raise ValueError(f"unknown gradient type {g['type']}")


def directions(params):
    d = np.asarray(params['gradient'].get('direction', [1, 0, 0]), np.float64)
    d = d.reshape(-1, 3).T
    return d / np.linalg.norm(d, axis=0)


def simulation_gradient_main(params, substrate_file):
    N = int(params['num_spins'])
    compartment = params.get('compartment', 'intra') or 'intra'
    nseg = int(params['nseg'])
    D = params['D0_intra'] if compartment == 'intra' else params['D0_extra']
    sg3, fibers = build_geometry(substrate_file, D)
    gw = waveform(params)
    dirs = directions(params)
    sim = DwiSim3d(sg3, N, diffdir=dirs)
    sim.set_segments(nseg, nseg, nseg)
    if compartment == 'intra':
        sim.setup(structures=list(range(len(fibers))))
    elif compartment == 'extra':
        sim.setup(structures=[len(fibers)])
    else:
        sim.setup()
    t0 = time.time()
    phase = sim.simulate_multi_directions(gw)  # returns host arrays: the walk is complete
    walk_s = time.time() - t0
    bvals = np.asarray(params.get('bvalues', [0.0, 1.0, 2.0, 3.0]), np.float64)
    amps = gw.amplitude_for_b(bvals)
    S = np.array([[np.mean(np.exp(1j * a * phase[d])) for a in amps] for d in range(dirs.shape[1])])
    target = os.path.dirname(os.path.dirname(substrate_file))
    out_dir = os.path.join(target, 'sim', 'DWIdata')
    os.makedirs(out_dir, exist_ok=True)
    base = os.path.splitext(os.path.basename(substrate_file))[0]
    path = os.path.join(out_dir, f"dwi_{compartment}_{params['gradient']['type']}_{N}spins_{base}.pkl")
    with open(path, 'wb') as f:
        pickle.dump({"phase": phase, "directions": dirs, "bvalues": bvals, "signal": S,
                     "b_unit": gw.calculate_bvalue_from_wave()}, f)
    write_run_record(os.path.splitext(path)[0] + '.json', substrate=os.path.abspath(substrate_file),
                     compartment=compartment, num_spins=N, steps=int(len(gw.wave)), time_step_ms=float(gw.dt),
                     nseg=nseg, directions=int(dirs.shape[1]), bvalues=bvals.tolist(), sim_time_s=float(walk_s))
    print(f"gradient simulation completed: {path}")
    return path
