"""Narrow-pulse driver: D(t) and K(t) of one substrate file
(the reference's cli/simulation_main.py:19-149).

Loads the substrate pickle, splits fibres and adds z-periodic pads, builds one
structure per fibre with the compartment's D, seeds walkers in the requested
compartment, then walks all steps in fused launches that accumulate the
per-step displacement moments on the device (the reference launches a walk
and a moment kernel per step).  Writes
``<substrate dir>/../sim/ADCdata/diffcoeff_<compartment>_<nseg>segments_<N>spins_<name>_TABLEtime<s>sec_SIMtime<s>sec_timestep<dt>ms.pkl``
holding ``np.column_stack((Dx, Dy, Dz, t))`` as the reference does, the
kurtoses beside it, and a JSON record of the run's timings and sizes.

Two differences from the reference's loop (its simulation_main.py:90-111),
both on purpose.  The walk takes exactly nt = int(sim_time / time_step)
steps; the reference's float-accumulated ``current_time < nt*time_step``
test sometimes takes one more, whose moments land past its arrays.  Row k
holds the moments after step k + 1 at t = (k + 1) * time_step; the
reference's saved ``diff_time[1:]`` is shifted by one step and ends in 0.
"""
from __future__ import annotations

import json
import os
import pickle
import time

import numpy as np
import torch

from .. import _lib as L
from ..diffsim3d import DiffSim3d
from ..geometry import SimGeometry3D, Structure3D
from ..substrates import ingest_on_device, load_pickle


def build_geometry(substrate_file, D, T2=100, rho=1):
    """The driver's ingestion (simulation_main.py:37-54): the pickle's matrix
    split into fibres at z == L/2 and z-padded from each fibre's partner,
    done on the GPU (substrates.ingest_on_device, bit-identical to the
    reference's split_matrix_to_list + createBoundaryZ), then one structure
    per fibre."""
    arr, L_box, box = load_pickle(substrate_file)
    rows, _, lengths = ingest_on_device(arr, L_box, box[2])
    r = rows.cpu().numpy()
    fibers = np.split(r, np.cumsum(lengths)[:-1]) if len(lengths) else []
    sg3 = SimGeometry3D(box[0], box[1], box[2], D, T2, rho)
    for f in fibers:
        sg3.add_structure(Structure3D(f[:, 0], f[:, 1], f[:, 2], f[:, 3], D, T2, rho))
    return sg3, fibers


def narrow_pulse(sim: DiffSim3d, nt: int, dt: float):
    """Walk nt steps with moments on the device.  Returns (t, D[3], K[3])."""
    moments = torch.zeros((nt, 6), dtype=torch.float64, device="cuda")
    zeros = np.zeros(nt, np.float32)
    sim.run_fused(zeros, zeros, dt, L.MODE_SIG | L.MODE_MOMENTS, steps_per_launch=L.MOMENT_STEPS,
                  moments=moments)
    m = moments.cpu().numpy()
    n = float(sim.nspins)
    t = dt * np.arange(1, nt + 1)
    Dv = m[:, :3] / (2 * t[:, None] * n)
    K = (m[:, 3:] / n) / (m[:, :3] / n) ** 2 - 3.0
    return t, Dv, K


def write_run_record(path, **fields):
    """The run's metrics as JSON beside its pickles (the reference keeps its
    timings only in the output file name): table and walk seconds, walkers,
    steps, and walker-steps/s of the walk."""
    rec = dict(fields)
    walk_s = float(rec.get("sim_time_s") or 0.0)
    rec["walker_steps_per_s"] = (rec["num_spins"] * rec["steps"] / walk_s) if walk_s > 0 else None
    with open(path, "w") as f:
        json.dump(rec, f, indent=1)
    return rec


def simulation_main(params, substrate_file):
    sim_time = float(params['sim_time'])
    dt = float(params['time_step'])
    N = int(params['num_spins'])
    compartment = params.get('compartment', 'intra') or 'intra'
    nseg = int(params['nseg'])
    D = params['D0_intra'] if compartment == 'intra' else params['D0_extra']
    target = os.path.dirname(os.path.dirname(substrate_file))
    sg3, fibers = build_geometry(substrate_file, D)
    nt = int(sim_time / dt)
    t0 = time.time()
    sim = DiffSim3d(sg3, N)
    sim.set_segments(nseg, nseg, nseg)
    if compartment == 'intra':
        sim.setup(structures=list(range(len(fibers))))
    elif compartment == 'extra':
        sim.setup(structures=[len(fibers)])
    else:
        sim.setup()
    table_time = round(time.time() - t0, 2)
    t1 = time.time()
    t, Dv, K = narrow_pulse(sim, nt, dt)
    torch.cuda.synchronize()
    walk_s = time.time() - t1
    sim_elapsed = round(walk_s, 2)
    base = os.path.splitext(os.path.basename(substrate_file))[0]
    name = (f"diffcoeff_{compartment}_{nseg}segments_{N}spins_{base}_TABLEtime{table_time}sec_"
            f"SIMtime{sim_elapsed}sec_timestep{dt}ms")
    out_dir = os.path.join(target, 'sim', 'ADCdata')
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, name + '.pkl')
    with open(path, 'wb') as f:
        pickle.dump(np.column_stack((Dv[:, 0], Dv[:, 1], Dv[:, 2], t)), f)
    with open(os.path.join(out_dir, name + '_kurtosis.pkl'), 'wb') as f:
        pickle.dump(np.column_stack((K[:, 0], K[:, 1], K[:, 2], t)), f)
    write_run_record(os.path.join(out_dir, name + '.json'), substrate=os.path.abspath(substrate_file),
                     compartment=compartment, num_spins=N, steps=nt, time_step_ms=dt, nseg=nseg,
                     table_time_s=float(table_time), sim_time_s=float(walk_s), D_final=Dv[-1].tolist(),
                     K_final=K[-1].tolist())
    print(f"simulation completed: {path}")
    return path
