"""Statistics against the reference's own kernel on the GPU.

The reference's randomWalk3d_phase_multidirr (sim3d_kernel.cu:719-943),
compiled from its source with its template filled in (baseline/_ref, built
where the reference tree is present), walks the single beaded axon (40
spheres + z images, 8x8x40 um, cells 1x1x8) with 1e4 intra-axonal walkers,
D = 2, PGSE 20/10/30 ms at dt = 10 us (3000 launches), x and z, |G| 0..300
mT/m in 8 steps, with its own cuRAND draws.  The fused walk runs the same
seeded walkers with its Philox draws.  The two are independent Monte Carlo
estimates: per (direction, |G|) the difference is compared with its
standard error sqrt((var_ref + var_ours) / N), var of the complex per-walker
signal (cos and sin).  Bar: every cell within 3 sigma, allowing one of the 14
non-trivial cells to lie between 3 and 4 sigma (a 3-sigma criterion over 14
cells fails by chance about 4 % of the time).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _complex_var(phase, amps):
    arg = amps[None, :, None] * phase[:, None, :]
    return np.cos(arg).var(axis=2) + np.sin(arg).var(axis=2)


def test_signal_matches_reference_kernel_within_3_sigma():
    from baseline.reference_gpu import RefGpuWalk, built
    from nozomi_b200 import engine
    from nozomi_b200.simulate import DwiRun, Tuning, device_substrate
    from nozomi_b200.substrates import beaded_axon
    from nozomi_b200.waveforms import PGDiffWaveform, step_tables
    if built("single_axon_1e4") is None:
        pytest.skip("baseline/_ref/single_axon_1e4.so not built (the reference source tree was absent at build)")
    sub = beaded_axon()
    dsub = device_substrate(sub, D=2.0, nseg=(1, 1, 8))
    ref = RefGpuWalk("single_axon_1e4")
    N = ref.N
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.01)
    G, Ga = step_tables(pg)
    dirs = np.array([[1.0, 0.0], [0.0, 0.0], [0.0, 1.0]])
    amps = np.linspace(0.0, 3.0, 8)
    x0, lab0 = engine.seed(dsub, [0], N, key=31 ^ 0x5EED)

    K, seg = dsub.padded_segments()
    ref.setup(torch.from_numpy(sub.spheres().astype(np.float32)).cuda(), seg, K, x0, 2,
              torch.from_numpy(dirs.astype(np.float32)).cuda())
    ref.initstates(12345)
    dt = np.float32(pg.dt)
    for n in range(G.size):
        ref.step(dt, G[n], Ga[n])
    torch.cuda.synchronize()
    ph_ref = ref.phase.view(2, N).double().cpu().numpy()
    S_ref = np.exp(1j * amps[None, :, None] * ph_ref[:, None, :]).mean(axis=2)
    # the reference keeps every walker inside the axon; so must both runs
    assert np.all(np.isfinite(ph_ref))

    run = DwiRun(dsub, pg, dirs, amps, N, seed=31, targets=[0], tuning=Tuning(steps_per_launch=500))
    run.prepare(x0, lab0).walk()
    S = run.signal()
    ph = run.phase().double().cpu().numpy()
    wk = run.walkers()
    assert int((wk.label != 0).sum()) == 0

    sigma = np.sqrt((_complex_var(ph_ref, amps) + _complex_var(ph, amps)) / N)
    z = np.abs(S - S_ref)[:, 1:] / sigma[:, 1:]
    print("z per (direction, |G|):", np.round(z, 2).tolist())
    assert np.abs(S[:, 0] - 1).max() < 1e-12 and np.abs(S_ref[:, 0] - 1).max() < 1e-12
    assert z.max() <= 4.0, z
    assert int((z > 3.0).sum()) <= 1, z


def test_packed_signal_matches_reference_kernel():
    """The headline workload: the reference's own kernel (packed_1e6 build,
    block 1000, one launch per waveform sample, cuRAND draws) against the
    fused walk on the packed substrate, 1e6 walkers from the same seeded
    positions, all 6000 steps, 30 directions x b in {1, 2, 3} ms/um^2 (90
    cells).  Independent Monte Carlo estimates: no cell beyond 4 sigma and at
    most 2 of the 90 beyond 3 sigma (a 3-sigma criterion over 90 cells fails
    by chance in about a fifth of runs).  NOZOMI_PACKED_STATS=<path> writes
    the z-scores as JSON."""
    import json
    import os
    from baseline.reference_gpu import RefGpuWalk, built
    from nozomi_b200 import engine
    from nozomi_b200.simulate import DwiRun, Tuning, device_substrate
    from nozomi_b200.waveforms import step_tables
    from nozomi_b200.workloads import packed_workload
    if built("packed_1e6") is None:
        pytest.skip("baseline/_ref/packed_1e6.so not built (the reference source tree was absent at build)")
    sub, pg, dirs, bvals = packed_workload()
    amps = pg.amplitude_for_b(bvals)
    ref = RefGpuWalk("packed_1e6")
    N = ref.N
    dsub_ref = device_substrate(sub, D=2.0, T2=100.0, cell=1.0)
    K, seg = dsub_ref.padded_segments()
    x0, lab0 = engine.seed(dsub_ref, list(range(sub.nstructures + 1)), N, key=1000 ^ 0x5EED)
    ref.setup(torch.from_numpy(sub.spheres().astype(np.float32)).cuda(), seg, K, x0, dirs.shape[1],
              torch.from_numpy(dirs.astype(np.float32)).cuda())
    ref.initstates(777)
    G, Ga = step_tables(pg)
    dt = np.float32(pg.dt)
    for n in range(G.size):
        ref.step(dt, G[n], Ga[n])
    torch.cuda.synchronize()
    ph_ref = ref.phase.view(dirs.shape[1], N).double().cpu().numpy()
    del ref, seg

    tuning = Tuning(cell=0.5, near_margin=0.5, coarsen=8, steps_per_launch=2000)
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=tuning.cell, near_margin=tuning.near_margin)
    run = DwiRun(dsub, pg, dirs, amps, N, seed=1000, tuning=tuning)
    run.prepare(x0, lab0).walk()
    ph = run.phase().double().cpu().numpy()

    zs = []
    for b in range(1, amps.size):
        e_ref = np.exp(1j * amps[b] * ph_ref)
        e = np.exp(1j * amps[b] * ph)
        S_ref, S = e_ref.mean(axis=1), e.mean(axis=1)
        var = (e_ref.real.var(axis=1) + e_ref.imag.var(axis=1) + e.real.var(axis=1) + e.imag.var(axis=1))
        zs.append(np.abs(S - S_ref) / np.sqrt(var / N))
    z = np.array(zs)
    path = os.environ.get("NOZOMI_PACKED_STATS")
    if path:
        with open(path, "w") as f:
            json.dump({"z": z.tolist(), "max": float(z.max()), "beyond_3": int((z > 3).sum()), "cells": int(z.size),
                       "mean_abs_S_by_b": [float(np.abs(np.exp(1j * a * ph).mean(axis=1)).mean()) for a in amps]},
                      f, indent=1)
    print("max z", float(z.max()), "beyond 3 sigma", int((z > 3).sum()), "of", z.size)
    assert z.max() <= 4.0, z
    assert int((z > 3.0).sum()) <= 2, z
