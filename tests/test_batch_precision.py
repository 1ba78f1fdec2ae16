"""The signal-error bar of the batched and served paths against the FP64
oracle, on jobs drawn from the mixed workload's distribution: substrates of
10-500 beaded axons, 2000-8000 steps at dt = 5 us, 6-60 directions uniform on
the sphere, b in {0, 1, 2, 3} ms/um^2 (seed 4, the batched workload's
generator), with walker counts cut to 1000-3000 so the CPU oracle finishes in
seconds.  Every job keeps its full step count.

Per job, three comparisons on the same seeded walkers and draws:

  positions  the batched walk's final positions against the oracle's FP32
             walk (the reference's arithmetic), bit for bit;
  accrual    the batched signal against the FP64 signal of the same FP32
             trajectories (the oracle sums every phase increment in FP64):
             the error of the FP32 Kahan phase and FP32 per-walker cos/sin,
             bar 1e-3 (the target signal error);
  walk       the batched signal against the full-FP64 oracle walk.  FP32 and
             FP64 collision decisions in the 1e-4 um tolerance shells round
             differently and decorrelate the walkers, so the two walks agree
             statistically: bar 4 standard errors of a difference of two
             independent N-walker means (the largest over up to 60 x 4 cells).

The served path (requests admitted while others run) must give the batched
result to FP64 summation order.  Set NOZOMI_BATCH_PRECISION_REPORT=<path> to
write the per-job errors as JSON.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def jobs():
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.workloads import mixed_specs
    specs = mixed_specs(seed=4, n_jobs=6, walkers=(1000, 3000))
    tuning = Tuning()
    cache = SubstrateCache()
    run = BatchRun(specs, tuning=tuning, threads=128, cache=cache).step()
    return specs, tuning, cache, run, run.signals()


def _oracle_geometry(dsub):
    from oracle import oracle as oz
    return oz.Geometry(dsub.spheres.cpu().numpy(), dsub.nstructures, dsub.L, dsub.nseg, dsub.cell_start.cpu().numpy(),
                       dsub.cell_count.cpu().numpy(), dsub.cell_items.cpu().numpy()[:dsub.n_items],
                       dsub.D.cpu().numpy(), dsub.T2.cpu().numpy())


def test_batched_signal_error_against_fp64_oracle(jobs):
    from nozomi_b200 import engine
    from nozomi_b200.waveforms import step_tables
    from oracle import oracle as oz
    specs, tuning, cache, run, sig = jobs
    report = []
    for i, sp in enumerate(specs):
        dsub = cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning)
        g = _oracle_geometry(dsub)
        N = sp.N
        x0 = run.positions[i][0].cpu().numpy()
        G, Ga = step_tables(sp.gwave)
        nt, dt = G.size, float(sp.gwave.dt)
        dirs = np.asarray(sp.dirs, np.float64)
        amps = np.asarray(sp.amplitudes, np.float64).ravel()
        # the FP32 trajectories of the oracle, with their phase summed in FP64
        sp32, s032, phi = x0.copy(), x0.copy(), np.zeros((6, N), np.float32)
        ph = np.zeros((dirs.shape[1], N))
        oz.walk_f32(g, oz.philox(sp.seed), oz.MODE_PHI, sp32, s032, 0, nt, dt, G=G, Garea=Ga, phi=phi,
                    diffdir=dirs.astype(np.float32), phase64=ph, counters=False)
        wk = engine.Walkers(torch.empty((3, N), device="cuda"), torch.empty((3, N), device="cuda"),
                            phi=torch.empty((6, N), device="cuda"))
        run.final_state(i).to_walkers_by_id(wk)
        np.testing.assert_array_equal(wk.spins.cpu().numpy(), sp32)
        exact = oz.signal_phase(ph, amps)
        accrual = float(np.abs(sig[i] - exact).max())
        # the full-FP64 walk with the same draws
        x64 = x0.astype(np.float64)
        ph64 = np.zeros((dirs.shape[1], N))
        oz.walk_f64(g, oz.philox(sp.seed), oz.MODE_PHASE, x64, x64.copy(), 0, nt, dt, G=G.astype(np.float64),
                    Garea=Ga.astype(np.float64), phase=ph64, diffdir=dirs)
        S64 = oz.signal_phase(ph64, amps)
        arg = amps[None, :, None] * ph64[:, None, :]
        sigma = np.sqrt(2 * (np.cos(arg).var(axis=2) + np.sin(arg).var(axis=2)) / N)
        walk = np.abs(sig[i] - S64)
        ok = sigma > 0
        report.append({"job": i, "walkers": N, "steps": nt, "directions": int(dirs.shape[1]),
                       "spheres": int(dsub.S), "accrual_max_err": accrual, "walk_max_abs_err": float(walk.max()),
                       "walk_max_err_in_sigma": float((walk[ok] / sigma[ok]).max())})
    print(json.dumps(report))
    path = os.environ.get("NOZOMI_BATCH_PRECISION_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(report, f, indent=1)
    for r in report:
        assert r["accrual_max_err"] <= 1e-3, r
        assert r["walk_max_err_in_sigma"] <= 4.0, r


def test_served_equals_batched_on_the_same_jobs(jobs):
    """The same six jobs as requests: two at once, the others arriving while
    those run.  Each result is the batched one (and so within the FP64 bars
    above) to FP64 summation order."""
    from nozomi_b200.serve import Server
    specs, tuning, cache, run, sig = jobs
    srv = Server(tuning=tuning, threads=128, cache=cache)
    tickets = [srv.submit(specs[0]), srv.submit(specs[1])]
    srv.round()
    tickets += [srv.submit(sp) for sp in specs[2:4]]
    srv.round()
    tickets += [srv.submit(sp) for sp in specs[4:]]
    srv.drain()
    for i, t in enumerate(tickets):
        assert t.error is None, t.error
        np.testing.assert_allclose(t.signal, sig[i], rtol=0, atol=1e-12)
