"""Batched walk (many substrates and protocols in one persistent launch per
chunk): each job's result equals the same job run alone, the single-substrate
fused path, the plain per-step path (to FP32 phase rounding) and, for
positions, the oracle bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _specs():
    from nozomi_b200.batch import JobSpec
    from nozomi_b200.substrates import axon_bundle
    from nozomi_b200.workloads import pgse, unit_directions
    rng = np.random.default_rng(9)
    specs = []
    for i, (na, N, steps, nd) in enumerate([(10, 3000, 400, 6), (25, 5000, 900, 12), (12, 2000, 250, 9),
                                            (18, 4096, 700, 7)]):
        gw = pgse(steps)
        specs.append(JobSpec(axon_bundle(na, seed=100 + i), gw, unit_directions(rng, nd),
                             gw.amplitude_for_b([0.0, 1.0, 2.5]), N, seed=777 + i, key=("t", i)))
    return specs


@pytest.fixture(scope="module")
def batch_result():
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.simulate import Tuning
    specs = _specs()
    cache = SubstrateCache()
    tuning = Tuning(steps_per_launch=200)
    run = BatchRun(specs, tuning=tuning, threads=128, cache=cache).step()
    return specs, cache, tuning, run, run.signals()


def test_batch_equals_alone(batch_result):
    from nozomi_b200.batch import BatchRun
    specs, cache, tuning, run, sig = batch_result
    for i, sp in enumerate(specs):
        alone = BatchRun([sp], tuning=tuning, threads=64, cache=cache).step().signals()[0]
        np.testing.assert_allclose(alone, sig[i], rtol=0, atol=1e-12)


def test_batch_equals_single_substrate_fused(batch_result):
    from nozomi_b200.simulate import DwiRun
    specs, cache, tuning, run, sig = batch_result
    for i, sp in enumerate(specs):
        dsub = cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning)
        r = DwiRun(dsub, sp.gwave, sp.dirs, sp.amplitudes, sp.N, seed=sp.seed, tuning=tuning).prepare()
        np.testing.assert_allclose(r.walk().signal(), sig[i], rtol=0, atol=1e-12)


def test_batch_equals_plain_path(batch_result):
    from nozomi_b200 import engine
    from nozomi_b200.plain import run_plain
    specs, cache, tuning, run, sig = batch_result
    for i, sp in enumerate(specs[:2]):
        dsub = cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning)
        x, _ = run.positions[i]
        out = run_plain(dsub, sp, x).cpu().numpy()
        np.testing.assert_allclose((out[0] + 1j * out[1]) / sp.N, sig[i], rtol=0, atol=2e-5)


def test_batch_positions_match_oracle(batch_result):
    from nozomi_b200 import engine
    from nozomi_b200.waveforms import step_tables
    from oracle import oracle as oz
    specs, cache, tuning, run, sig = batch_result
    i = 2
    sp = specs[i]
    dsub = cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning)
    st = run.final_state(i)
    N = sp.N
    wk = engine.Walkers(torch.empty((3, N), device="cuda"), torch.empty((3, N), device="cuda"),
                        phi=torch.empty((6, N), device="cuda"))
    st.to_walkers_by_id(wk)
    x0 = run.positions[i][0].cpu().numpy()
    g = oz.Geometry(dsub.spheres.cpu().numpy(), dsub.nstructures, dsub.L, dsub.nseg, dsub.cell_start.cpu().numpy(),
                    dsub.cell_count.cpu().numpy(), dsub.cell_items.cpu().numpy()[:dsub.n_items], dsub.D.cpu().numpy(),
                    dsub.T2.cpu().numpy())
    G, Ga = step_tables(sp.gwave)
    spins, spins0, phi = x0.copy(), x0.copy(), np.zeros((6, N), np.float32)
    oz.walk_f32(g, oz.philox(sp.seed), oz.MODE_PHI, spins, spins0, 0, G.size, sp.gwave.dt, G=G, Garea=Ga, phi=phi)
    np.testing.assert_array_equal(wk.spins.cpu().numpy(), spins)
    np.testing.assert_array_equal(wk.phi.cpu().numpy(), phi)


def test_batch_graph_replay_is_repeatable(batch_result):
    from nozomi_b200.batch import BatchRun
    specs, cache, tuning, run, sig = batch_result
    b = BatchRun(specs, tuning=tuning, threads=128, cache=cache, positions=run.positions)
    b.step()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        b.step()
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        for s, ref in zip(b.signals(), sig):
            np.testing.assert_allclose(s, ref, rtol=0, atol=1e-12)


def test_autotune_small(tmp_path):
    from nozomi_b200.autotune import autotune
    specs = _specs()
    space = {"threads": [64, 128], "cell": [1.0], "near_margin": [0.5, None], "steps_per_launch": [100, 200],
             "coarsen": [4]}
    cache_file = tmp_path / "tune.json"
    t, threads, rep = autotune(specs, space=space, trial_steps=200, max_walkers=2000, max_jobs=2,
                               cache_file=cache_file)
    assert threads in (64, 128) and t.steps_per_launch in (100, 200) and not rep["cached"]
    assert len(rep["trials"]) >= 3
    t2, threads2, rep2 = autotune(specs, space=space, cache_file=cache_file)
    assert rep2["cached"] and threads2 == threads and t2 == t


@pytest.mark.parametrize("threads", [128, 256])
def test_staged_records_equal_global_records(batch_result, threads):
    """nz_walk_batch_staged (each job's records copied into the CTA's shared
    memory when they fit) against the same batch reading its records from
    global memory: signals and every walker's state bit for bit, with the
    capacity between the jobs' record counts so that some jobs are staged
    and some are not; no copy timed out."""
    import dataclasses
    from nozomi_b200 import _lib as L
    from nozomi_b200.batch import BatchRun
    specs, cache, tuning, run, sig = batch_result
    S = sorted(cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning).S for sp in specs)
    assert S[0] < S[-1]
    staged = dataclasses.replace(tuning, stage=S[len(S) // 2])
    ref = BatchRun(specs, tuning=tuning, threads=threads, cache=cache).step()
    got = BatchRun(specs, tuning=staged, threads=threads, cache=cache).step()
    for i in range(len(specs)):
        # the signal sums to FP64 summation order (walkers of one re-binning
        # bin may be stored in any order); every walker's state, by walker id,
        # bit for bit
        np.testing.assert_allclose(got.signals()[i], ref.signals()[i], rtol=0, atol=1e-12)
        a, b = got.final_state(i), ref.final_state(i)
        ia = torch.argsort(a.org[:, 3].view(torch.int32))
        ib = torch.argsort(b.org[:, 3].view(torch.int32))
        for name in ("pos", "org", "phi", "comp"):
            x, y = getattr(a, name)[ia].view(torch.int32), getattr(b, name)[ib].view(torch.int32)
            assert torch.equal(x, y), (i, name)
        flags = a.comp[:, 3].view(torch.int32)
        assert not bool(((flags & L.FLAG_STAGE_TIMEOUT) != 0).any())


def test_staged_batch_refusals():
    """Staging is for index lists and at most MAX_STAGE_RECORDS records."""
    import ctypes
    from nozomi_b200 import _lib as L
    lib = L.load()
    occ = ctypes.c_int(0)
    assert lib.nz_batch_occupancy_staged(L.MODE_PHI | L.LIST_IDX16, 128, 4096, ctypes.byref(occ)) == 0
    assert occ.value >= 1
    assert lib.nz_batch_occupancy_staged(L.MODE_PHI, 128, 4096, ctypes.byref(occ)) != 0  # record lists
    assert lib.nz_batch_occupancy_staged(L.MODE_PHI | L.LIST_IDX16, 128, L.MAX_STAGE_RECORDS + 1,
                                         ctypes.byref(occ)) != 0
