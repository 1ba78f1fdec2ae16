"""Sharding over processes: walker ranges, job assignment, the one exchange
(a sum of signal sums) over a world-size-2 gloo process group on the CPU with
the oracle as each rank's walker, a rank that fails between steps, and, on the
GPU, shards walked one after another against the unsharded fused run."""
import os
import socket
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partitions():
    from nozomi_b200.shard import shard_range
    for N in (0, 1, 7, 1000, 1001, 999_999):
        for world in (1, 2, 3, 8):
            parts = [shard_range(N, world, r) for r in range(world)]
            assert parts[0][0] == 0
            for (f0, c0), (f1, _) in zip(parts, parts[1:]):
                assert f0 + c0 == f1
            assert sum(c for _, c in parts) == N
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_shard_jobs_balanced():
    from nozomi_b200.shard import shard_jobs
    rng = np.random.default_rng(3)
    costs = np.exp(rng.uniform(np.log(1e4), np.log(1e7), 64))
    for world in (1, 2, 4, 8):
        a = shard_jobs(costs, world)
        assert sorted(j for r in a for j in r) == list(range(costs.size))
        loads = [costs[r].sum() for r in a]
        assert max(loads) - min(loads) <= costs.max()  # greedy LPT bound
        assert a == shard_jobs(costs, world)  # deterministic: every rank computes the same


def _oracle_problem():
    from nozomi_b200.substrates import beaded_axon
    from nozomi_b200.waveforms import PGDiffWaveform, step_tables
    from oracle import oracle as oz
    sub = beaded_axon()
    sph = sub.spheres()
    nseg = (1, 1, 8)
    st, ct, it = oz.cells(sph, sub.L, nseg)
    g = oz.Geometry(sph.astype(np.float32), sub.nstructures, sub.L, nseg, st, ct, it,
                    np.full(2, 2.0, np.float32), np.full(2, 100.0, np.float32))
    pg = PGDiffWaveform(5.0, 2.0, 3.5, time_step=0.01)
    G, Ga = step_tables(pg)
    dirs = np.array([[1.0, 0.0, 0.6], [0.0, 0.0, 0.0], [0.0, 1.0, 0.8]])
    amps = np.array([0.0, 1.0, 2.0, 3.0])
    return g, G, Ga, pg.dt, dirs, amps


def _oracle_shard(g, G, Ga, dt, dirs, amps, N, key, first, count):
    """Seed and walk walkers [first, first + count) with the oracle; returns
    positions [3, count] and signal sums [2, ndir, nb]."""
    from oracle import oracle as oz
    x, lab, left = oz.seed(g, [0], count, key ^ 0x5EED, id0=first)
    assert left == 0
    sp, s0, phi = x.copy(), x.copy(), np.zeros((6, count), np.float32)
    oz.walk_f32(g, oz.philox(key, id0=first), oz.MODE_PHI, sp, s0, 0, G.size, dt, G=G, Garea=Ga, phi=phi)
    S = oz.signal_phi(phi, dirs, amps) * count
    return sp, np.stack([S.real, S.imag])


def _gloo_rank(rank, world, port, out_dir, N, key):
    import torch.distributed as dist
    from nozomi_b200.shard import reduce_sums, shard_range
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from nozomi_b200.shard import init_process_group
    init_process_group("gloo", timeout_s=60)
    first, count = shard_range(N, world, rank)
    prob = _oracle_problem()
    sp, sums = _oracle_shard(*prob, N, key, first, count)
    t = torch.from_numpy(sums.copy())
    reduce_sums(t)
    parts = [None] * world
    dist.all_gather_object(parts, (first, sp))
    if rank == 0:
        pos = np.concatenate([p for _, p in sorted(parts, key=lambda q: q[0])], axis=1)
        np.savez(os.path.join(out_dir, "sharded.npz"), sums=t.numpy(), pos=pos)
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_walk_equals_unsharded_gloo(tmp_path):
    """Two gloo ranks, each the oracle walking its walker range: positions
    are the unsharded run's bit for bit and the all-reduced signal sums equal
    the unsharded sums to FP64 summation order."""
    import torch.multiprocessing as mp
    N, key, world = 600, 77, 2
    mp.start_processes(_gloo_rank, args=(world, _free_port(), str(tmp_path), N, key), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / "sharded.npz")
    g, G, Ga, dt, dirs, amps = _oracle_problem()
    sp, sums = _oracle_shard(g, G, Ga, dt, dirs, amps, N, key, 0, N)
    np.testing.assert_array_equal(got["pos"], sp)
    np.testing.assert_allclose(got["sums"], sums, rtol=0, atol=1e-9 * N)
    # and not trivially: a different key moves the walkers
    sp2, _ = _oracle_shard(g, G, Ga, dt, dirs, amps, 50, key + 1, 0, 50)
    assert not np.array_equal(sp2, sp[:, :50])


def _failing_rank(rank, world, port, out_dir):
    import torch.distributed as dist
    from nozomi_b200.shard import AbortFlag, ShardAborted, init_process_group, reduce_sums
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    init_process_group("gloo", timeout_s=5)
    flag = AbortFlag(dist.distributed_c10d._get_default_store())
    outcome = "completed"
    t0 = time.monotonic()
    try:
        for step in range(3):
            t = torch.full((4,), float(rank + 1), dtype=torch.float64)  # the step's partial sums
            if rank == 1 and step == 1:
                flag.raise_abort(rank, "injected failure between steps")
                raise RuntimeError("injected failure")
            if rank == 0 and step == 1:
                time.sleep(0.5)  # rank 1 fails while rank 0 is still in the step's local work
            flag.check()
            reduce_sums(t)
            assert float(t[0]) == 3.0
    except ShardAborted as e:
        outcome = f"aborted: {e}"
    except RuntimeError as e:
        outcome = f"error: {e}"
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{outcome}\n{time.monotonic() - t0:.3f}\n")
    # no barrier and no destroy: the other rank has left


def test_rank_failure_between_steps_gloo(tmp_path):
    """A rank fails between steps and raises the store flag: the other rank
    learns of it before its next collective and stops with ShardAborted, in
    bounded time, instead of waiting in the all-reduce."""
    import torch.multiprocessing as mp
    mp.start_processes(_failing_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = (tmp_path / "rank0.txt").read_text().split("\n")
    r1 = (tmp_path / "rank1.txt").read_text().split("\n")
    assert r1[0].startswith("error: injected failure")
    assert r0[0].startswith("aborted: rank 1: injected failure between steps"), r0
    assert float(r0[1]) < 30


@pytest.mark.gpu
def test_sharded_gpu_equals_unsharded():
    """Shards of a fused run walked one after another on one GPU (the ranks'
    work without a process group; their sums added on the host) against the
    unsharded run: positions bit for bit, signal to FP64 summation order."""
    from nozomi_b200.shard import ShardedDwiRun
    from nozomi_b200.simulate import DwiRun, Tuning, device_substrate
    from nozomi_b200.substrates import axon_bundle
    from nozomi_b200.workloads import pgse, unit_directions
    sub = axon_bundle(12, seed=5)
    tuning = Tuning(steps_per_launch=150)
    dsub = device_substrate(sub, D=2.0, cell=tuning.cell, near_margin=tuning.near_margin)
    gw = pgse(400)
    dirs = unit_directions(np.random.default_rng(2), 6)
    amps = gw.amplitude_for_b([0.0, 1.0, 3.0])
    N, seed = 10_001, 42
    full = DwiRun(dsub, gw, dirs, amps, N, seed=seed, tuning=tuning).prepare().walk()
    ref_sig = full.signal()
    ref_pos = full.walkers().spins.cpu().numpy()
    for world in (2, 3):
        sums, pos = 0, []
        for rank in range(world):
            sh = ShardedDwiRun(dsub, gw, dirs, amps, N, seed=seed, rank=rank, world=world, tuning=tuning)
            sh.prepare().walk()
            sums = sums + sh.local_sums().cpu().numpy()
            pos.append(sh.run.walkers().spins.cpu().numpy())
        np.testing.assert_array_equal(np.concatenate(pos, axis=1), ref_pos)
        np.testing.assert_allclose((sums[0] + 1j * sums[1]) / N, ref_sig, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_prepare_from_host_buffers_equals_device_buffers():
    """prepare() given the seeded positions and labels as pinned host tensors
    and as numpy arrays (the end-to-end call's inputs) walks to the same
    positions and sums, bit for bit, as given the device tensors."""
    import torch
    from nozomi_b200.shard import ShardedDwiRun
    from nozomi_b200.simulate import Tuning, device_substrate
    from nozomi_b200.substrates import axon_bundle
    from nozomi_b200.workloads import pgse, unit_directions
    sub = axon_bundle(12, seed=5)
    tuning = Tuning(steps_per_launch=150)
    dsub = device_substrate(sub, D=2.0, cell=tuning.cell, near_margin=tuning.near_margin)
    gw = pgse(400)
    dirs = unit_directions(np.random.default_rng(2), 6)
    amps = gw.amplitude_for_b([0.0, 1.0, 3.0])
    sh = ShardedDwiRun(dsub, gw, dirs, amps, 8_193, seed=7, rank=1, world=2, tuning=tuning)
    x0, lab0 = sh.run.initial_positions()
    ref = sh.prepare(x0, lab0).walk().local_sums().cpu().numpy()
    ref_pos = sh.run.walkers().spins.cpu().numpy()
    for x, lab in ((x0.cpu().pin_memory(), lab0.cpu().pin_memory()), (x0.cpu().numpy(), lab0.cpu().numpy())):
        got = sh.prepare(x, lab).walk().local_sums().cpu().numpy()
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_array_equal(sh.run.walkers().spins.cpu().numpy(), ref_pos)
    with pytest.raises(TypeError):
        sh.prepare(x0.cpu()[:2], lab0.cpu())
    with pytest.raises(TypeError):
        sh.prepare(x0.cpu(), lab0.cpu()[:-1])


def test_oracle_seed_range_is_a_slice_of_the_full_seeding():
    """Walkers [id0, id0 + n) seeded alone are walkers id0.. of one seeding of
    the whole run (positions and labels), the property sharded runs rest on."""
    from oracle import oracle as oz
    g = _oracle_problem()[0]
    full, lab, left = oz.seed(g, [0, 1], 900, 4321)
    assert left == 0
    for id0, n in ((0, 300), (300, 250), (550, 350)):
        part, plab, pleft = oz.seed(g, [0, 1], n, 4321, id0=id0)
        assert pleft == 0
        np.testing.assert_array_equal(part, full[:, id0:id0 + n])
        np.testing.assert_array_equal(plab, lab[id0:id0 + n])
