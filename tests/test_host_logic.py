"""Host logic that needs no GPU: the synthetic workload generators (seeded,
within their stated ranges), the serving loop's memory footprint and latency
statistics, and the autotuner's workload signature."""
import numpy as np
import pytest

pytest.importorskip("torch")


def _small_specs(seed=4, n=5):
    from nozomi_b200.workloads import mixed_specs
    return mixed_specs(seed=seed, n_jobs=n, axons=(10, 14), walkers=(1e4, 1e5), steps=(2000, 3000))


def test_mixed_specs_seeded_and_in_range():
    a, b = _small_specs(), _small_specs()
    for x, y in zip(a, b):
        assert (x.N, x.nsteps, x.seed, x.key) == (y.N, y.nsteps, y.seed, y.key)
        np.testing.assert_array_equal(x.dirs, y.dirs)
        assert 1e4 <= x.N <= 1e5 and x.N % 1000 == 0
        assert 2000 <= x.nsteps <= 3000
        assert 6 <= x.dirs.shape[1] <= 60
        np.testing.assert_allclose(np.linalg.norm(x.dirs, axis=0), 1.0, atol=1e-12)
        assert x.amplitudes[0] == 0.0 and np.all(np.diff(x.amplitudes) > 0)
        assert 10 <= x.substrate.nstructures <= 14
    assert [s.seed for s in _small_specs(seed=5)] != [s.seed for s in a]


def test_request_stream_poisson_and_reuse():
    from nozomi_b200.workloads import request_stream
    reqs = request_stream(50.0, 4.0, seed=5, axons=(10, 12), walkers=(1e4, 2e4), steps=(2000, 2100))
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 4.0
    assert 120 <= len(reqs) <= 280  # 200 expected at 50 req/s over 4 s
    keys = [r.spec.key for r in reqs]
    reused = sum(1 for i, k in enumerate(keys) if k in keys[:i])
    assert 0.5 < reused / len(keys) < 0.9  # substrates drawn again with probability 0.7
    again = request_stream(50.0, 4.0, seed=5, axons=(10, 12), walkers=(1e4, 2e4), steps=(2000, 2100))
    assert [r.arrival for r in again] == list(t) and [r.spec.N for r in again] == [r.spec.N for r in reqs]
    capped = request_stream(50.0, 4.0, seed=5, axons=(10, 12), walkers=(1e4, 2e4), steps=(2000, 2100),
                            max_requests=7)
    assert len(capped) == 7


def test_serving_footprint_and_latency_stats():
    from nozomi_b200.serve import Ticket, footprint, latency_stats
    from nozomi_b200.simulate import Tuning
    specs = _small_specs(n=2)
    small, big = sorted(specs, key=lambda s: s.N)
    assert footprint(big, Tuning()) > footprint(small, Tuning()) > 2 * 64 * small.N
    tickets = []
    for i, lat in enumerate(np.linspace(0.1, 1.0, 100)):
        t = Ticket(i, small, arrival=10.0)
        t.completed = 10.0 + lat
        tickets.append(t)
    failed = Ticket(100, small, arrival=0.0)
    failed.completed, failed.error = 50.0, "cancelled"
    st = latency_stats(tickets + [failed])
    assert st["n"] == 100
    assert abs(st["p50_s"] - 0.55) < 1e-9 and abs(st["max_s"] - 1.0) < 1e-12
    assert 0.98 < st["p99_s"] <= 1.0
    assert latency_stats([failed]) == {"n": 0}


def test_autotune_signature():
    from nozomi_b200.autotune import signature
    a = _small_specs()
    assert signature(a) == signature(_small_specs())
    b = _small_specs()
    b[0] = __import__("dataclasses").replace(b[0], N=b[0].N * 50)
    assert signature(b) != signature(a)


def test_rebinning_kernel_count_follows_the_scan_threshold():
    """The launch counts bench.py reports: a re-binning launches bin count,
    scan and scatter, the scan as three kernels above SCAN_SINGLE_KEYS bins
    (the mirror of kScanSingle in csrc/kernels.cuh), none for no walkers."""
    import re
    from pathlib import Path
    from nozomi_b200 import _lib as L
    from nozomi_b200.engine import FusedState, box_grid
    src = (Path(__file__).resolve().parents[1] / "nozomi_b200" / "csrc" / "kernels.cuh").read_text()
    assert int(re.search(r"kScanSingle = (\d+);", src).group(1)) == L.SCAN_SINGLE_KEYS
    st = object.__new__(FusedState)  # only N is read: no device buffers needed
    st.N = 1000
    packed = box_grid((40.0, 40.0, 80.0), (80, 80, 160))  # 0.5 um cells of the packed box
    assert FusedState.sort_bins(packed, 8) == 10 * 10 * 20
    assert st.sort_kernels(packed, 8) == 3
    assert FusedState.sort_bins(packed, 8, nlabels=201) == 402_000
    assert st.sort_kernels(packed, 8, nlabels=201) == 5
    edge = box_grid((32.0, 32.0, 32.0), (32, 32, 32))
    assert FusedState.sort_bins(edge, 1) == L.SCAN_SINGLE_KEYS and st.sort_kernels(edge, 1) == 3
    assert st.sort_kernels(edge, 1, nlabels=2) == 5
    st.N = 0
    assert st.sort_kernels(packed, 8, nlabels=201) == 0


def test_substrate_cache_lru_and_id_keys(monkeypatch):
    """The device-substrate cache: hits, least-recently-used eviction beyond
    its budget, and id()-keyed entries that keep their host substrate alive
    (so a freed substrate's id cannot alias a new one while cached)."""
    import gc
    import weakref
    from nozomi_b200 import batch
    from nozomi_b200.simulate import Tuning

    class FakeDevice:
        def nbytes(self):
            return 100

    monkeypatch.setattr(batch, "device_substrate", lambda sub, **kw: FakeDevice())

    class Sub:
        pass

    cache = batch.SubstrateCache(budget_bytes=250)
    t = Tuning()
    a, b, c = Sub(), Sub(), Sub()
    da = cache.get(id(a), a, 2.0, 100.0, t)
    assert cache.get(id(a), a, 2.0, 100.0, t) is da and (cache.hits, cache.misses) == (1, 1)
    assert cache.get(id(a), a, 1.0, 100.0, t) is not da  # another D is another entry
    ref = weakref.ref(a)
    del a
    gc.collect()
    assert ref() is not None  # held by the cache while its entry lives
    cache.get(id(b), b, 2.0, 100.0, t)  # third entry: 300 bytes > 250, the oldest goes
    assert len(cache.items) == 2 and cache.nbytes() == 200
    cache.get(id(c), c, 2.0, 100.0, t)
    gc.collect()
    assert ref() is None  # both of a's entries evicted: a is freed
    assert set(cache.items) == set(cache.hosts)


def test_autotune_choice_cache_is_robust(tmp_path):
    """The autotuner's per-(GPU, workload) cache: a stored choice reads back
    as the same Tuning; a corrupt file, a missing signature or an entry with
    unknown Tuning fields is a miss, not an error; stores keep other entries."""
    import dataclasses
    from nozomi_b200.autotune import cached_choice, load_choices, store_choice
    from nozomi_b200.simulate import Tuning
    p = tmp_path / "sub" / "autotune.json"
    assert cached_choice(p, "abc") is None
    t = Tuning(cell=0.5, near_margin=None, steps_per_launch=2000, coarsen=8)
    store_choice(p, "abc", {"tuning": dataclasses.asdict(t), "threads": 128, "trial_walker_steps_per_s": 1e10})
    store_choice(p, "def", {"tuning": {"no_such_field": 1}, "threads": 64})
    got = cached_choice(p, "abc")
    assert got is not None and got[0] == t and got[1] == 128
    assert cached_choice(p, "def") is None and cached_choice(p, "zzz") is None
    assert set(load_choices(p)) == {"abc", "def"}
    assert not list(p.parent.glob("*.tmp"))
    p.write_text('{"abc": {"tuning": ')  # a torn write by an older version
    assert load_choices(p) == {} and cached_choice(p, "abc") is None


def _store_many(path, tag, n):
    from nozomi_b200.autotune import store_choice
    for i in range(n):
        store_choice(path, f"{tag}-{i}", {"tuning": {}, "threads": 128})


def test_autotune_stores_from_several_processes_keep_every_entry(tmp_path):
    """Four processes each store 15 different signatures into one cache file
    at the same time: the locked read-modify-write keeps all 60 entries and
    leaves no temporary or half-written file."""
    import multiprocessing as mp
    from nozomi_b200.autotune import load_choices
    ctx = mp.get_context("spawn")
    p = tmp_path / "autotune.json"
    procs = [ctx.Process(target=_store_many, args=(str(p), f"p{k}", 15)) for k in range(4)]
    for q in procs:
        q.start()
    for q in procs:
        q.join(120)
        assert q.exitcode == 0
    assert set(load_choices(p)) == {f"p{k}-{i}" for k in range(4) for i in range(15)}
    assert not list(tmp_path.glob("*.tmp"))


def _build_bundle(cache_dir, out):
    import os
    os.environ["NOZOMI_B200_CACHE"] = cache_dir
    import numpy as np
    from nozomi_b200 import workloads
    s = workloads.bundle(12, 5)
    np.save(out, s.spheres())


def test_cached_substrate_built_by_several_processes_at_once(tmp_path):
    """Ranks of one job build the same cached substrate at the same time on a
    fresh machine: every process gets the same substrate, the cache ends with
    one complete file and no temporary files."""
    import multiprocessing as mp
    import numpy as np
    ctx = mp.get_context("spawn")
    cache = tmp_path / "cache"
    procs = [ctx.Process(target=_build_bundle, args=(str(cache), str(tmp_path / f"s{i}.npy"))) for i in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    arrs = [np.load(tmp_path / f"s{i}.npy") for i in range(3)]
    assert all(np.array_equal(a, arrs[0]) for a in arrs[1:])
    assert len(list(cache.glob("bundle_*.pkl"))) == 1 and not list(cache.glob("*.tmp"))


def test_record_order_of_the_index_lists():
    """The index form's records: spheres sorted by structure (stable), the
    first record of each structure, each sphere's record; an empty substrate
    still gets one-row arrays."""
    import numpy as np
    from nozomi_b200.engine import record_order
    sid = np.array([2, 0, 1, 0, 2, 1, 0], np.float64)
    sph = np.vstack([np.arange(7) * 1.0, np.arange(7) * 2.0, np.arange(7) * 3.0, np.full(7, 0.5), sid])
    rec4, rec_sid, sid_start, perm = record_order(sph, 3)
    np.testing.assert_array_equal(rec_sid, [0, 0, 0, 1, 1, 2, 2])
    np.testing.assert_array_equal(sid_start, [0, 3, 5, 7, 7])
    np.testing.assert_array_equal(rec4[:, 0], [1, 3, 6, 2, 5, 0, 4])
    for s in range(7):
        np.testing.assert_array_equal(rec4[perm[s]], sph[:4, s].astype(np.float32))
    rec4, rec_sid, sid_start, perm = record_order(np.zeros((5, 0)), 0)
    assert rec4.shape == (1, 4) and rec_sid.shape == (1,) and perm.shape == (1,)
    np.testing.assert_array_equal(sid_start, [0, 0])


def test_stream_substrates_generated_in_workers_equal_in_process(tmp_path, monkeypatch):
    """Substrates generated by spawned worker processes (then read back from
    the disk cache) equal the ones generated in this process; requests of one
    substrate share one object."""
    from nozomi_b200 import workloads
    keys = [(10, 11), (11, 12), (10, 13), (10, 11)]
    monkeypatch.setenv("NOZOMI_B200_CACHE", str(tmp_path / "w"))
    monkeypatch.setattr(workloads, "CACHE", tmp_path / "w")
    par = workloads.bundles(keys, workers=2)
    monkeypatch.setenv("NOZOMI_B200_CACHE", str(tmp_path / "s"))
    monkeypatch.setattr(workloads, "CACHE", tmp_path / "s")
    seq = workloads.bundles(keys, workers=1)
    assert sorted(par) == sorted(seq) == sorted(set(keys))
    for k in seq:
        np.testing.assert_array_equal(par[k].spheres(), seq[k].spheres())
    reqs = workloads.request_stream(40.0, 2.0, seed=3, axons=(10, 11), walkers=(1e4, 2e4), steps=(2000, 2100))
    by_key = {}
    for r in reqs:
        assert by_key.setdefault(r.spec.key, r.spec.substrate) is r.spec.substrate


def test_shedding_rule():
    """A request is shed when backlog plus request exceed the limit at the
    measured rate; never without a limit or before a rate is known."""
    from nozomi_b200.serve import would_shed
    assert not would_shed(1e12, 1e9, None, 1.0)       # no rate yet
    assert not would_shed(1e12, 1e9, 1e10, None)      # no limit
    assert not would_shed(4e9, 1e9, 1e10, 1.0)        # 0.5 s of work
    assert would_shed(1e10, 1e9, 1e10, 1.0)           # 1.1 s of work
    assert not would_shed(9e9, 1e9, 1e10, 1.0)       # exactly 1 s: kept


def test_batch_item_table_covers_every_walker_longest_first():
    """Each active job's walkers in runs of at most `threads`, every walker
    once; items ordered by remaining work (walkers x this chunk's steps,
    clamped to the job), ties in job then walker order; inactive jobs and
    empty activity give no items."""
    from nozomi_b200.batch import item_table
    jobs = [{"N": 1000, "nsteps": 3000}, {"N": 300, "nsteps": 800}, {"N": 129, "nsteps": 5000},
            {"N": 5000, "nsteps": 100}]
    it = item_table(jobs, [0, 1, 2], 128, 500, 1000)
    assert it.dtype == np.int32 and it.shape[1] == 3
    for j in (0, 1, 2):
        mine = it[it[:, 0] == j]
        cover = np.zeros(jobs[j]["N"], int)
        for _, first, count in mine:
            assert 1 <= count <= 128
            cover[first:first + count] += 1
        assert (cover == 1).all()
    assert not (it[:, 0] == 3).any()
    steps = np.minimum(1000, np.array([jobs[j]["nsteps"] - 500 for j in it[:, 0]]))
    work = steps * it[:, 2]
    assert (np.diff(work) <= 0).all()
    for i in range(len(it) - 1):  # ties keep job, then walker order
        if work[i] == work[i + 1]:
            assert (it[i, 0], it[i, 1]) < (it[i + 1, 0], it[i + 1, 1])
    assert item_table(jobs, [], 128, 0, 100).shape == (0, 3)
