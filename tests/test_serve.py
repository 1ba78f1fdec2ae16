"""Serving with continuous batching: requests admitted while others run give
the result they get alone; admission respects the memory budget; a bad
request fails alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _spec(i, na, N, steps, nd, targets=None):
    from nozomi_b200.batch import JobSpec
    from nozomi_b200.substrates import axon_bundle
    from nozomi_b200.workloads import pgse, unit_directions
    rng = np.random.default_rng(50 + i)
    gw = pgse(steps)
    return JobSpec(axon_bundle(na, seed=200 + (i % 3)), gw, unit_directions(rng, nd), gw.amplitude_for_b([0.0, 1.0, 3.0]),
                   N, seed=9000 + i, key=("s", i % 3), targets=targets)


def test_served_equals_alone():
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.serve import Server
    from nozomi_b200.simulate import Tuning
    tuning = Tuning(steps_per_launch=150)
    specs = [_spec(i, na, N, st, nd) for i, (na, N, st, nd) in
             enumerate([(10, 3000, 600, 6), (20, 5000, 400, 9), (15, 2048, 900, 7), (12, 4000, 300, 12),
                        (10, 1000, 750, 8)])]
    # fixed 150-step rounds, so the requests overlap over several rounds
    srv = Server(tuning=tuning, threads=128, min_steps=150, max_steps=150)
    tickets = [srv.submit(specs[0]), srv.submit(specs[1])]
    srv.round()                       # two requests running
    tickets.append(srv.submit(specs[2]))
    srv.round()                       # a third joins mid-way
    tickets += [srv.submit(specs[3]), srv.submit(specs[4])]
    srv.drain()
    assert srv.rounds >= 5 and all(t.completed is not None and t.error is None for t in tickets)
    cache = SubstrateCache()
    for t, sp in zip(tickets, specs):
        alone = BatchRun([sp], tuning=tuning, threads=64, cache=cache).step().signals()[0]
        np.testing.assert_allclose(t.signal, alone, rtol=0, atol=1e-12)
        assert t.latency > 0


def test_admission_by_memory_budget():
    """With a substrate cache of its own budget, requests are admitted into
    all of hbm_budget: two of four fit at once.  Without one, the server's
    own cache takes a quarter and requests the rest."""
    from nozomi_b200.batch import SubstrateCache
    from nozomi_b200.serve import Server, footprint
    from nozomi_b200.simulate import Tuning
    tuning = Tuning(steps_per_launch=200)
    specs = [_spec(i, 10, 4000, 400, 6) for i in range(4)]
    budget = footprint(specs[0], tuning) + footprint(specs[1], tuning) + 1
    srv = Server(tuning=tuning, hbm_budget=budget, cache=SubstrateCache())
    for sp in specs:
        srv.submit(sp)
    peak = 0
    while srv.waiting or srv.resident:
        srv._admit()
        peak = max(peak, len(srv.resident))
        assert srv.used <= budget
        srv.round()
    assert peak == 2 and len(srv.done) == 4
    own = Server(tuning=tuning, hbm_budget=4 * budget)
    assert own.cache.budget == budget and own.budget == 3 * budget


def test_requests_arriving_during_a_round_are_staged_then_served():
    """The request loop admits arrivals while a round runs on the GPU: their
    set-up goes to the side stream, they join a later round, and every result
    equals the request alone (time-bounded rounds, chunk sizes vary)."""
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.serve import Server
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.workloads import Request
    tuning = Tuning(steps_per_launch=200)
    specs = [_spec(i, 10 + 3 * i, 20000, 1500, 6 + i) for i in range(4)]
    srv = Server(tuning=tuning, threads=128, round_s=0.01, min_steps=50)
    staged_seen = []
    real_admit = srv._admit

    def admit():
        real_admit()
        staged_seen.append(len(srv.staged))
    srv._admit = admit
    reqs = [Request(0.0, specs[0]), Request(0.0, specs[1]), Request(0.05, specs[2]), Request(0.1, specs[3])]
    done = srv.serve(reqs)
    assert len(done) == 4 and all(t.error is None for t in done)
    assert max(staged_seen) >= 1 and srv.rounds >= 3
    cache = SubstrateCache()
    for t in done:
        alone = BatchRun([t.spec], tuning=tuning, threads=64, cache=cache).step().signals()[0]
        np.testing.assert_allclose(t.signal, alone, rtol=0, atol=1e-12)


def test_bad_request_fails_alone():
    from nozomi_b200.serve import Server
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.batch import JobSpec
    from nozomi_b200.substrates import Substrate
    from nozomi_b200.workloads import pgse
    gw = pgse(200)
    tiny = Substrate([np.array([[0.0, 0.0, 0.0, 1e-7]])], (10.0, 10.0, 10.0))
    bad = JobSpec(tiny, gw, np.eye(3), [0.0, 1.0], 500, seed=1, targets=[0], key="tiny")
    srv = Server(tuning=Tuning(steps_per_launch=100))
    tb = srv.submit(bad)
    tg = srv.submit(_spec(0, 10, 1000, 200, 6))
    srv.drain()
    assert tb.error is not None and tg.error is None and tg.signal is not None


def test_cancel_deadline_oom_and_invalid_substrate_fail_alone(monkeypatch):
    """Host-side failure injection: a request cancelled while resident, one
    past its deadline, one whose admission runs out of device memory (a fake
    allocation failure) and one with a NaN radius each end with an error; the
    others complete with the result they get alone."""
    from nozomi_b200 import engine
    from nozomi_b200.batch import BatchRun, JobSpec, SubstrateCache
    from nozomi_b200.serve import Server
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.substrates import axon_bundle
    tuning = Tuning(steps_per_launch=100)
    good = [_spec(i, 10, 1500, 400, 6) for i in range(3)]
    victim = _spec(7, 10, 2000, 600, 6)  # same cache key and substrate as good[1]
    late = _spec(8, 10, 1000, 300, 6)
    oom = _spec(9, 10, 1000, 300, 6)
    nan_sub = axon_bundle(10, seed=3)
    f0 = np.array(nan_sub.fibers[0], dtype=np.float64)
    f0[0, 3] = np.nan
    nan_sub.fibers[0] = f0
    nan_req = JobSpec(nan_sub, good[0].gwave, good[0].dirs, good[0].amplitudes, 1000, seed=5, key="nan")
    real_seed = engine.seed

    def seed(sub, targets, N, key, **kw):
        if key == oom.seed ^ 0x5EED:
            raise torch.cuda.OutOfMemoryError("injected: CUDA out of memory")
        return real_seed(sub, targets, N, key, **kw)
    monkeypatch.setattr(engine, "seed", seed)
    srv = Server(tuning=tuning, threads=128)
    tg = [srv.submit(good[0]), srv.submit(victim)]
    srv.round()
    assert srv.cancel(tg[1]) and not srv.cancel(tg[1])
    tl = srv.submit(late, deadline_s=0.0)
    to, tn = srv.submit(oom), srv.submit(nan_req)
    tg += [srv.submit(good[1]), srv.submit(good[2])]
    srv.drain()
    assert tg[1].error == "cancelled"
    assert tl.error.startswith("deadline exceeded")
    assert to.error.startswith("out of device memory at admission")
    assert "non-finite" in tn.error
    assert srv.used == 0 and not srv.active and not srv.waiting
    cache = SubstrateCache()
    for t, sp in zip([tg[0], tg[2], tg[3]], good):
        assert t.error is None
        alone = BatchRun([sp], tuning=tuning, threads=64, cache=cache).step().signals()[0]
        np.testing.assert_allclose(t.signal, alone, rtol=0, atol=1e-12)


def test_overload_sheds_new_requests_and_serves_the_rest():
    """With max_backlog_s, requests arriving while the backlog already needs
    longer than that are shed at once (shed and error set, no device work);
    the others are served and equal their result alone."""
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.serve import Server
    from nozomi_b200.simulate import Tuning
    tuning = Tuning(steps_per_launch=150)
    srv = Server(tuning=tuning, threads=128, min_steps=150, max_steps=150, max_backlog_s=1e-6)
    first = srv.submit(_spec(0, 10, 3000, 600, 6))  # no rate measured yet: admitted
    srv.round()
    assert srv.rate and srv.backlog_walker_steps() > 0
    late = [srv.submit(_spec(i, 12, 4000, 600, 7)) for i in range(1, 4)]  # 1 us of backlog is exceeded
    srv.drain()
    assert first.error is None and not first.shed
    assert all(t.shed and t.error.startswith("shed") and t.signal is None for t in late)
    alone = BatchRun([first.spec], tuning=tuning, threads=64, cache=SubstrateCache()).step().signals()[0]
    np.testing.assert_allclose(first.signal, alone, rtol=0, atol=1e-12)
