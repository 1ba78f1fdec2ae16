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
    srv = Server(tuning=tuning, threads=128)
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
    from nozomi_b200.serve import Server, footprint
    from nozomi_b200.simulate import Tuning
    tuning = Tuning(steps_per_launch=200)
    specs = [_spec(i, 10, 4000, 400, 6) for i in range(4)]
    budget = footprint(specs[0], tuning) + footprint(specs[1], tuning) + 1
    srv = Server(tuning=tuning, hbm_budget=budget)
    for sp in specs:
        srv.submit(sp)
    peak = 0
    while srv.waiting or srv.active:
        srv._admit()
        peak = max(peak, len(srv.active))
        assert srv.used <= budget
        srv.round()
    assert peak == 2 and len(srv.done) == 4


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
