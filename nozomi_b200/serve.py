"""Serving: a request loop with continuous batching.

Requests (a ``JobSpec``: substrate, waveform, directions, amplitudes, walkers,
seed) arrive at any time.  The server works in rounds, and a round's GPU work
overlaps the admission of the next requests:

  * admission: waiting requests are taken oldest first while the device
    memory they need (two packed walker states, their share of the
    re-binning scratch, protocol tables) fits the budget.  An admitted
    request's set-up (its substrate's cell lists on a cache miss, seeding,
    packing) runs on a side stream while the current round runs on the
    compute stream; it joins the rounds once that set-up has completed.
    Walker state then stays resident until the request completes;
  * a round: the walkers of every resident request are re-binned in one pass
    (``nz_batch_sort``) and advanced by one chunk in one ``nz_walk_batch``
    launch, each request from its own step.  The chunk is sized so a round
    takes about ``round_s`` seconds at the throughput measured over the last
    rounds (between ``min_steps`` and ``max_steps`` steps), so new requests
    join within about a round whatever the load;
  * requests whose protocol ends in the round have their signal reduced on
    the device and copied to pinned host memory in the same round; the host
    polls the round's completion event (admitting arrivals meanwhile) rather
    than blocking on the stream, then hands those signals back and frees the
    requests' memory.

Draws are keyed by (request seed, walker id, step), so a request's result is
the one it gets alone, whatever the rounds' chunk sizes (tests/test_serve.py).

Memory: with no cache given, the server keeps a SubstrateCache of a quarter
of ``hbm_budget`` for cell lists and admits requests into the other three
quarters, so both together stay within ``hbm_budget`` (the cache may exceed
its share by the one substrate in use).  A cache passed in brings its own
budget; requests then get all of ``hbm_budget``.

Failures stay with their request: a request whose substrate is invalid,
whose target structures have no volume, or whose admission runs out of
device memory completes at once with ``error`` set; ``cancel`` withdraws a
waiting or resident request between rounds; a request with a deadline
(seconds after arrival, a host-side watchdog checked every round) that is
not done by then is cancelled with an error.  The other requests go on.

Overload: with ``max_backlog_s`` set, a request is shed at submission (it
completes at once with ``shed`` and ``error`` set) when the walker-steps
already waiting or resident plus its own would take longer than that at the
throughput of the recent rounds; without it every request waits its turn,
and above the device's throughput the wait grows with the backlog.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import engine
from . import _lib as L
from .batch import JobSpec, SubstrateCache, _items, _job_table, _sort_table, batch_grid, launch_batch, list_groups
from .simulate import Tuning
from .substrates import cell_grid
from .waveforms import step_tables


@dataclass
class Ticket:
    rid: int
    spec: JobSpec
    arrival: float
    admitted: float = None
    completed: float = None
    signal: np.ndarray = None
    error: str = None
    deadline: float = None
    shed: bool = False
    job: dict = field(default=None, repr=False)

    @property
    def latency(self):
        return None if self.completed is None else self.completed - self.arrival


def would_shed(backlog_walker_steps: float, request_walker_steps: float, rate: float | None,
               max_backlog_s: float | None) -> bool:
    """True when the backlog plus the request would take longer than
    max_backlog_s at `rate` walker-steps/s (never before a rate is known,
    nor without a limit)."""
    if max_backlog_s is None or not rate:
        return False
    return (float(backlog_walker_steps) + float(request_walker_steps)) / float(rate) > float(max_backlog_s)


def footprint(spec: JobSpec, tuning: Tuning) -> int:
    """Device bytes a request holds while resident: two packed states (64 B
    per walker each), its share of the one-pass re-binning scratch (a bin
    per walker, histogram and cursor over its (label, bin) keys), its
    protocol tables, directions and amplitudes, and its signal sums."""
    N = int(spec.N)
    nx, ny, nz = cell_grid(spec.substrate.L, tuning.cell)
    c = int(tuning.coarsen)
    keys = (-(-nx // c)) * (-(-ny // c)) * (-(-nz // c)) * (spec.substrate.nstructures + 1 if tuning.by_label else 1)
    ndir = int(np.asarray(spec.dirs).shape[1])
    nb = int(np.asarray(spec.amplitudes).size)
    return 2 * 64 * N + 4 * N + 8 * keys + 8 * spec.nsteps + 4 * (3 * ndir + nb) + 16 * ndir * nb


class Server:
    def __init__(self, tuning: Tuning | None = None, threads: int = 128, hbm_budget: int = 40 << 30,
                 cache: SubstrateCache | None = None, round_s: float = 0.05, min_steps: int = 100,
                 max_steps: int = 4000, max_backlog_s: float | None = None):
        engine.require_cuda()
        self.max_backlog_s = max_backlog_s
        self.tuning = tuning or Tuning()
        self.threads = threads
        if cache is None:
            cache = SubstrateCache(budget_bytes=hbm_budget // 4)
            self.budget = hbm_budget - cache.budget
        else:
            self.budget = hbm_budget
        self.cache = cache
        self.round_s, self.min_steps, self.max_steps = float(round_s), int(min_steps), int(max_steps)
        self.waiting: list[Ticket] = []
        self.staged: list[Ticket] = []   # admitted, set-up in flight on the side stream
        self.active: list[Ticket] = []
        self.done: list[Ticket] = []
        self.used = 0
        self.rounds = 0
        self.walker_steps = 0
        self.next_id = 0
        self.rate = None  # walker-steps/s of recent rounds
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.compute = torch.cuda.current_stream(dev)
        self.side = torch.cuda.Stream(dev)
        self.grids = {lk: batch_grid(threads, lk, self.tuning.stage) for lk in (0, 2, 4)}
        self.queue = torch.zeros(3, dtype=torch.int32, device=dev)
        self.sort_scratch = torch.empty(1, dtype=torch.uint8, device=dev)
        self.clock = time.perf_counter
        self.on_wait = None  # called while a round runs (the request loop submits arrivals there)

    @property
    def resident(self) -> list:
        return self.staged + self.active

    # -- requests ------------------------------------------------------------------
    def submit(self, spec: JobSpec, arrival: float | None = None, deadline_s: float | None = None) -> Ticket:
        """Queue a request; deadline_s: seconds after arrival after which it
        is cancelled if not complete."""
        t = Ticket(self.next_id, spec, self.clock() if arrival is None else arrival)
        if deadline_s is not None:
            t.deadline = t.arrival + float(deadline_s)
        self.next_id += 1
        if self.max_backlog_s is not None and would_shed(self.backlog_walker_steps(), spec.walker_steps, self.rate,
                                                         self.max_backlog_s):
            t.shed = True
            self._fail(t, f"shed: the backlog exceeds {self.max_backlog_s:.3g} s at the current throughput")
            return t
        self.waiting.append(t)
        return t

    def backlog_walker_steps(self) -> int:
        """Walker-steps of the waiting and resident requests still to run."""
        ws = sum(t.spec.walker_steps for t in self.waiting)
        return ws + sum(t.job["N"] * (t.job["nsteps"] - t.job["offset"]) for t in self.resident)

    def _fail(self, t: Ticket, why: str):
        t.error = why
        t.completed = self.clock()
        if t.job is not None:
            self.used -= t.job["bytes"]
            t.job = None
        self.done.append(t)

    def cancel(self, t: Ticket, why: str = "cancelled") -> bool:
        """Withdraw a waiting or resident request (between rounds: none of its
        work is in flight then, except a set-up, which is waited for).
        Returns False if it already completed."""
        if t in self.waiting:
            self.waiting.remove(t)
        elif t in self.staged:
            t.job["ready"].synchronize()
            self.staged.remove(t)
        elif t in self.active:
            self.active.remove(t)
        else:
            return False
        self._fail(t, why)
        return True

    def _watchdog(self):
        now = self.clock()
        for t in [t for t in self.waiting + self.resident if t.deadline is not None and now > t.deadline]:
            self.cancel(t, f"deadline exceeded ({t.deadline - t.arrival:.3g} s after arrival)")

    def _admit(self):
        """Admit waiting requests that fit; their set-up is enqueued on the
        side stream (host work here overlaps the compute stream's round)."""
        while self.waiting:
            t = self.waiting[0]
            need = footprint(t.spec, self.tuning)
            if self.resident and self.used + need > self.budget:
                break
            self.waiting.pop(0)
            sp = t.spec
            try:
                with torch.cuda.stream(self.side):
                    sub = self.cache.get(sp.key if sp.key is not None else id(sp.substrate), sp.substrate, sp.D,
                                         sp.T2, self.tuning)
                    G, Ga = step_tables(sp.gwave)
                    targets = list(range(sub.nstructures + 1)) if sp.targets is None else list(sp.targets)
                    x, lab = engine.seed(sub, targets, sp.N, key=sp.seed ^ 0x5EED)
                    wk = engine.Walkers(x, x.clone(), phi=torch.zeros((6, sp.N), device=self.dev), label=lab)
                    dirs = torch.as_tensor(np.asarray(sp.dirs, np.float32), device=self.dev).contiguous()
                    amps = torch.as_tensor(np.asarray(sp.amplitudes, np.float32).ravel(), device=self.dev)
                    j = {"sub": sub, "G": torch.from_numpy(G).to(self.dev), "Garea": torch.from_numpy(Ga).to(self.dev),
                         "nsteps": int(G.size), "dt": float(sp.gwave.dt), "N": int(sp.N),
                         "draws": engine.philox_draws(sp.seed, 0), "dirs": dirs, "amps": amps,
                         "buf": [engine.FusedState.from_walkers(wk), engine.FusedState(sp.N)], "cur": 0,
                         "offset": 0, "bytes": need,
                         "out": torch.zeros((2, dirs.shape[1], amps.numel()), dtype=torch.float64, device=self.dev),
                         "host_out": torch.empty((2, dirs.shape[1], amps.numel()), dtype=torch.float64,
                                                 pin_memory=True),
                         "ready": torch.cuda.Event()}
                    j["ready"].record(self.side)
            except engine.NozomiError as e:  # a bad request fails alone; the others go on
                self._fail(t, str(e))
                continue
            except torch.cuda.OutOfMemoryError as e:  # so does one whose admission runs out of memory
                self._fail(t, f"out of device memory at admission: {str(e).splitlines()[0]}")
                continue
            t.job = j
            t.admitted = self.clock()
            self.used += need
            self.staged.append(t)

    def _promote(self, wait: bool = False):
        """Staged requests whose set-up has completed join the rounds."""
        for t in list(self.staged):
            if wait:
                t.job["ready"].synchronize()
            if t.job["ready"].query():
                self.staged.remove(t)
                self.active.append(t)

    def _chunk_steps(self, walkers: int) -> int:
        if self.rate is None:
            return int(self.tuning.steps_per_launch)
        k = int(self.round_s * self.rate / max(walkers, 1))
        return max(self.min_steps, min(self.max_steps, k))

    # -- one round -------------------------------------------------------------------
    def round(self):
        """Admit, advance every resident request by one chunk, retire the
        finished ones.  Returns the tickets completed in this round."""
        self._watchdog()
        self._promote()
        if not self.active:
            self._admit()
            self._promote(wait=True)
            if not self.active:
                return []
        lib = L.load()
        jobs = [t.job for t in self.active]
        k = self._chunk_steps(sum(j["N"] for j in jobs))
        stream = ctypes.c_void_p(self.compute.cuda_stream)
        with torch.cuda.stream(self.compute):
            pairs = [(j, j["buf"][j["cur"]], j["buf"][j["cur"] ^ 1]) for j in jobs]
            for j in jobs:
                j["cur"] ^= 1
            sort, n_sort, tw, tk = _sort_table(pairs, self.tuning.coarsen, self.tuning.by_label)
            need = int(lib.nz_batch_sort_scratch_bytes(tw, tk))
            if self.sort_scratch.numel() < need:
                self.sort_scratch = torch.empty(need, dtype=torch.uint8, device=self.dev)
            table = _job_table(jobs, [j["buf"][j["cur"]] for j in jobs])
            plan = self._as_plan(jobs)
            groups = [(lk, _items(plan, grp, self.threads, 0, k))
                      for lk, grp in sorted(list_groups(jobs, range(len(jobs))).items())]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.compute)
            L.check(lib.nz_batch_sort(ctypes.c_void_p(sort.data_ptr()), n_sort, tw, tk,
                                      ctypes.c_void_p(self.sort_scratch.data_ptr()), self.sort_scratch.numel(),
                                      stream), "nz_batch_sort")
            self.queue.zero_()
            for g, (lk, items) in enumerate(groups):
                launch_batch(table, len(jobs), items, lk, 0, k, self.queue.data_ptr() + 4 * g, self.grids[lk],
                             self.threads, self.tuning.stage, stream)
            e1.record(self.compute)
            finished, ws = [], 0
            for t in self.active:
                j = t.job
                adv = min(k, j["nsteps"] - j["offset"])
                ws += adv * j["N"]
                j["offset"] += adv
                if j["offset"] >= j["nsteps"]:
                    j["out"].zero_()
                    j["buf"][j["cur"]].signal(j["dirs"], j["amps"], j["out"])
                    j["host_out"].copy_(j["out"], non_blocking=True)
                    finished.append(t)
            done = torch.cuda.Event()
            done.record(self.compute)
        # while the round runs: admissions (their set-up on the side stream)
        # and, from the request loop, new arrivals
        self._admit()
        while not done.query():
            if self.on_wait is not None:
                self.on_wait()
                self._admit()
            time.sleep(2e-4)
        self.walker_steps += ws
        ms = e0.elapsed_time(e1)
        if ms > 0:
            r = ws / (ms * 1e-3)
            self.rate = r if self.rate is None else 0.5 * (self.rate + r)
        for t in finished:
            s = t.job["host_out"].numpy()
            t.signal = (s[0] + 1j * s[1]) / t.job["N"]
            t.completed = self.clock()
            self.used -= t.job["bytes"]
            t.job = None
            self.active.remove(t)
            self.done.append(t)
        self.rounds += 1
        return finished

    @staticmethod
    def _as_plan(jobs):
        # _items reads nsteps relative to the launch's step0; resident jobs start at their offsets
        return [{"nsteps": j["nsteps"] - j["offset"], "N": j["N"]} for j in jobs]

    def drain(self):
        while self.waiting or self.resident:
            self.round()
        return self.done

    def serve(self, requests, time_limit: float | None = None, deadline_s: float | None = None):
        """Replay a request stream (workloads.Request list, arrival times in
        seconds from now) in real time; returns the completed tickets."""
        start = self.clock()
        pending = sorted(requests, key=lambda r: r.arrival)
        i = 0

        def arrivals():
            nonlocal i
            now = self.clock() - start
            while i < len(pending) and pending[i].arrival <= now:
                self.submit(pending[i].spec, start + pending[i].arrival, deadline_s=deadline_s)
                i += 1

        self.on_wait = arrivals
        try:
            while i < len(pending) or self.waiting or self.resident:
                arrivals()
                if not self.waiting and not self.resident:
                    now = self.clock() - start
                    time.sleep(max(0.0, min(0.01, pending[i].arrival - now)) if i < len(pending) else 0)
                    continue
                self.round()
                if time_limit is not None and self.clock() - start > time_limit:
                    break
        finally:
            self.on_wait = None
        return self.done


def latency_stats(tickets) -> dict:
    lat = np.array([t.latency for t in tickets if t.latency is not None and t.error is None])
    if lat.size == 0:
        return {"n": 0}
    return {"n": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
