"""Serving: a request loop with continuous batching.

Requests (a ``JobSpec``: substrate, waveform, directions, amplitudes, walkers,
seed) arrive at any time.  The server works in rounds.  At the start of a
round it admits waiting requests, oldest first, while the device memory they
need (walker state, re-binning scratch, and the substrate's cell lists unless
already cached) fits the budget; an admitted request's walkers are seeded and
packed on the device and stay resident until it completes.  Then every
resident request is re-binned and advanced by one chunk of steps in a single
``nz_walk_batch`` launch, each from its own step (the job's step offset).
Requests whose protocol is done have their signal reduced on the device and
copied back; their memory is freed for the next admissions.  Work of
requests admitted at different times overlaps on the device from the round
after their admission.

Draws are keyed by (request seed, walker id, step), so a request's result is
the one it gets alone (tests/test_serve.py).

Failures stay with their request: a request whose substrate is invalid,
whose target structures have no volume, or whose admission runs out of
device memory completes at once with ``error`` set; ``cancel`` withdraws a
waiting or resident request between rounds; a request with a deadline
(seconds after arrival, a host-side watchdog checked every round) that is
not done by then is cancelled with an error.  The other requests go on.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import engine
from . import _lib as L
from .batch import JobSpec, SubstrateCache, _job_table, _items
from .simulate import Tuning
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
    job: dict = field(default=None, repr=False)

    @property
    def latency(self):
        return None if self.completed is None else self.completed - self.arrival


def footprint(spec: JobSpec, tuning: Tuning) -> int:
    """Device bytes a request holds while resident: two packed states
    (64 B per walker each), re-binning scratch, its protocol tables."""
    N = spec.N
    return 2 * 64 * N + 4 * N + 8 * (1 << 20) + 8 * spec.nsteps


class Server:
    def __init__(self, tuning: Tuning | None = None, threads: int = 128, hbm_budget: int = 40 << 30,
                 cache: SubstrateCache | None = None):
        engine.require_cuda()
        self.tuning = tuning or Tuning()
        self.threads = threads
        self.budget = hbm_budget
        self.cache = cache or SubstrateCache(budget_bytes=hbm_budget // 4)
        self.waiting: list[Ticket] = []
        self.active: list[Ticket] = []
        self.done: list[Ticket] = []
        self.used = 0
        self.rounds = 0
        self.walker_steps = 0
        self.next_id = 0
        dev = torch.device("cuda", torch.cuda.current_device())
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        occ = ctypes.c_int(0)
        L.check(L.load().nz_batch_occupancy(L.MODE_PHI, threads, ctypes.byref(occ)), "nz_batch_occupancy")
        self.grid = sms * max(1, occ.value)
        self.queue = torch.zeros(1, dtype=torch.int32, device=dev)
        self.clock = time.perf_counter

    # -- requests ------------------------------------------------------------------
    def submit(self, spec: JobSpec, arrival: float | None = None, deadline_s: float | None = None) -> Ticket:
        """Queue a request; deadline_s: seconds after arrival after which it
        is cancelled if not complete."""
        t = Ticket(self.next_id, spec, self.clock() if arrival is None else arrival)
        if deadline_s is not None:
            t.deadline = t.arrival + float(deadline_s)
        self.next_id += 1
        self.waiting.append(t)
        return t

    def _fail(self, t: Ticket, why: str):
        t.error = why
        t.completed = self.clock()
        if t.job is not None:
            self.used -= t.job["bytes"]
            t.job = None
        self.done.append(t)

    def cancel(self, t: Ticket, why: str = "cancelled") -> bool:
        """Withdraw a waiting or resident request (between rounds: none of its
        work is in flight then).  Returns False if it already completed."""
        if t in self.waiting:
            self.waiting.remove(t)
        elif t in self.active:
            self.active.remove(t)
        else:
            return False
        self._fail(t, why)
        return True

    def _watchdog(self):
        now = self.clock()
        for t in [t for t in self.waiting + self.active if t.deadline is not None and now > t.deadline]:
            self.cancel(t, f"deadline exceeded ({t.deadline - t.arrival:.3g} s after arrival)")

    def _admit(self):
        while self.waiting:
            t = self.waiting[0]
            need = footprint(t.spec, self.tuning)
            if self.active and self.used + need > self.budget:
                break
            self.waiting.pop(0)
            sp = t.spec
            try:
                sub = self.cache.get(sp.key if sp.key is not None else id(sp.substrate), sp.substrate, sp.D, sp.T2,
                                     self.tuning)
                G, Ga = step_tables(sp.gwave)
                dev = torch.device("cuda", torch.cuda.current_device())
                targets = list(range(sub.nstructures + 1)) if sp.targets is None else list(sp.targets)
                x, lab = engine.seed(sub, targets, sp.N, key=sp.seed ^ 0x5EED)
                wk = engine.Walkers(x, x.clone(), phi=torch.zeros((6, sp.N), device=dev), label=lab)
                j = {"sub": sub, "G": torch.from_numpy(G).to(dev), "Garea": torch.from_numpy(Ga).to(dev),
                     "nsteps": int(G.size), "dt": float(sp.gwave.dt), "N": int(sp.N),
                     "draws": engine.philox_draws(sp.seed, 0),
                     "dirs": torch.as_tensor(np.asarray(sp.dirs, np.float32), device=dev).contiguous(),
                     "amps": torch.as_tensor(np.asarray(sp.amplitudes, np.float32).ravel(), device=dev),
                     "buf": [engine.FusedState.from_walkers(wk), engine.FusedState(sp.N)], "cur": 0,
                     "scratch": None, "offset": 0, "bytes": need}
            except engine.NozomiError as e:  # a bad request fails alone; the others go on
                self._fail(t, str(e))
                continue
            except torch.cuda.OutOfMemoryError as e:  # so does one whose admission runs out of memory
                self._fail(t, f"out of device memory at admission: {str(e).splitlines()[0]}")
                continue
            t.job = j
            t.admitted = self.clock()
            self.used += need
            self.active.append(t)

    # -- one round -------------------------------------------------------------------
    def round(self):
        """Admit, advance every resident request by one chunk, retire the
        finished ones.  Returns the tickets completed in this round."""
        self._watchdog()
        self._admit()
        if not self.active:
            return []
        k = self.tuning.steps_per_launch
        nl_on = self.tuning.by_label
        jobs = [t.job for t in self.active]
        for j in jobs:
            src, dst = j["buf"][j["cur"]], j["buf"][j["cur"] ^ 1]
            j["scratch"] = src.sort_into(dst, j["sub"].grid, self.tuning.coarsen, j["scratch"],
                                         nlabels=j["sub"].nstructures + 1 if nl_on else 0)
            j["cur"] ^= 1
        table = _job_table(jobs, [j["buf"][j["cur"]] for j in jobs])
        items = _items(self._as_plan(jobs), list(range(len(jobs))), self.threads, 0, k)
        self.queue.zero_()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        L.check(L.load().nz_walk_batch(ctypes.c_void_p(table.data_ptr()), len(jobs), ctypes.c_void_p(items.data_ptr()),
                                       int(items.shape[0]), L.MODE_PHI, 0, k, ctypes.c_void_p(self.queue.data_ptr()),
                                       self.grid, self.threads, stream), "nz_walk_batch")
        finished = []
        for t in self.active:
            j = t.job
            adv = min(k, j["nsteps"] - j["offset"])
            self.walker_steps += adv * j["N"]
            j["offset"] += adv
            if j["offset"] >= j["nsteps"]:
                out = j["buf"][j["cur"]].signal(j["dirs"], j["amps"])
                t.job["out"] = out
                finished.append(t)
        for t in finished:
            s = t.job["out"].cpu().numpy()  # synchronises: the round's work is complete
            t.signal = (s[0] + 1j * s[1]) / t.job["N"]
            t.completed = self.clock()
            self.used -= t.job["bytes"]
            t.job = None
            self.active.remove(t)
            self.done.append(t)
        if not finished:
            torch.cuda.current_stream().synchronize()
        self.rounds += 1
        return finished

    @staticmethod
    def _as_plan(jobs):
        # _items reads nsteps relative to the launch's step0; resident jobs start at their offsets
        return [{"nsteps": j["nsteps"] - j["offset"], "N": j["N"]} for j in jobs]

    def drain(self):
        while self.waiting or self.active:
            self.round()
        return self.done

    def serve(self, requests, time_limit: float | None = None, deadline_s: float | None = None):
        """Replay a request stream (workloads.Request list, arrival times in
        seconds from now) in real time; returns the completed tickets."""
        start = self.clock()
        pending = sorted(requests, key=lambda r: r.arrival)
        i = 0
        while i < len(pending) or self.waiting or self.active:
            now = self.clock() - start
            while i < len(pending) and pending[i].arrival <= now:
                self.submit(pending[i].spec, start + pending[i].arrival, deadline_s=deadline_s)
                i += 1
            if not self.waiting and not self.active:
                time.sleep(max(0.0, min(0.01, pending[i].arrival - now)) if i < len(pending) else 0)
                continue
            self.round()
            if time_limit is not None and self.clock() - start > time_limit:
                break
        return self.done


def latency_stats(tickets) -> dict:
    lat = np.array([t.latency for t in tickets if t.latency is not None and t.error is None])
    if lat.size == 0:
        return {"n": 0}
    return {"n": int(lat.size), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max())}
