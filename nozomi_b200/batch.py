"""Batched walk: many (substrate, protocol, walkers) jobs in one persistent
work-queue kernel per chunk of steps, the whole run captured as a CUDA graph.

The reference runs one substrate at a time with one launch per waveform
sample (diffsim3d.py:246-261).  Here every job of a batch advances together:

  * each job's walkers are split into items of `threads` walkers; per chunk
    of ``steps_per_launch`` steps, one launch of ``nz_walk_batch`` runs every
    item of every job that still has steps, CTAs taking items from a queue
    (longest first) until it is empty;
  * between chunks every active job's walkers are re-binned by (label, cell);
  * after the last chunk each job's signal is reduced on the device;
  * draws are keyed by (job seed, walker id, step), so a job's result does not
    depend on what it was batched with (test_batch.py checks alone vs mixed).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import engine
from . import _lib as L
from .simulate import Tuning, device_substrate
from .substrates import Substrate
from .waveforms import step_tables


@dataclass
class JobSpec:
    """One solve: a substrate, a gradient waveform, directions [3, ndir],
    wave amplitudes (units of 100 mT/m), walkers and a seed."""
    substrate: Substrate
    gwave: object
    dirs: np.ndarray
    amplitudes: np.ndarray
    N: int
    seed: int
    D: float = 2.0
    T2: float = 100.0
    targets: list | None = None
    key: object = None      # substrate cache key (default: the substrate object)

    @property
    def nsteps(self) -> int:
        return int(np.asarray(self.gwave.wave).size)

    @property
    def walker_steps(self) -> int:
        return self.N * self.nsteps


class SubstrateCache:
    """Device substrates (cell lists and near lists) kept resident between
    batches, least recently used dropped first beyond ``budget_bytes``.

    Callers without a key of their own pass ``id(substrate)``.  An entry
    therefore holds its host substrate too: while the entry lives the object
    cannot be freed, so its id cannot be reused by another substrate."""

    def __init__(self, budget_bytes: int = 40 << 30):
        self.budget = budget_bytes
        self.items: dict = {}
        self.hosts: dict = {}
        self.order: list = []
        self.hits = 0
        self.misses = 0

    def get(self, key, substrate: Substrate, D, T2, tuning: Tuning) -> engine.DeviceSubstrate:
        k = (key, float(D), float(T2), tuning.cell, tuning.near_margin)
        if k in self.items:
            self.hits += 1
            self.order.remove(k)
            self.order.append(k)
            return self.items[k]
        self.misses += 1
        d = device_substrate(substrate, D=D, T2=T2, cell=tuning.cell, near_margin=tuning.near_margin)
        self.items[k] = d
        self.hosts[k] = substrate
        self.order.append(k)
        while self.nbytes() > self.budget and len(self.order) > 1:
            old = self.order.pop(0)
            del self.items[old]
            del self.hosts[old]
        return d

    def nbytes(self) -> int:
        return sum(d.nbytes() for d in self.items.values())


def _job_table(jobs, states) -> torch.Tensor:
    """nz_job[] on the device (bytes)."""
    arr = (L.Job * len(jobs))()
    for i, (j, st) in enumerate(zip(jobs, states)):
        arr[i].sub = j["sub"].struct()
        arr[i].G = j["G"].data_ptr()
        arr[i].Garea = j["Garea"].data_ptr()
        arr[i].nsteps = j["nsteps"]
        arr[i].dt = np.float32(j["dt"])
        arr[i].draws = j["draws"]
        arr[i].mode = L.MODE_PHI
        arr[i].state = st.struct()
        arr[i].moments = None
        arr[i].step_offset = int(j.get("offset", 0))
    raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
    return torch.from_numpy(raw).cuda()


def _items(jobs, active, threads, s0, k) -> torch.Tensor:
    """Items of the active jobs, longest remaining work first."""
    rows = []
    for j in active:
        steps = min(k, jobs[j]["nsteps"] - s0)
        for first in range(0, jobs[j]["N"], threads):
            rows.append((steps * min(threads, jobs[j]["N"] - first), j, first, min(threads, jobs[j]["N"] - first)))
    rows.sort(key=lambda r: -r[0])
    it = np.array([[r[1], r[2], r[3]] for r in rows], np.int32).reshape(-1, 3)
    return torch.from_numpy(it).cuda()


class BatchRun:
    def __init__(self, specs: list, tuning: Tuning | None = None, threads: int = 128, cache: SubstrateCache | None = None,
                 positions: list | None = None):
        engine.require_cuda()
        self.tuning = tuning or Tuning()
        self.threads = int(threads)
        self.cache = cache or SubstrateCache()
        self.specs = specs
        dev = torch.device("cuda", torch.cuda.current_device())
        self.jobs = []
        for i, sp in enumerate(specs):
            sub = self.cache.get(sp.key if sp.key is not None else id(sp.substrate), sp.substrate, sp.D, sp.T2,
                                 self.tuning)
            G, Ga = step_tables(sp.gwave)
            d = np.asarray(sp.dirs, np.float64)
            self.jobs.append({
                "sub": sub, "G": torch.from_numpy(G).to(dev), "Garea": torch.from_numpy(Ga).to(dev),
                "nsteps": int(G.size), "dt": float(sp.gwave.dt), "N": int(sp.N),
                "draws": engine.philox_draws(sp.seed, 0),
                "dirs": torch.from_numpy(d.astype(np.float32)).to(dev).contiguous(),
                "amps": torch.as_tensor(np.asarray(sp.amplitudes, np.float32).ravel(), device=dev),
                "targets": list(range(sub.nstructures + 1)) if sp.targets is None else list(sp.targets),
                "seed": int(sp.seed),
            })
        self.positions = positions
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        occ = ctypes.c_int(0)
        L.check(L.load().nz_batch_occupancy(L.MODE_PHI, self.threads, ctypes.byref(occ)), "nz_batch_occupancy")
        self.grid = sms * max(1, occ.value)
        self._planned = False

    # -- set-up ------------------------------------------------------------------
    def seed_positions(self):
        """Seed every job's walkers on the device: list of (positions, labels)."""
        out = []
        for j in self.jobs:
            out.append(engine.seed(j["sub"], j["targets"], j["N"], key=j["seed"] ^ 0x5EED))
        return out

    def prepare(self, positions=None):
        """Pack walker state (both ping-pong buffers), plan the chunks and
        upload their job tables and item lists."""
        if positions is None:
            positions = self.positions if self.positions is not None else self.seed_positions()
        self.positions = positions
        for j, (x, lab) in zip(self.jobs, positions):
            if "buf" not in j:  # allocated once: the chunk tables point at these buffers
                j["buf"] = [engine.FusedState(j["N"]), engine.FusedState(j["N"])]
                j["scratch"] = None
            wk = engine.Walkers(x, x.clone(), phi=torch.zeros((6, j["N"]), device=x.device), label=lab)
            j["buf"][0].pack(wk)
            j["cur"] = 0
        if not self._planned:
            self._plan()
        return self

    def _plan(self):
        k = self.tuning.steps_per_launch
        nmax = max(j["nsteps"] for j in self.jobs)
        self.chunks = []
        cur = [0] * len(self.jobs)
        for s0 in range(0, nmax, k):
            active = [i for i, j in enumerate(self.jobs) if j["nsteps"] > s0]
            for i in active:
                cur[i] ^= 1
            states = [self.jobs[i]["buf"][cur[i]] for i in range(len(self.jobs))]
            self.chunks.append({"s0": s0, "s1": s0 + k, "active": active, "table": _job_table(self.jobs, states),
                                "items": _items(self.jobs, active, self.threads, s0, k)})
        self.final_cur = cur
        self.queue = torch.zeros(len(self.chunks), dtype=torch.int32, device="cuda")
        self.out = [torch.zeros((2, j["dirs"].shape[1], j["amps"].numel()), dtype=torch.float64, device="cuda")
                    for j in self.jobs]
        self._planned = True

    # -- the run -------------------------------------------------------------------
    def run(self):
        lib = L.load()
        nl_on = self.tuning.by_label
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        self.queue.zero_()
        for c in self.chunks:
            for i in c["active"]:
                j = self.jobs[i]
                src, dst = j["buf"][j["cur"]], j["buf"][j["cur"] ^ 1]
                j["scratch"] = src.sort_into(dst, j["sub"].grid, self.tuning.coarsen, j["scratch"],
                                             nlabels=j["sub"].nstructures + 1 if nl_on else 0)
                j["cur"] ^= 1
            qi = self.chunks.index(c)
            L.check(lib.nz_walk_batch(ctypes.c_void_p(c["table"].data_ptr()), len(self.jobs),
                                      ctypes.c_void_p(c["items"].data_ptr()), int(c["items"].shape[0]), L.MODE_PHI,
                                      c["s0"], c["s1"], ctypes.c_void_p(self.queue.data_ptr() + 4 * qi), self.grid,
                                      self.threads, stream), "nz_walk_batch")
        for j, out in zip(self.jobs, self.out):
            out.zero_()
            j["buf"][j["cur"]].signal(j["dirs"], j["amps"], out)
        return self

    def step(self):
        """prepare + run: one pass of the batch from its initial positions."""
        return self.prepare().run()

    def launches(self) -> int:
        """Library kernels of one step (prepare + run): a pack per job; per
        chunk each active job's re-binning (FusedState.sort_kernels) and one
        batched walk; a signal per job."""
        nl_on = self.tuning.by_label
        n = sum(1 for j in self.jobs if j["N"]) * 2  # pack and signal
        for c in self.chunks:
            for i in c["active"]:
                j = self.jobs[i]
                n += j["buf"][0].sort_kernels(j["sub"].grid, self.tuning.coarsen,
                                              j["sub"].nstructures + 1 if nl_on else 0)
            n += 1 if c["items"].shape[0] else 0
        return n

    def signals(self) -> list:
        res = []
        for j, out in zip(self.jobs, self.out):
            s = out.cpu().numpy()
            res.append((s[0] + 1j * s[1]) / j["N"])
        return res

    def walker_steps(self) -> int:
        return sum(j["N"] * j["nsteps"] for j in self.jobs)

    def final_state(self, i: int) -> engine.FusedState:
        return self.jobs[i]["buf"][self.final_cur[i]]
