"""Batched walk: many (substrate, protocol, walkers) jobs in one persistent
work-queue kernel per chunk of steps, the whole run captured as a CUDA graph.

The reference runs one substrate at a time with one launch per waveform
sample (diffsim3d.py:246-261).  Here every job of a batch advances together:

  * each job's walkers are split into items of `threads` walkers; per chunk
    of ``steps_per_launch`` steps, one launch of ``nz_walk_batch`` runs every
    item of every job that still has steps, CTAs taking items from a queue
    (longest first) until it is empty;
  * before every chunk the walkers of all its jobs are re-binned by (label,
    cell) in one pass (``nz_batch_sort``: one bin count, one scan, one
    scatter over every job's walkers);
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
        k = (key, float(D), float(T2), tuning.cell, tuning.near_margin, tuning.lists, tuning.near_shape)
        if k in self.items:
            self.hits += 1
            self.order.remove(k)
            self.order.append(k)
            return self.items[k]
        self.misses += 1
        d = device_substrate(substrate, D=D, T2=T2, cell=tuning.cell, near_margin=tuning.near_margin,
                             lists=tuning.lists, near_shape=tuning.near_shape)
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


def _sort_table(pairs, coarsen, by_label):
    """nz_sort_job[] of one chunk's re-binning (bytes on the device), with
    the total walker and key counts.  pairs: (job dict, source state,
    destination state) of every active job."""
    lib = L.load()
    arr = (L.SortJob * max(1, len(pairs)))()
    tw = tk = 0
    for i, (j, src, dst) in enumerate(pairs):
        g = j["sub"].grid
        nl = j["sub"].nstructures + 1 if by_label else 0
        keys = int(lib.nz_sort_job_keys(L.byref(g), int(coarsen), nl))
        if keys <= 0:
            raise L.NozomiError(f"re-binning: bad grid or coarsening for job {i}")
        arr[i].inp, arr[i].out = src.struct(), dst.struct()
        arr[i].grid = g
        arr[i].coarsen, arr[i].nlabels = int(coarsen), nl
        arr[i].walker_offset, arr[i].key_offset = tw, tk
        tw += src.N
        tk += keys
    if tw >= 2 ** 31 or tk >= 2 ** 31:
        raise L.NozomiError(f"re-binning: {tw} walkers / {tk} keys in one chunk exceed the int range")
    raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
    return torch.from_numpy(raw).cuda(), len(pairs), tw, tk


LIST_BITS = {0: 0, 2: L.LIST_IDX16, 4: L.LIST_IDX32}


def list_groups(jobs, active) -> dict:
    """Active jobs by the list form of their substrate (idx_bytes): one
    batched launch per form."""
    groups = {}
    for i in active:
        groups.setdefault(jobs[i]["sub"].idx_bytes, []).append(i)
    return groups


def batch_grid(threads: int, lk: int, stage: int = 0) -> int:
    """Persistent grid of the batched walk: CTAs resident per SM x SMs
    (with `stage` records of shared memory per CTA for index lists)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    occ = ctypes.c_int(0)
    lib = L.load()
    if stage and lk:
        L.check(lib.nz_batch_occupancy_staged(L.MODE_PHI | LIST_BITS[lk], int(threads), int(stage),
                                              ctypes.byref(occ)), "nz_batch_occupancy_staged")
    else:
        L.check(lib.nz_batch_occupancy(L.MODE_PHI | LIST_BITS[lk], int(threads), ctypes.byref(occ)),
                "nz_batch_occupancy")
    return sms * max(1, occ.value)


def launch_batch(table, n_jobs: int, items, lk: int, s0: int, s1: int, queue_ptr: int, grid: int, threads: int,
                 stage: int, stream) -> None:
    """One batched walk launch over `items` (list form lk): nz_walk_batch, or
    nz_walk_batch_staged when `stage` records per CTA are staged (index lists
    only; record lists are never staged)."""
    lib = L.load()
    args = (ctypes.c_void_p(table.data_ptr()), int(n_jobs), ctypes.c_void_p(items.data_ptr()), int(items.shape[0]),
            L.MODE_PHI | LIST_BITS[lk], int(s0), int(s1), ctypes.c_void_p(queue_ptr), int(grid), int(threads))
    if stage and lk:
        L.check(lib.nz_walk_batch_staged(*args, int(stage), stream), "nz_walk_batch_staged")
    else:
        L.check(lib.nz_walk_batch(*args, stream), "nz_walk_batch")


def item_table(jobs, active, threads, s0, k) -> np.ndarray:
    """[n, 3] int32 items (job, first walker, count) of the active jobs: each
    job's walkers in runs of at most `threads`, longest remaining work
    (walkers x steps of this chunk, [s0, s0 + k) clamped to the job) first,
    ties in job, then walker order."""
    parts, work = [], []
    for j in active:
        N = int(jobs[j]["N"])
        steps = min(k, jobs[j]["nsteps"] - s0)
        first = np.arange(0, N, threads, dtype=np.int64)
        count = np.minimum(threads, N - first)
        parts.append(np.stack([np.full(first.size, j), first, count], axis=1))
        work.append(steps * count)
    if not parts:
        return np.zeros((0, 3), np.int32)
    it, w = np.concatenate(parts), np.concatenate(work)
    return np.ascontiguousarray(it[np.argsort(-w, kind="stable")].astype(np.int32))


def _items(jobs, active, threads, s0, k) -> torch.Tensor:
    """item_table on the current GPU."""
    return torch.from_numpy(item_table(jobs, active, threads, s0, k)).cuda()


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
        # bytes copied host -> device per step: protocol tables, directions
        # and amplitudes above, plus positions given as host arrays and the
        # chunk tables (added by prepare)
        self.h2d_bytes = sum(j["G"].numel() * 8 + j["dirs"].numel() * 4 + j["amps"].numel() * 4 for j in self.jobs)
        self.grids = {lk: batch_grid(self.threads, lk, self.tuning.stage)
                      for lk in {j["sub"].idx_bytes for j in self.jobs}}
        self.grid = max(self.grids.values())
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
        upload their job tables, re-binning tables and item lists.

        positions: per job (positions [3, N], labels [N] or None) as device
        tensors, or as host arrays (numpy or CPU tensors, pinned for an
        asynchronous copy), which are copied to the device here; None: the
        positions given at construction, else walkers seeded on the device."""
        if positions is None:
            positions = self.positions if self.positions is not None else self.seed_positions()
        dev = torch.device("cuda", torch.cuda.current_device())
        placed = []
        for x, lab in positions:
            if not (isinstance(x, torch.Tensor) and x.is_cuda):
                x = torch.as_tensor(x, dtype=torch.float32)
                self.h2d_bytes += x.numel() * 4
                x = x.to(dev, non_blocking=True)
            if lab is not None and not (isinstance(lab, torch.Tensor) and lab.is_cuda):
                lab = torch.as_tensor(lab, dtype=torch.int32)
                self.h2d_bytes += lab.numel() * 4
                lab = lab.to(dev, non_blocking=True)
            placed.append((x, lab))
        self.positions = placed
        for j, (x, lab) in zip(self.jobs, placed):
            if "buf" not in j:  # allocated once: the chunk tables point at these buffers
                j["buf"] = [engine.FusedState(j["N"]), engine.FusedState(j["N"])]
            wk = engine.Walkers(x, x.clone(), phi=torch.zeros((6, j["N"]), device=x.device), label=lab)
            j["buf"][0].pack(wk)
        if not self._planned:
            self._plan()
        return self

    def _plan(self):
        k = self.tuning.steps_per_launch
        nmax = max(j["nsteps"] for j in self.jobs)
        self.chunks = []
        cur = [0] * len(self.jobs)
        need = 0
        for s0 in range(0, nmax, k):
            active = [i for i, j in enumerate(self.jobs) if j["nsteps"] > s0]
            pairs = [(self.jobs[i], self.jobs[i]["buf"][cur[i]], self.jobs[i]["buf"][cur[i] ^ 1]) for i in active]
            for i in active:
                cur[i] ^= 1
            states = [self.jobs[i]["buf"][cur[i]] for i in range(len(self.jobs))]
            sort, n_sort, tw, tk = _sort_table(pairs, self.tuning.coarsen, self.tuning.by_label)
            need = max(need, int(L.load().nz_batch_sort_scratch_bytes(tw, tk)))
            launches = []
            for lk, grp in sorted(list_groups(self.jobs, active).items()):
                items = _items(self.jobs, grp, self.threads, s0, k)
                launches.append((lk, items))
                self.h2d_bytes += items.numel() * 4
            ws = sum(min(k, self.jobs[i]["nsteps"] - s0) * self.jobs[i]["N"] for i in active)
            self.chunks.append({"s0": s0, "s1": s0 + k, "active": active, "table": _job_table(self.jobs, states),
                                "launches": launches, "sort": sort, "n_sort": n_sort, "sort_walkers": tw,
                                "sort_keys": tk, "walker_steps": ws})
            self.h2d_bytes += sort.numel() + self.chunks[-1]["table"].numel()
        self.final_cur = cur
        self.sort_scratch = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
        self.queue = torch.zeros(3 * len(self.chunks), dtype=torch.int32, device="cuda")
        self.out = [torch.zeros((2, j["dirs"].shape[1], j["amps"].numel()), dtype=torch.float64, device="cuda")
                    for j in self.jobs]
        self._planned = True

    # -- the run -------------------------------------------------------------------
    def run(self, events: list | None = None):
        """Every chunk: one re-binning of all its jobs, one batched walk; then
        each job's signal.  events: if a list, (start, end) CUDA events of each
        batched walk launch are appended to it."""
        lib = L.load()
        cs = torch.cuda.current_stream()
        stream = ctypes.c_void_p(cs.cuda_stream)
        self.queue.zero_()
        for qi, c in enumerate(self.chunks):
            L.check(lib.nz_batch_sort(ctypes.c_void_p(c["sort"].data_ptr()), c["n_sort"], c["sort_walkers"],
                                      c["sort_keys"], ctypes.c_void_p(self.sort_scratch.data_ptr()),
                                      self.sort_scratch.numel(), stream), "nz_batch_sort")
            if events is not None:
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(cs)
            for g, (lk, items) in enumerate(c["launches"]):
                launch_batch(c["table"], len(self.jobs), items, lk, c["s0"], c["s1"],
                             self.queue.data_ptr() + 4 * (3 * qi + g), self.grids[lk], self.threads,
                             self.tuning.stage, stream)
            if events is not None:
                e1.record(cs)
                events.append((e0, e1))
        for i, (j, out) in enumerate(zip(self.jobs, self.out)):
            out.zero_()
            j["buf"][self.final_cur[i]].signal(j["dirs"], j["amps"], out)
        return self

    def step(self):
        """prepare + run: one pass of the batch from its initial positions."""
        return self.prepare().run()

    def launches(self) -> int:
        """Library kernels of one step (prepare + run): a pack per job; per
        chunk the re-binning of all its jobs (bin count, the key scan: one
        kernel, or three above SCAN_SINGLE_KEYS keys, scatter) and one batched
        walk; a signal per job."""
        n = sum(1 for j in self.jobs if j["N"]) * 2  # pack and signal
        for c in self.chunks:
            if c["sort_walkers"]:
                n += 2 + (1 if c["sort_keys"] <= L.SCAN_SINGLE_KEYS else 3)
            n += sum(1 for _, items in c["launches"] if items.shape[0])
        return n

    def signals(self) -> list:
        """Per job S[d][b] (complex, normalised by N), copied to the host."""
        res = []
        for j, out in zip(self.jobs, self.out):
            s = out.cpu().numpy()
            res.append((s[0] + 1j * s[1]) / j["N"])
        return res

    def d2h_bytes(self) -> int:
        return sum(out.numel() * out.element_size() for out in self.out)

    def walker_steps(self) -> int:
        return sum(j["N"] * j["nsteps"] for j in self.jobs)

    def final_state(self, i: int) -> engine.FusedState:
        return self.jobs[i]["buf"][self.final_cur[i]]


def simulate_batch(specs: list, positions=None, tuning: Tuning | None = None, threads: int = 128,
                   cache: SubstrateCache | None = None, stats: dict | None = None) -> list:
    """Signals of many solves at once: S[d][b] (complex, per job) for every
    JobSpec, walked together in persistent batched launches.

    positions: per job (positions [3, N], labels [N] or None) on the host or
    the device, or None to seed every job on the device.  cache: a
    SubstrateCache to keep the cell lists of repeated substrates between
    calls.  stats: if a dict, receives the bytes copied host -> device
    ("h2d_bytes") and device -> host ("d2h_bytes") by this call."""
    run = BatchRun(specs, tuning=tuning, threads=threads, cache=cache)
    out = run.prepare(positions).run().signals()
    if stats is not None:
        stats["h2d_bytes"] = int(run.h2d_bytes)
        stats["d2h_bytes"] = int(run.d2h_bytes())
    return out
