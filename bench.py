"""Benchmark of the spin random walk: walker-steps/s on the packed-substrate
workload (200 beaded axons, 20,000 spheres + periodic images, 40x40x80 um box,
1e6 walkers per GPU, PGSE 20/10/30 ms at dt = 5 us = 6000 steps, 30 directions
x b in {0, 1, 2, 3} ms/um^2).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One step = one pass of the hot path over one batch: every walker through all
6000 time steps (fused launches with re-binning between them) plus the signal
reduction, inputs (seeded positions, substrate, protocol) resident in HBM.
`value` is the whole-job walker-steps/s (all ranks; walkers are sharded,
weak scaling, no data-path collective).  `e2e` is the same metric through the
public call with host buffers: positions copied in from pinned memory and the
signal copied out every step.

--impl reference: the reference has no CPU implementation of the walk; the
reference arm times the reference's own kernel source compiled for the CPU
(oracle/_ref, built where the reference tree is present: its launches run as
OpenMP loops over walkers on the host cores) on a bounded sample of the same
workload, or, without that build, the oracle's C restatement of the kernel.
--impl reference_gpu: the reference's kernel compiled for sm_100a (baseline/_ref)
launched on this GPU one waveform sample at a time, as the reference does.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = ("packed substrate: 200 beaded axons x 100 spheres (lognormal r0 1.0/0.3 um, bead amplitude "
            "U[0.2,0.5]), periodic 40x40x80 um box, 1e6 walkers/GPU over intra+extra space, D=2.0 um^2/ms, "
            "PGSE delta=10 Delta=20 te=30 ms at dt=5 us (6000 steps), 30 directions x b={0,1,2,3} ms/um^2")


# the configuration profiled with ncu, its DRAM read + write bytes per
# walk_fused_kernel launch (1e6 walkers x 2000 steps) and its warp
# instructions per walker-step
PROFILED_SHAPE = (1_000_000, 0.5, 0.5, 2000)
PROFILED_TRAFFIC_BYTES = 9_966_812_000 + 94_345_472
PROFILED_WARP_INST_PER_WALKER_STEP = 56.5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference_gpu"],
                    help="reference: the reference's walk on the host cores; reference_gpu: the reference's own "
                         "CUDA kernel (baseline/_ref build) on this GPU, one launch per waveform sample")
    ap.add_argument("--ref-samples", type=int, default=600,
                    help="reference_gpu: waveform samples (launches) timed, after --warmup x 10 untimed")
    ap.add_argument("--walkers", type=int, default=1_000_000)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU work of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cell", type=float, default=None)
    ap.add_argument("--steps-per-launch", type=int, default=None)
    ap.add_argument("--coarsen", type=int, default=None)
    ap.add_argument("--by-label", type=int, default=None, help="re-bin by (label, bin): 1, or by bin only: 0")
    ap.add_argument("--near-margin", type=float, default=None, help="near-list margin in um (0: none)")
    ap.add_argument("--narrow-walkers", type=float, default=5e5, help="narrow: walkers")
    ap.add_argument("--narrow-ms", type=float, default=100.0, help="narrow: simulated time, ms")
    ap.add_argument("--workload", default="packed", choices=["packed", "batched", "serving", "narrow"],
                    help="packed: one packed substrate (default); batched: 64 mixed substrates, batched vs plain; "
                         "serving: Poisson request streams, continuous batching, p50/p99 latency; "
                         "narrow: the narrow-pulse simulation CLI path on a calibration-like substrate")
    ap.add_argument("--rates", default="5,20,50,100,200", help="serving: request rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="serving: arrival window per rate")
    ap.add_argument("--serve-cell", type=float, default=1.5, help="serving: cell edge of the cached lists, um")
    ap.add_argument("--serve-coarsen", type=int, default=8, help="serving: re-binning bins in cells per axis")
    ap.add_argument("--max-requests", type=int, default=200, help="serving: requests per rate at most")
    ap.add_argument("--jobs", type=int, default=64, help="batched: number of substrates")
    ap.add_argument("--walker-scale", type=float, default=1.0, help="batched: scale of the walker counts")
    ap.add_argument("--threads", type=int, default=128, help="batched: walkers per CTA")
    ap.add_argument("--plain-every", type=int, default=1, help="batched: time the plain path on every k-th job")
    ap.add_argument("--autotune", action="store_true", help="batched: pick the launch shape with the autotuner")
    return ap.parse_args()


def workload():
    from nozomi_b200.workloads import packed_workload
    return packed_workload()


# ---------------------------------------------------------------------------
# CPU side: the oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_sample(sub, pg, dirs, cell, seconds, rank_seed=0, work=True):
    """Time the oracle on a bounded sample sized to about `seconds` of work.
    Returns (walker-steps/s, cores, sample description, work per walker-step)."""
    from oracle import oracle as oz
    from nozomi_b200.substrates import cell_grid
    from nozomi_b200.waveforms import step_tables
    cores = os.cpu_count() or 1
    sph = sub.spheres()
    nseg = cell_grid(sub.L, cell)
    st, ct, it = oz.cells(sph, sub.L, nseg)
    ns = sub.nstructures
    g = oz.Geometry(sph.astype(np.float32), ns, sub.L, nseg, st, ct, it, np.full(ns + 1, 2.0, np.float32),
                    np.full(ns + 1, 100.0, np.float32))
    G, Ga = step_tables(pg)
    nw = 64 * cores
    spins, _, left = oz.seed(g, list(range(ns + 1)), nw, key0=rank_seed ^ 0x5EED)
    probe_steps = 20
    sp, s0, phi = spins.copy(), spins.copy(), np.zeros((6, nw), np.float32)
    t = time.perf_counter()
    oz.walk_f32(g, oz.philox(rank_seed), oz.MODE_PHI, sp, s0, 0, probe_steps, pg.dt, G=G, Garea=Ga, phi=phi,
                counters=False, nthreads=cores)
    rate = nw * probe_steps / (time.perf_counter() - t)
    nsteps = int(np.clip(seconds * rate / nw, 20, G.size))
    if nsteps == G.size:  # the whole protocol is short: add walkers instead
        nw = int(np.clip(seconds * rate / G.size, nw, 4_000_000))
        spins, _, left = oz.seed(g, list(range(ns + 1)), nw, key0=rank_seed ^ 0x5EED)
    sp, s0, phi = spins.copy(), spins.copy(), np.zeros((6, nw), np.float32)
    t = time.perf_counter()
    oz.walk_f32(g, oz.philox(rank_seed), oz.MODE_PHI, sp, s0, 0, nsteps, pg.dt, G=G, Garea=Ga, phi=phi,
                counters=False, nthreads=cores)
    el = time.perf_counter() - t
    value = nw * nsteps / el
    wk = None
    if work:
        nwk = min(nw, 2048)
        sp, s0, phi = spins[:, :nwk].copy(), spins[:, :nwk].copy(), np.zeros((6, nwk), np.float32)
        r = oz.walk_f32(g, oz.philox(rank_seed), oz.MODE_PHI, sp, s0, 0, min(nsteps, 200), pg.dt, G=G, Garea=Ga,
                        phi=phi, counters=False, work=True, nthreads=cores)
        n = nwk * min(nsteps, 200)
        wk = {"iterations": r["work"][0] / n, "spheres_in_reach": r["work"][1] / n, "solves_in_reach": r["work"][2] / n}
    sample = f"{nw} walkers x {nsteps} steps (steps 0..{nsteps - 1} of the protocol), {el:.1f} s"
    return value, cores, sample, wk


REF_CPU_BUILD = "packed_cpu_16k"
REF_CPU_KIND = ("the reference's own sim3d_kernel.cu (randomWalk3d_phase_multidirr, template filled as DiffSim3d "
                "does, padded set_segments table at 1 um cells) compiled for the CPU with host stand-ins for its "
                "CUDA headers (oracle/refshim): each kernel launch runs its 1000-thread blocks as OpenMP "
                "iterations over walkers; curand_normal reads the oracle's Philox normals")


class ReferenceCpu:
    """The reference kernel's CPU build (oracle/_ref, named build) walking
    the first N walkers of the packed workload, launch by launch."""

    def __init__(self, sub, pg, dirs, key=1000):
        import ctypes
        from oracle import oracle as oz
        from oracle.build import reference_named
        b = reference_named(REF_CPU_BUILD)
        if b is None:
            raise FileNotFoundError(f"oracle/_ref build {REF_CPU_BUILD} is absent")
        so, pars = b
        self.lib = ctypes.CDLL(str(so))
        P, f, i = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
        self.lib.ref_run_walk_multidir.argtypes = [i, i, i, f, P, P, P, P, P, f, f, P, i]
        self.lib.ref_run_initstates.argtypes = [i, i, i]
        self.lib.ref_set_philox.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
        from nozomi_b200.substrates import cell_grid
        from nozomi_b200.waveforms import step_tables
        self.N = N = int(pars["nspins"])
        nseg = cell_grid(sub.L, 1.0)
        if (int(pars["nLx"]), int(pars["nLy"]), int(pars["nLz"])) != tuple(nseg) or int(pars["nspheres"]) != sub.S:
            raise ValueError("the reference CPU build does not match this workload")
        sph64 = sub.spheres()
        st, ct, it = oz.cells(sph64, sub.L, nseg)
        self.K = K = int(pars["nspheres_per_seg"])
        if int(ct.max()) != K:
            raise ValueError(f"cell table K={int(ct.max())} but the build has {K}")
        self.seg = oz.segments(sph64, sub.L, nseg, K)
        ns = sub.nstructures
        g = oz.Geometry(sph64.astype(np.float32), ns, sub.L, nseg, st, ct, it, np.full(ns + 1, 2.0, np.float32),
                        np.full(ns + 1, 100.0, np.float32))
        x, _, left = oz.seed(g, list(range(ns + 1)), N, key ^ 0x5EED)
        self.spins = np.ascontiguousarray(x.reshape(-1))
        self.spins0 = self.spins.copy()
        self.ndir = dirs.shape[1]
        self.phase = np.zeros(self.ndir * N, np.float32)
        self.sph = np.ascontiguousarray(sph64.astype(np.float32))
        self.dd = np.ascontiguousarray(dirs.astype(np.float32))
        self.G, self.Ga = step_tables(pg)
        self.dt = float(pg.dt)
        self.lib.ref_run_initstates(N // 1000, 1000, 1000)
        self.lib.ref_set_philox(key, 0, 0)
        self.n = 0

    def run(self, nsteps):
        """Launch the next nsteps waveform samples (wrapping to the start)."""
        f = float
        for _ in range(nsteps):
            n = self.n % self.G.size
            self.lib.ref_run_walk_multidir(self.N // 1000, 1000, n, f(self.dt), self.sph.ctypes.data,
                                           self.seg.ctypes.data, self.spins.ctypes.data, self.spins0.ctypes.data,
                                           self.phase.ctypes.data, f(self.G[n]), f(self.Ga[n]), self.dd.ctypes.data,
                                           self.ndir)
            self.n += 1


def reference_cpu_sample(sub, pg, dirs, seconds, steps=1, warmup=0):
    """Time the reference kernel's CPU build: `warmup` + `steps` samples of
    about `seconds` each.  Returns (walker-steps/s, cores, sample text, ms per
    timed sample)."""
    cores = os.cpu_count() or 1
    r = ReferenceCpu(sub, pg, dirs)
    t = time.perf_counter()
    r.run(5)
    rate = r.N * 5 / (time.perf_counter() - t)
    per = int(np.clip(seconds * rate / r.N, 5, r.G.size))
    r.run(per * warmup)
    t = time.perf_counter()
    r.run(per * steps)
    el = time.perf_counter() - t
    sample = (f"{r.N} walkers x {per} launches per step x {steps} step(s) (waveform samples "
              f"{5 + per * warmup}..{5 + per * (warmup + steps) - 1}), {el:.1f} s, padded K={r.K}")
    return r.N * per * steps / el, cores, sample, el * 1e3 / steps


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sub, pg, dirs, bvals = workload()
    from oracle.build import build_oracle
    build_oracle()
    try:
        value, cores, sample, ms_step = reference_cpu_sample(sub, pg, dirs, args.cpu_seconds / 2, steps=args.steps,
                                                             warmup=args.warmup)
        kind, how = "reference", REF_CPU_KIND
    except (FileNotFoundError, ValueError) as e:  # no reference build on this host: the C restatement
        total_t, total_ws = 0.0, 0
        for i in range(args.warmup + args.steps):
            v, cores, sample, _ = cpu_sample(sub, pg, dirs, args.cell or 1.0, args.cpu_seconds / 2, rank_seed=i,
                                             work=False)
            if i >= args.warmup:
                total_ws += 1
                total_t += 1.0 / v
        value = total_ws / total_t
        ms_step = None  # samples of differing walker counts: no common step time
        kind, how = "port", f"oracle/walk_oracle.c, the C restatement of the kernel, OpenMP over walkers ({e})"
    line = {"impl": "reference", "metric": "walker-steps/s", "value": value, "unit": "walker-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cell_um": 1.0},
            "cpu_baseline": {"value": value, "unit": "walker-steps/s", "cores": cores, "kind": kind,
                             "sample": sample + "; " + how},
            "e2e": {"value": value, "unit": "walker-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
def _hex_id(v) -> str:
    """A GPU UUID in comparable form: lower-case hex digits only."""
    s = str(v).lower()
    if s.startswith("gpu-"):
        s = s[4:]
    return "".join(c for c in s if c in "0123456789abcdef")


class Clocks:
    """nvidia-smi sampling during the timed region.  Every GPU of the machine
    is sampled with its UUID and PCI bus id; the summary keeps the rows of the
    CUDA device this process runs on (nvidia-smi's index need not be CUDA's
    under CUDA_VISIBLE_DEVICES)."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = Path("/tmp") / f"nz_clocks_{os.getpid()}.csv"
        self.uuid, self.bus = None, None
        try:
            import torch
            props = torch.cuda.get_device_properties(torch.cuda.current_device())
            self.uuid = _hex_id(getattr(props, "uuid", "")) or None
            self.bus = getattr(props, "pci_bus_id", None)
        except Exception:  # device identity is a refinement; the index is the fallback
            pass

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,uuid,pci.bus_id")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        text = self.path.read_text()
        self.path.unlink(missing_ok=True)
        return self.summarise(text, uuid=self.uuid, bus=self.bus, index=self.index)

    @staticmethod
    def summarise(text, uuid=None, bus=None, index=None):
        """Median SM clock, the maximum and the throttle reasons seen in
        nvidia-smi's csv,noheader,nounits lines (the query of start()), over
        the rows of one GPU: the one whose UUID, else PCI bus, else index
        matches; all rows when nothing identifies it."""
        rows = [r.split(", ") for r in text.strip().splitlines() if r.strip()]
        mine = []
        if uuid:
            mine = [r for r in rows if len(r) > 9 and _hex_id(r[9]) == _hex_id(uuid)]
        if not mine and bus is not None:
            def bus_of(r):
                try:
                    return int(r[10].split(":")[1], 16)
                except (IndexError, ValueError):
                    return None
            mine = [r for r in rows if len(r) > 10 and bus_of(r) == int(bus)]
        if not mine and index is not None:
            mine = [r for r in rows if r[0].strip() == str(index)]
        rows = mine or rows
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        mx = float(rows[0][2]) if len(rows[0]) > 2 and rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from nozomi_b200 import engine, _lib as L
    from nozomi_b200.shard import ShardedDwiRun, reduce_sums
    from nozomi_b200.simulate import Tuning, device_substrate

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        # a short collective timeout: a rank that died ends the others' next
        # collective with an error instead of a hang (set-up before the first
        # barrier takes well under this)
        from nozomi_b200.shard import init_process_group
        init_process_group("nccl", timeout_s=180)
    engine.require_cuda()
    sub, pg, dirs, bvals = workload()
    # launch shape tuned for this workload (profiles/walk_fused_packed_tuning.md):
    # 0.5 um cells, near margin 0.5 um, re-binning bins of 8^3 cells, 2000 steps per launch
    tuning = Tuning(cell=0.5, near_margin=0.5, coarsen=8, steps_per_launch=2000)
    if args.cell:
        tuning.cell = args.cell
    if args.steps_per_launch:
        tuning.steps_per_launch = args.steps_per_launch
    if args.coarsen:
        tuning.coarsen = args.coarsen
    if args.by_label is not None:
        tuning.by_label = bool(args.by_label)
    if args.near_margin is not None:
        tuning.near_margin = args.near_margin if args.near_margin > 0 else None
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=tuning.cell, near_margin=tuning.near_margin)
    # the one-time cell build (member lists, near lists, per-entry records) is
    # outside the metric; it is timed on a second build, the first having
    # loaded the library and warmed the allocator
    torch.cuda.synchronize()
    tb = time.perf_counter()
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=tuning.cell, near_margin=tuning.near_margin)
    torch.cuda.synchronize()
    cell_build_ms = (time.perf_counter() - tb) * 1e3
    amps = pg.amplitude_for_b(bvals)
    N = args.walkers
    # walkers [rank*N, (rank+1)*N) of one run of N*world walkers; the signal
    # sums are all-reduced once per step (the path's one exchange)
    shard = ShardedDwiRun(dsub, pg, dirs, amps, N * world, seed=1000, rank=rank, world=world, tuning=tuning)
    run = shard.run
    x0, lab0 = run.initial_positions()
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def one_step(walk_events=None, x=None):
        run.prepare(x0 if x is None else x, lab0)
        run.walk(walk_events)
        return run.signal_sums()


    # FP32 peak of this GPU (probe kernel), before the timed region
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    probe_out = torch.zeros(sms * 16, device="cuda")
    lib = L.load()
    iters = 4096
    for _ in range(2):
        L.check(lib.nz_probe_fma(sms * 16, iters, probe_out.data_ptr(), stream.cuda_stream), "probe")
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record(stream)
    L.check(lib.nz_probe_fma(sms * 16, iters, probe_out.data_ptr(), stream.cuda_stream), "probe")
    pe1.record(stream)
    torch.cuda.synchronize()
    fp32_peak_tflops = sms * 16 * 256 * iters * 8 * 2 / (pe0.elapsed_time(pe1) * 1e-3) / 1e12

    for _ in range(args.warmup):
        one_step()
        flush.zero_()
    barrier()
    # one step captured as a CUDA graph (pack, re-bins, fused launches, signal)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        sig_static = one_step()
    graph.replay()
    barrier()

    clocks = Clocks(local)
    clocks.start()
    step_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the step's events)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        graph.replay()
        reduce_sums(sig_static)
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms += e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    sig = sig_static.clone()

    # the same step launched eagerly with CUDA events around every fused launch:
    # the dominant kernel's average duration and its share of the step
    walk_ms, n_walk = 0.0, 0
    flush.zero_()
    torch.cuda.synchronize()
    ev = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    one_step(ev)
    e1.record(stream)
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1)
    # library kernels of one step (pack; per chunk the re-binning's bin count,
    # histogram scan and scatter, and the fused walk; the signal), as counted
    # by the run while it launched them
    launches_per_step = run.launches
    walk_ms = sum(a.elapsed_time(b) for a, b in ev)
    n_walk = len(ev)

    t_local = torch.tensor([step_ms, walk_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    step_ms, walk_ms = float(t_local[0]), float(t_local[1])
    ws_per_step = N * run.nsteps * world
    value = ws_per_step * args.steps / (step_ms * 1e-3)
    S = sig.cpu().numpy()
    S = (S[0] + 1j * S[1]) / (N * world)

    # end to end with host buffers: positions copied from pinned host memory
    # into the graph's input, the step replayed, the signal copied back
    x_host = x0.cpu().pin_memory()
    e2e_ms = 0.0
    out_bytes = 0
    host = torch.empty_like(sig_static, device="cpu").pin_memory()
    for i in range(args.e2e_steps + 1):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        x0.copy_(x_host, non_blocking=True)
        graph.replay()
        reduce_sums(sig_static)
        host.copy_(sig_static, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        out_bytes = host.numel() * host.element_size()
        if i > 0:  # first pass warms the path
            e2e_ms += e0.elapsed_time(e1)
    t_local = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    e2e_value = ws_per_step * args.e2e_steps / (float(t_local[0]) * 1e-3)
    del graph

    line = None
    if rank == 0:
        walk_launch_ms = walk_ms / max(n_walk, 1)
        per_launch_ws = N * tuning.steps_per_launch
        kernel_ws_s = N * run.nsteps / (walk_ms * 1e-3)
        cpu = None
        wk = None
        if world == 1 and not args.no_cpu_baseline:
            v, cores, sample, wk = cpu_sample(sub, pg, dirs, tuning.cell, args.cpu_seconds / 2)
            port = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "port",
                    "sample": sample + "; oracle/walk_oracle.c, OpenMP over walkers"}
            try:
                v, cores, sample, _ = reference_cpu_sample(sub, pg, dirs, args.cpu_seconds / 2)
                cpu = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "reference",
                       "sample": sample + "; " + REF_CPU_KIND, "port": port}
            except (FileNotFoundError, ValueError) as e:
                cpu = dict(port, reference_unavailable=str(e))
        peaks = {}
        pk = ROOT / "MEASURED_PEAKS.json"
        if pk.exists():
            peaks = json.loads(pk.read_text())
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        # HBM view: walker state read + written once per launch (4 x float4 each way)
        state_bytes = N * 128
        # DRAM bytes of one launch from an ncu capture of this configuration
        # (profiles/walk_fused_packed1e6_ncu.md); none for other shapes
        traffic = None
        if (N, tuning.cell, tuning.near_margin, tuning.steps_per_launch) == PROFILED_SHAPE:
            traffic = PROFILED_TRAFFIC_BYTES
        roof_hbm = {"bound": "hbm", "achieved": state_bytes / (walk_launch_ms * 1e-3) / 1e9, "peak": hbm_peak,
                    "unit": "GB/s", "traffic": traffic, "algorithmic_bytes_per_launch": state_bytes,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs" if pk.exists() else "fallback 6.65 TB/s"}
        roof_hbm["frac"] = roof_hbm["achieved"] / hbm_peak
        roof_fp32 = None
        if wk is not None:
            F_alg = 10 * wk["spheres_in_reach"] + 36 * wk["solves_in_reach"] + 6 * dirs.shape[1]
            ach = kernel_ws_s * F_alg / 1e12
            roof_fp32 = {"bound": "fp32", "achieved": ach, "peak": fp32_peak_tflops, "unit": "TFLOP/s",
                         "frac": ach / fp32_peak_tflops, "flops_per_walker_step": F_alg, "work_per_walker_step": wk,
                         "peak_source": "nz_probe_fma on this GPU (8 FFMA chains/thread)"}
        # the bound that binds this kernel: instruction issue (4 warp-instructions
        # per SM per cycle), with the warp-instructions per walker-step counted
        # by ncu for the profiled shape
        roof_issue = None
        if traffic is not None and clk and clk.get("sm_mhz"):
            peak = sms * 4 * clk["sm_mhz"] * 1e6
            ach = PROFILED_WARP_INST_PER_WALKER_STEP * kernel_ws_s
            roof_issue = {"bound": "issue", "achieved": ach, "peak": peak, "unit": "warp-instructions/s",
                          "frac": ach / peak, "warp_instructions_per_walker_step": PROFILED_WARP_INST_PER_WALKER_STEP,
                          "peak_source": f"{sms} SMs x 4 issue slots x median SM clock under load"}
        line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded packed-axon substrate, seeded walkers)",
                "config": {"workload": WORKLOAD, "walkers_per_gpu": N, "time_steps": run.nsteps,
                           "directions": int(dirs.shape[1]), "bvalues": bvals.tolist(),
                           "cell_um": tuning.cell, "steps_per_launch": tuning.steps_per_launch,
                           "rebin_coarsen": tuning.coarsen, "rebin_by_label": tuning.by_label, "near_margin_um": tuning.near_margin,
                           "near_list_entries": int(dsub.near[2].numel()) if dsub.near is not None else 0,
                           "spheres": sub.S, "cells": dsub.ncell,
                           "cell_list_entries": dsub.n_items, "l2": "256 MiB flush between timed steps",
                           "parallelism": f"walkers sharded over {world} GPU(s) by walker-id range; "
                                          "one all-reduce of the signal sums per step"},
                "e2e": {"value": e2e_value, "unit": "walker-steps/s",
                        "h2d_bytes_per_step": int(x_host.numel() * x_host.element_size()),
                        "d2h_bytes_per_step": int(out_bytes)},
                "gpu_launches": launches_per_step * args.steps,
                "kernel": {"name": "walk_fused_kernel", "launches": n_walk, "avg_launch_ms": walk_launch_ms,
                           "walker_steps_per_launch": per_launch_ws, "kernel_walker_steps_per_s": kernel_ws_s,
                           "share_of_step": walk_ms / eager_ms, "eager_step_ms": eager_ms,
                           "timing": "value from CUDA-graph replays of the step; kernel figures from one eager "
                                     "step with events around each fused launch"},
                "cell_build": {"ms": cell_build_ms, "timing": "wall clock of one device_substrate build "
                               "(host preparation, cell and near lists, per-entry records), synchronised on "
                               "both sides; once per substrate, not part of value"},
                "roofline": roof_hbm, "roofline_fp32": roof_fp32, "roofline_issue": roof_issue,
                "cpu_baseline": cpu, "clocks": clk,
                "signal_b0_mean": float(np.mean(np.abs(S[:, 0]))),
                "signal_mean_by_b": [float(np.mean(S[:, b].real)) for b in range(S.shape[1])]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


BATCH_WORKLOAD = ("batched mixed workload: {jobs} substrates of 10-500 beaded axons (40 spheres at 1 um, radii "
                  "U[0.5,1.5], z-periodic, packed at area fraction 0.35), walkers log-uniform 1e4-1e6 (x{scale}), "
                  "2000-8000 steps at dt=5 us (PGSE delta=te/3, Delta=2te/3), 6-60 directions, b={{0,1,2,3}} "
                  "ms/um^2, seed 4")


def run_batched(args):
    import torch
    from nozomi_b200 import engine
    from nozomi_b200.batch import BatchRun, SubstrateCache
    from nozomi_b200.plain import run_plain
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.workloads import mixed_specs
    import torch.distributed as dist
    from nozomi_b200.shard import init_process_group, shard_jobs
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if world > 1:
        init_process_group("nccl", timeout_s=180)
    engine.require_cuda()
    all_specs = mixed_specs(seed=4, n_jobs=args.jobs, walker_scale=args.walker_scale)
    # over several GPUs the jobs shard whole, longest first onto the least
    # loaded rank; no data crosses ranks
    mine = shard_jobs([sp.walker_steps for sp in all_specs], world)[rank] if world > 1 else range(len(all_specs))
    specs = [all_specs[i] for i in mine]
    tuning = Tuning()
    if args.steps_per_launch:
        tuning.steps_per_launch = args.steps_per_launch
    if args.near_margin is not None:
        tuning.near_margin = args.near_margin if args.near_margin > 0 else None
    tune_report = None
    threads = args.threads
    if args.autotune:
        from nozomi_b200.autotune import autotune
        tuning, threads, tune_report = autotune(specs)
    cache = SubstrateCache()
    run = BatchRun(specs, tuning=tuning, threads=threads, cache=cache)
    stream = torch.cuda.current_stream()
    run.step()
    for _ in range(max(0, args.warmup - 1)):
        run.step()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        run.step()
    torch.cuda.synchronize()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    ms = 0.0
    for _ in range(args.steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        graph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    clk = clocks.stop()
    del graph
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t[0])
    ws = sum(sp.walker_steps for sp in all_specs)
    value = ws * args.steps / (ms * 1e-3)
    sig_batched = run.signals()
    if world > 1:  # the plain comparison is a one-GPU measurement
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic (seeded substrates, protocols and walkers)",
                              "config": {"workload": BATCH_WORKLOAD.format(jobs=len(all_specs),
                                                                           scale=args.walker_scale),
                                         "jobs": len(all_specs), "walker_steps_per_step": ws,
                                         "parallelism": f"jobs sharded whole over {world} GPUs"},
                              "clocks": clk}), flush=True)
        return 0
    # the plain per-substrate path, one job after another, launched from the
    # host, on cell lists of the default shape (1 um cells; not the batch's
    # tuned shape, which the plain kernel does not benefit from)
    sel = list(range(0, len(specs), args.plain_every))
    plain_ms, plain_ws, err = 0.0, 0, 0.0
    plain_tuning, plain_cache = Tuning(), SubstrateCache()
    for i in sel:
        sp = specs[i]
        dsub = plain_cache.get(sp.key, sp.substrate, sp.D, sp.T2, plain_tuning)
        x = run.positions[i][0]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = run_plain(dsub, sp, x)
        e1.record(stream)
        torch.cuda.synchronize()
        plain_ms += e0.elapsed_time(e1)
        plain_ws += sp.N * sp.nsteps
        o = out.cpu().numpy()
        err = max(err, float(np.abs((o[0] + 1j * o[1]) / sp.N - sig_batched[i]).max()))
    plain_value = plain_ws / (plain_ms * 1e-3)
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded substrates, protocols and walkers)",
            "config": {"workload": BATCH_WORKLOAD.format(jobs=len(specs), scale=args.walker_scale),
                       "jobs": len(specs), "walker_steps_per_step": ws, "threads": threads,
                       "steps_per_launch": tuning.steps_per_launch, "near_margin_um": tuning.near_margin,
                       "cell_um": tuning.cell, "rebin_coarsen": tuning.coarsen,
                       "persistent_grid": run.grid, "chunks": len(run.chunks)},
            "autotune": None if tune_report is None else {
                "cached": tune_report["cached"], "choice": {"threads": threads, **dataclasses.asdict(tuning)},
                "trials": len(tune_report.get("trials", [])),
                "trial_walker_steps_per_s": tune_report.get("trial_walker_steps_per_s")},
            "gpu_launches": run.launches() * args.steps,
            "plain": {"value": plain_value, "unit": "walker-steps/s", "jobs_timed": len(sel),
                      "walker_steps_timed": plain_ws, "cell_um": plain_tuning.cell,
                      "launch": "one plain-kernel launch per step from the host, "
                      "per-direction phase in HBM, substrates one after another"},
            "speedup_vs_plain": value / plain_value,
            "max_signal_diff_batched_vs_plain": err, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    import torch
    if int(os.environ.get("RANK", "0")) != 0:  # a one-GPU request loop
        return 0
    from nozomi_b200 import engine
    from nozomi_b200.batch import SubstrateCache
    from nozomi_b200.plain import run_plain
    from nozomi_b200.serve import Server, latency_stats
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.workloads import request_stream
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    engine.require_cuda()
    # the cell lists and re-binning of the autotuner's choice for this
    # substrate distribution (1.5 um cells, 12 um bins); a round is 500 steps
    tuning = Tuning(cell=args.serve_cell, coarsen=args.serve_coarsen, steps_per_launch=500)
    if args.steps_per_launch:
        tuning.steps_per_launch = args.steps_per_launch
    cache = SubstrateCache()
    per_rate = []
    all_done = []
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    for rate in [float(r) for r in args.rates.split(",")]:
        reqs = request_stream(rate, min(args.serve_seconds, args.max_requests / rate), seed=5,
                              max_requests=args.max_requests)
        # warm the substrate cache's first entries so every rate starts from the same state
        srv = Server(tuning=tuning, threads=args.threads, cache=cache)
        t0 = time.perf_counter()
        done = srv.serve(reqs)
        wall = time.perf_counter() - t0
        st = latency_stats(done)
        st.update({"rate_req_s": rate, "requests": len(reqs), "walker_steps": srv.walker_steps,
                   "walker_steps_per_s": srv.walker_steps / wall, "wall_s": wall, "rounds": srv.rounds,
                   "failed": sum(t.error is not None for t in done)})
        per_rate.append(st)
        all_done += done
    clk = clocks.stop()
    # the plain per-substrate kernel on a sample of the same requests, one
    # after another, on cell lists of the default shape (1 um cells)
    sample = all_done[:: max(1, len(all_done) // 8)][:8]
    stream = torch.cuda.current_stream()
    pms, pws = 0.0, 0
    plain_cache = SubstrateCache()
    for t in sample:
        sp = t.spec
        dsub = plain_cache.get(sp.key, sp.substrate, sp.D, sp.T2, Tuning())
        x, _ = engine.seed(dsub, list(range(dsub.nstructures + 1)), sp.N, key=sp.seed ^ 0x5EED)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_plain(dsub, sp, x)
        e1.record(stream)
        torch.cuda.synchronize()
        pms += e0.elapsed_time(e1)
        pws += sp.N * sp.nsteps
    plain_value = pws / (pms * 1e-3)
    total_ws = sum(r["walker_steps"] for r in per_rate)
    total_wall = sum(r["wall_s"] for r in per_rate)
    value = total_ws / total_wall
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1,
            "steps": len(per_rate), "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Poisson request streams)",
            "config": {"workload": "serving: Poisson arrivals per rate, substrates of 10-500 beaded axons reused "
                                   "with probability 0.7, 1e4-5e5 walkers, 2000-8000 steps at 5 us, 6-60 directions, "
                                   "b<=3 ms/um^2, seed 5", "rates": args.rates,
                       "arrival_window_s": args.serve_seconds, "max_requests_per_rate": args.max_requests,
                       "steps_per_launch": tuning.steps_per_launch, "threads": args.threads,
                       "cell_um": tuning.cell, "rebin_coarsen": tuning.coarsen},
            "per_rate": per_rate,
            "plain": {"value": plain_value, "unit": "walker-steps/s", "requests_timed": len(sample),
                      "launch": "one plain-kernel launch per step, requests one after another"},
            "speedup_vs_plain": value / plain_value, "substrate_cache": {"hits": cache.hits, "misses": cache.misses},
            "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_gpu(args):
    """The reference's own kernel, randomWalk3d_phase_multidirr, compiled from
    its source with its %-template filled in for this workload (baseline/_ref,
    built where the reference tree is present) and launched as
    DwiSim3d.simulate_multi_directions does: block 1000, one launch per
    waveform sample, cuRAND XORWOW draws, the padded cell table of
    set_segments.  The walkers are the ones the fused arm seeds.  Times
    --ref-samples launches; walker-steps/s = walkers x launches / time."""
    import torch
    from baseline.reference_gpu import RefGpuWalk
    from nozomi_b200 import engine
    from nozomi_b200.simulate import device_substrate
    from nozomi_b200.waveforms import step_tables
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    engine.require_cuda()
    sub, pg, dirs, bvals = workload()
    ref = RefGpuWalk("packed_1e6")
    N = ref.N
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=1.0)
    K, seg = dsub.padded_segments()
    x0, _ = engine.seed(dsub, list(range(sub.nstructures + 1)), N, key=1000 ^ 0x5EED)
    sph = torch.from_numpy(sub.spheres().astype(np.float32)).cuda()
    dd = torch.from_numpy(dirs.astype(np.float32)).cuda()
    ref.setup(sph, seg, K, x0, dirs.shape[1], dd)
    ref.initstates(1000)
    G, Ga = step_tables(pg)
    dt = np.float32(pg.dt)
    nwarm = max(3, args.warmup) * 10
    for n in range(nwarm):
        ref.step(dt, G[n], Ga[n])
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n1 = min(G.size, nwarm + args.ref_samples)
    e0.record(stream)
    for n in range(nwarm, n1):
        ref.step(dt, G[n], Ga[n])
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    launches = n1 - nwarm
    value = N * launches / (ms * 1e-3)
    line = {"impl": "reference_gpu", "metric": "walker-steps/s", "value": value, "unit": "walker-steps/s",
            "n_gpus": 1, "steps": launches, "warmup": nwarm, "ms_per_step": ms / launches,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded packed-axon substrate, seeded walkers)",
            "config": {"workload": WORKLOAD, "walkers": N, "cell_um": 1.0, "padded_cell_table_K": K,
                       "samples_timed": f"waveform samples {nwarm}..{n1 - 1} of {G.size}",
                       "kernel": "randomWalk3d_phase_multidirr (sim3d_kernel.cu:719-943), block 1000, "
                                 "one launch per sample"},
            "gpu_launches": launches, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


NARROW_WORKLOAD = ("narrow-pulse D(t)/K(t) simulation through the drop-in API (the simulation CLI path): "
                   "500 beaded axons (base diameter 1.68/0.45 um, beads +20-50 %, spheres every 0.5 um) packed "
                   "to VF 0.65 in a periodic 50 um cube, 5e5 intra-axonal walkers, D=2.25 um^2/ms, dt=2 us, "
                   "100 ms (5e4 steps), T2 weighting and displacement moments every step, nseg 20")
# The reference's published run of this kind: 5e5 spins x 5e4 steps in about
# 1 h at nseg 20 (docs/2_calibration.md:103; RTX A5000, wall time including
# table build and I/O): 6.94e6 walker-steps/s.
NARROW_PUBLISHED = 5e5 * 5e4 / 3600.0


def run_narrow(args):
    """The simulation CLI's work (cli/simulation_main.py): DiffSim3d with
    set_segments(20, 20, 20), intra-axonal seeding, then every step walked
    with its displacement moments on the device.  `value` from CUDA events
    around the walk; `e2e` from the wall clock of set-up plus walk plus the
    moments copied back, like the reference's TABLEtime + SIMtime."""
    import torch
    from nozomi_b200 import engine
    from nozomi_b200.cli.simulation_main import narrow_pulse
    from nozomi_b200.diffsim3d import DiffSim3d
    from nozomi_b200.workloads import calibration_substrate
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    engine.require_cuda()
    sub = calibration_substrate()
    N, dt, sim_time = int(args.narrow_walkers), 0.002, float(args.narrow_ms)
    nt = int(round(sim_time / dt))
    geom = sub.geometry(D=2.25, T2=100.0)
    stream = torch.cuda.current_stream()
    runs = []
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    for i in range(args.warmup + args.steps):
        if i == args.warmup:
            clocks.start()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        sim = DiffSim3d(geom, N)
        sim.set_segments(20, 20, 20)
        sim.setup(structures=list(range(sub.nstructures)), initstates_int=1234 + i)
        torch.cuda.synchronize()
        w1 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t, Dv, K = narrow_pulse(sim, nt, dt)  # ends with the moments copied to the host
        e1.record(stream)
        torch.cuda.synchronize()
        w2 = time.perf_counter()
        if i >= args.warmup:
            runs.append({"table_s": w1 - w0, "walk_ms": e0.elapsed_time(e1), "wall_s": w2 - w0,
                         "D_end": Dv[-1].tolist(), "K_end": K[-1].tolist()})
        del sim
    clk = clocks.stop()
    ws = N * nt
    walk_ms = float(np.mean([r["walk_ms"] for r in runs]))
    wall_s = float(np.mean([r["wall_s"] for r in runs]))
    value = ws / (walk_ms * 1e-3)
    e2e = ws / wall_s
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": walk_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": e2e / NARROW_PUBLISHED, "dtype": "f32",
            "data": "synthetic (seeded packed substrate, seeded walkers)",
            "config": {"workload": NARROW_WORKLOAD, "walkers": N, "time_steps": nt, "spheres": sub.S,
                       "volume_fraction": sub.meta.get("volume_fraction"),
                       "vs_baseline_basis": "e2e / 6.94e6 walker-steps/s, the reference's published run of "
                                            "this kind (RTX A5000, wall time incl. set-up)"},
            "e2e": {"value": e2e, "unit": "walker-steps/s",
                    "h2d_bytes_per_step": int(sub.S * 5 * 8), "d2h_bytes_per_step": int(nt * 6 * 8),
                    "wall_s": wall_s, "table_s": float(np.mean([r["table_s"] for r in runs]))},
            "runs": runs, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference_gpu":
        return run_reference_gpu(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "narrow":
        return run_narrow(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
