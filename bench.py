"""Benchmark of the spin random walk: walker-steps/s on one B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload batched|packed|serving|narrow]

Default workload (``batched``): the mixed workload the headline metric is
quoted on -- 64 independent substrates of 10-500 beaded axons, walker counts
log-uniform in [1e4, 1e6], 2000-8000 steps at dt = 5 us, per-substrate PGSE
protocols with 6-60 directions, b in {0, 1, 2, 3} ms/um^2 (seed 4) -- walked
together by the batched persistent work-queue kernel, the whole step captured
as a CUDA graph.  One step = every walker of every job through all of its
steps plus the signal reductions, inputs resident in HBM.  Beside `value` the
line reports:

  plain            the plain per-substrate path (one kernel launch per
                   waveform sample, per-direction phase in HBM, jobs one after
                   another) on every k-th job, and speedup_vs_plain;
  serving          the same distribution as Poisson request streams through
                   the continuous-batching server: p50/p99 latency and served
                   walker-steps/s per rate (5 and 20 req/s, stated windows);
  e2e              the same workload through the public batched call
                   (nozomi_b200.batch.simulate_batch) with positions in pinned
                   host memory and the signals copied back, every step;
  roofline         the dominant kernel's issue roofline (ncu-counted warp
                   instructions per walker-step x kernel walker-steps/s over
                   4 issue slots x SMs x clock), with the kernel-source hash
                   the counts were taken on; FP32 and HBM views beside it;
  cpu_baseline     the reference's own kernel compiled for the host cores on a
                   bounded sample of the same jobs.

--impl reference: the reference has no CPU implementation of the walk; the
reference arm times the reference's own kernel source compiled for the CPU
(oracle/_ref, built where the reference tree is present: its launches run as
OpenMP loops over walkers on the host cores) on a bounded sample of the same
workload's jobs, or, without that build, the oracle's C restatement of the
kernel.  --impl reference_gpu: the reference's kernel compiled for sm_100a
(baseline/_ref) launched on this GPU one waveform sample at a time, as the
reference does (packed workload).

--workload packed: one packed substrate (200 beaded axons, 20,000 spheres +
periodic images, 40x40x80 um box, 1e6 walkers per GPU, PGSE 20/10/30 ms at
dt = 5 us = 6000 steps, 30 directions x b in {0, 1, 2, 3} ms/um^2) through the
single-substrate fused walk.  --workload serving: the request streams alone.
--workload narrow: the narrow-pulse simulation CLI path.
"""
from __future__ import annotations

import argparse
import dataclasses
import hashlib
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
BATCH_WORKLOAD = ("batched mixed workload: {jobs} substrates of {a0}-{a1} beaded axons (40 spheres at 1 um, radii "
                  "U[0.5,1.5], z-periodic, packed at area fraction 0.35), walkers log-uniform 1e4-1e6 (x{scale}), "
                  "2000-8000 steps at dt=5 us (PGSE delta=te/3, Delta=2te/3), 6-60 directions, b={{0,1,2,3}} "
                  "ms/um^2, seed 4; all jobs in persistent work-queue launches under one CUDA graph")

# The sources the instruction and DRAM counts below depend on: the fused
# walk's kernel and the construction of the lists it scans (sha1 of their
# bytes).  The launch shape and the list form, chosen by the host code, are
# recorded beside the counts instead.
KERNEL_SOURCES = ("nozomi_b200/csrc/walk_fused.cu", "nozomi_b200/csrc/nz_common.cuh", "nozomi_b200/csrc/kernels.cuh",
                  "nozomi_b200/csrc/cells.cu", "nozomi_b200/engine.py")

# Per workload, from one ncu capture of walk_fused_kernel (--set full,
# --clock-control none) on a small case of that workload: warp instructions
# executed (smsp__inst_executed.sum) and DRAM bytes (dram__bytes_read.sum +
# dram__bytes_write.sum) of the captured launch, divided by the walker-steps
# that launch ran; kernel_sha: the sources' hash at capture.
PROFILED = {
    "packed": {"kernel_sha": "f9ddf04e9e187c30", "warp_inst_per_walker_step": 56.421,
               "dram_bytes_per_walker_step": 0.9975,
               "shape": {"cell": 0.5, "near_margin": 0.5, "coarsen": 8, "threads": 128, "lists": "index",
                         "near_shape": "round", "stage": 0},
               "capture": "walk_fused_kernel<PHI, idx16> launch 3 of `python bench.py --workload packed --walkers "
                          "1000000 --steps-per-launch 200 --steps 1 --warmup 1 --no-cpu-baseline --e2e-steps 0` "
                          "(200,000,000 walker-steps): 11,284,186,998 warp instructions, 199.5 MB DRAM"},
    "batched": {"kernel_sha": "f9ddf04e9e187c30", "warp_inst_per_walker_step": 41.074,
                "dram_bytes_per_walker_step": 0.2405,
                "shape": {"cell": 1.0, "near_margin": 0.5, "coarsen": 4, "threads": 256, "lists": "index",
                          "near_shape": "round", "stage": 0},
                "capture": "walk_fused_kernel<PHI, idx16> launch 2 of `python bench.py --walker-scale 0.1 --steps 1 "
                           "--warmup 1 --no-serving --no-plain --no-cpu-baseline --e2e-steps 0 --no-autotune --cell 1.0 "
                           "--coarsen 4 --steps-per-launch 2000 --threads 256` (64 jobs, 2,407,477,000 walker-steps): "
                           "98,884,211,945 warp instructions, 579.1 MB DRAM"},
}


def kernel_sha() -> str:
    h = hashlib.sha1()
    for rel in KERNEL_SOURCES:
        h.update((ROOT / rel).read_bytes())
    return h.hexdigest()[:16]


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="torch.distributed backend for --gpus N > 1 (gloo: host-side collectives, for checking the "
                         "multi-rank path where NCCL is not usable)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference_gpu"],
                    help="reference: the reference's walk on the host cores; reference_gpu: the reference's own "
                         "CUDA kernel (baseline/_ref build) on this GPU, one launch per waveform sample")
    ap.add_argument("--workload", default="batched", choices=["batched", "packed", "serving", "narrow"],
                    help="batched: 64 mixed substrates in persistent batched launches (default); packed: one "
                         "packed substrate; serving: Poisson request streams alone; narrow: the narrow-pulse "
                         "simulation CLI path on a calibration-like substrate")
    ap.add_argument("--ref-samples", type=int, default=600,
                    help="reference_gpu: waveform samples (launches) timed, after --warmup x 10 untimed")
    ap.add_argument("--walkers", type=int, default=1_000_000, help="packed: walkers per GPU")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=8.0,
                    help="target CPU work of the CPU baseline sample (and of each reference-arm step)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cell", type=float, default=None)
    ap.add_argument("--steps-per-launch", type=int, default=None)
    ap.add_argument("--coarsen", type=int, default=None)
    ap.add_argument("--by-label", type=int, default=None, help="re-bin by (label, bin): 1, or by bin only: 0")
    ap.add_argument("--near-margin", type=float, default=None, help="near-list margin in um (0: none)")
    ap.add_argument("--near-shape", default=None, choices=["round", "box"],
                    help="near lists by the Euclidean sphere-to-cell test (round) or the reference's box test")
    ap.add_argument("--lists", default=None, choices=["index", "records"],
                    help="the fused walk's list form: index (16/32-bit entries into one record array) or records "
                         "(per-entry sphere records)")
    ap.add_argument("--stage", type=int, default=None,
                    help="batched: records per CTA staged in shared memory by a bulk copy (nz_walk_batch_staged; "
                         "0: none, records read through L1/L2)")
    ap.add_argument("--narrow-walkers", type=float, default=5e5, help="narrow: walkers")
    ap.add_argument("--narrow-ms", type=float, default=100.0, help="narrow: simulated time, ms")
    ap.add_argument("--serve", default="5:30,20:10",
                    help="serving: rate:window pairs, requests per second and seconds of arrivals")
    ap.add_argument("--no-serving", action="store_true", help="batched: skip the serving leg")
    ap.add_argument("--serve-cell", type=float, default=None, help="serving: cell edge of the cached lists, um")
    ap.add_argument("--serve-coarsen", type=int, default=None, help="serving: re-binning bins in cells per axis")
    ap.add_argument("--max-requests", type=int, default=None, help="serving: requests per rate at most")
    ap.add_argument("--serve-max-backlog", type=float, default=None,
                    help="serving: shed a request on arrival when the backlog would take longer than this many "
                         "seconds at the recent throughput (default: no shedding)")
    ap.add_argument("--jobs", type=int, default=64, help="batched: number of substrates")
    ap.add_argument("--walker-scale", type=float, default=1.0, help="batched: scale of the walker counts")
    ap.add_argument("--axons", type=lambda v: [int(a) for a in v.split(",")], default=[10, 500],
                    help="batched: range of axon counts per substrate, lo,hi")
    ap.add_argument("--threads", type=int, default=128, help="batched: walkers per CTA")
    ap.add_argument("--plain-every", type=int, default=4, help="batched: time the plain path on every k-th job")
    ap.add_argument("--no-plain", action="store_true", help="batched: skip the plain-path comparison")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batched: the library's default launch shape instead of the autotuner's choice")
    return ap.parse_args(argv)


def load_peaks():
    """MEASURED_PEAKS.json of this machine (hbm_gbs, bf16_tflops, ...), or {}."""
    pk = ROOT / "MEASURED_PEAKS.json"
    return (json.loads(pk.read_text()), "MEASURED_PEAKS.json") if pk.exists() else ({}, None)


def rooflines(workload: str, kernel_ws_s: float, ws_per_launch: float, launch_ms: float, state_bytes: float,
              clk, sms: int, fp32_peak_tflops: float, f_alg: float | None, work=None, shape: dict | None = None):
    """The dominant kernel's rooflines: issue (the binding one), FP32 and HBM.
    kernel_ws_s: its walker-steps per second of kernel time; ws_per_launch:
    walker-steps of an average launch; state_bytes: algorithmic bytes of an
    average launch (walker state in and out); shape: the line's launch shape,
    compared with the one the counts were captured at (the instructions per
    walker-step depend on the cell size and the near margin)."""
    prof = PROFILED.get(workload, {})
    sha = kernel_sha()
    stale = prof.get("kernel_sha") != sha
    shape_ok = None
    if shape is not None and prof.get("shape"):
        shape_ok = all(shape.get(k) == v for k, v in prof["shape"].items())
    peaks, src = load_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    issue = None
    wi = prof.get("warp_inst_per_walker_step")
    if wi:
        peak = sms * 4 * mhz * 1e6
        ach = wi * kernel_ws_s
        db = prof.get("dram_bytes_per_walker_step")
        issue = {"bound": "issue", "achieved": ach, "peak": peak, "unit": "warp-instructions/s",
                 "frac": ach / peak, "warp_instructions_per_walker_step": wi,
                 "traffic": None if db is None else db * ws_per_launch,
                 "traffic_scaling": "DRAM bytes per walker-step of the captured launch x walker-steps of an "
                                    "average launch here",
                 "peak_source": f"{sms} SMs x 4 issue slots x median SM clock under load ({mhz:.0f} MHz)",
                 "counts_kernel_sha": prof.get("kernel_sha"), "kernel_sha": sha, "stale": stale,
                 "counts_shape": prof.get("shape"), "shape_matches": shape_ok, "capture": prof.get("capture")}
    fp32 = None
    if f_alg is not None:
        ach = kernel_ws_s * f_alg / 1e12
        fp32 = {"bound": "fp32", "achieved": ach, "peak": fp32_peak_tflops, "unit": "TFLOP/s",
                "frac": ach / fp32_peak_tflops, "flops_per_walker_step": f_alg, "work_per_walker_step": work,
                "peak_source": "nz_probe_fma on this GPU (8 FFMA chains per thread)"}
    hbm = {"bound": "hbm", "achieved": state_bytes / (launch_ms * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
           "algorithmic_bytes_per_launch": state_bytes,
           "peak_source": f"{src} hbm_gbs" if src else "fallback 6.65 TB/s"}
    hbm["frac"] = hbm["achieved"] / hbm_peak
    return issue, fp32, hbm


def fp32_peak(lib, L, stream, sms):
    """FP32 FMA throughput of this GPU (TFLOP/s) from the probe kernel."""
    import torch
    out = torch.zeros(sms * 16, device="cuda")
    iters = 4096
    for _ in range(2):
        L.check(lib.nz_probe_fma(sms * 16, iters, out.data_ptr(), stream.cuda_stream), "probe")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    L.check(lib.nz_probe_fma(sms * 16, iters, out.data_ptr(), stream.cuda_stream), "probe")
    e1.record(stream)
    torch.cuda.synchronize()
    return sms * 16 * 256 * iters * 8 * 2 / (e0.elapsed_time(e1) * 1e-3) / 1e12


def workload_packed():
    from nozomi_b200.workloads import packed_workload
    return packed_workload()


# ---------------------------------------------------------------------------
# CPU side: the oracle on the host cores
# ---------------------------------------------------------------------------
def cpu_sample(sub, pg, dirs, cell, seconds, rank_seed=0, work=True):
    """Time the oracle (the C restatement, OpenMP over walkers) on a bounded
    sample of one substrate and protocol, sized to about `seconds` of work.
    Returns (walker-steps/s, cores, sample description, work per walker-step:
    iterations, spheres and solves within reach, from the oracle's count
    mode on up to 2048 walkers x 200 steps)."""
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


REF_CPU_KIND = ("the reference's own sim3d_kernel.cu (randomWalk3d_phase_multidirr, template filled as DiffSim3d "
                "does, padded set_segments table at 1 um cells) compiled for the CPU with host stand-ins for its "
                "CUDA headers (oracle/refshim): each kernel launch runs its 1000-thread blocks as OpenMP "
                "iterations over walkers; curand_normal reads the oracle's Philox normals")


class ReferenceCpu:
    """A named CPU build of the reference kernel (oracle/_ref) walking its
    walkers (seeded over the whole substrate) through a protocol, launch by
    launch, as DwiSim3d.simulate_multi_directions does."""

    def __init__(self, build: str, sub, gwave, dirs, key=1000):
        import ctypes
        from oracle import oracle as oz
        from oracle.build import reference_named
        b = reference_named(build)
        if b is None:
            raise FileNotFoundError(f"oracle/_ref build {build} is absent")
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
            raise ValueError(f"the reference CPU build {build} does not match this substrate")
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
        self.dd = np.ascontiguousarray(np.asarray(dirs, np.float32))
        self.G, self.Ga = step_tables(gwave)
        self.dt = float(gwave.dt)
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


def reference_cases(workload: str):
    """(build name, substrate, waveform, directions) the reference arm walks:
    the packed workload, or jobs 0, 16, 32, 48 of the batched mixed workload."""
    if workload == "packed":
        sub, pg, dirs, _ = workload_packed()
        return [("packed_cpu_16k", sub, pg, dirs)], "the packed workload"
    from baseline.reference_gpu import BATCH_SAMPLE_JOBS
    from nozomi_b200.workloads import mixed_specs
    specs = mixed_specs(seed=4, n_jobs=64)
    cases = [(f"batched_job{i}_cpu_8k", specs[i].substrate, specs[i].gwave, np.asarray(specs[i].dirs))
             for i in BATCH_SAMPLE_JOBS]
    return cases, f"jobs {', '.join(map(str, BATCH_SAMPLE_JOBS))} of the batched workload"


def reference_cpu_sample(cases, seconds, steps=1, warmup=0):
    """Time the reference kernel's CPU builds: per step, every case for about
    seconds / len(cases).  Returns (walker-steps/s, cores, sample text, ms
    per timed step)."""
    cores = os.cpu_count() or 1
    refs = [ReferenceCpu(b, sub, gw, dirs) for b, sub, gw, dirs in cases]
    per = []
    for r in refs:
        t = time.perf_counter()
        r.run(3)
        rate = r.N * 3 / (time.perf_counter() - t)
        per.append(int(np.clip(seconds / len(refs) * rate / r.N, 3, r.G.size)))
    for r, k in zip(refs, per):
        r.run(k * warmup)
    t = time.perf_counter()
    for _ in range(steps):
        for r, k in zip(refs, per):
            r.run(k)
    el = time.perf_counter() - t
    ws = steps * sum(r.N * k for r, k in zip(refs, per))
    sample = "; ".join(f"{b}: {r.N} walkers x {k} launches per step, padded K={r.K}"
                       for (b, *_), r, k in zip(cases, refs, per))
    return ws / el, cores, f"{sample}; {steps} step(s), {el:.1f} s", el * 1e3 / steps


def port_sample(cases, seconds, cell=1.0, steps=1, warmup=0):
    """The oracle's C restatement on the same cases (no reference build)."""
    total_t, total_ws, texts, cores = 0.0, 0, [], 1
    for i in range(warmup + steps):
        for _, sub, gw, dirs in cases:
            v, cores, sample, _ = cpu_sample(sub, gw, dirs, cell, seconds / len(cases), rank_seed=i, work=False)
            if i >= warmup:
                total_ws += 1
                total_t += 1.0 / v
                texts.append(sample)
    return total_ws / total_t, cores, "; ".join(texts[:len(cases)])


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    workload = "packed" if args.workload == "packed" else "batched"
    cases, what = reference_cases(workload)
    from oracle.build import build_oracle
    build_oracle()
    try:
        value, cores, sample, ms_step = reference_cpu_sample(cases, args.cpu_seconds / 2, steps=args.steps,
                                                             warmup=args.warmup)
        kind, how = "reference", REF_CPU_KIND
    except (FileNotFoundError, ValueError) as e:  # no reference build on this host: the C restatement
        value, cores, sample = port_sample(cases, args.cpu_seconds / 2, steps=args.steps, warmup=args.warmup)
        ms_step = None  # samples of differing walker counts: no common step time
        kind, how = "port", f"oracle/walk_oracle.c, the C restatement of the kernel, OpenMP over walkers ({e})"
    wl = WORKLOAD if workload == "packed" else BATCH_WORKLOAD.format(jobs=args.jobs, scale=args.walker_scale,
                                                                       a0=args.axons[0], a1=args.axons[1])
    line = {"impl": "reference", "metric": "walker-steps/s", "value": value, "unit": "walker-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak" if workload == "packed" else "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl, "cell_um": 1.0, "sampled": what},
            "cpu_baseline": {"value": value, "unit": "walker-steps/s", "cores": cores, "kind": kind,
                             "sample": f"{what}: {sample}; {how}"},
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


def run_packed(args):
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
        init_process_group(args.dist_backend, timeout_s=180)
    engine.require_cuda()
    sub, pg, dirs, bvals = workload_packed()
    # launch shape tuned for this workload by sweeps on a B200: 0.5 um cells,
    # near margin 0.5 um, re-binning bins of 8^3 cells, 2000 steps per launch
    tuning = _tuning_from_args(args, Tuning(cell=0.5, near_margin=0.5, coarsen=8, steps_per_launch=2000))
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=tuning.cell, near_margin=tuning.near_margin,
                            lists=tuning.lists, near_shape=tuning.near_shape)
    # the one-time cell build (member lists, near lists, per-entry records) is
    # outside the metric; it is timed on a second build, the first having
    # loaded the library and warmed the allocator
    torch.cuda.synchronize()
    tb = time.perf_counter()
    dsub = device_substrate(sub, D=2.0, T2=100.0, cell=tuning.cell, near_margin=tuning.near_margin,
                            lists=tuning.lists, near_shape=tuning.near_shape)
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
    lib = L.load()
    fp32_peak_tflops = fp32_peak(lib, L, stream, sms)

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

    # end to end through the public call with host buffers: the shard's
    # prepare() copies the positions and labels from pinned host memory,
    # walk() launches the re-bins and fused walks eagerly, signal_sums()
    # reduces (and all-reduces over ranks); the sums are copied back
    x_host = x0.cpu().pin_memory()
    lab_host = lab0.cpu().pin_memory()
    e2e_ms = 0.0
    out_bytes = 0
    host = torch.empty_like(sig_static, device="cpu").pin_memory()
    for i in range(args.e2e_steps + 1):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = shard.prepare(x_host, lab_host).walk().signal_sums()
        host.copy_(out, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        out_bytes = host.numel() * host.element_size()
        if i > 0:  # first pass warms the path
            e2e_ms += e0.elapsed_time(e1)
    t_local = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    e2e_value = ws_per_step * args.e2e_steps / (float(t_local[0]) * 1e-3) if args.e2e_steps else None
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
                v, cores, sample, _ = reference_cpu_sample(reference_cases("packed")[0], args.cpu_seconds / 2)
                cpu = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "reference",
                       "sample": sample + "; " + REF_CPU_KIND, "port": port}
            except (FileNotFoundError, ValueError) as e:
                cpu = dict(port, reference_unavailable=str(e))
        F_alg = None
        if wk is not None:
            F_alg = 10 * wk["spheres_in_reach"] + 36 * wk["solves_in_reach"] + 6 * dirs.shape[1]
        # walker state read and written once per launch (4 x float4 each way)
        roof_issue, roof_fp32, roof_hbm = rooflines(
            "packed", kernel_ws_s, per_launch_ws, walk_launch_ms, N * 128, clk, sms, fp32_peak_tflops, F_alg, wk,
            shape={"cell": tuning.cell, "near_margin": tuning.near_margin, "coarsen": tuning.coarsen, "threads": 128,
                   "lists": tuning.lists, "near_shape": tuning.near_shape, "stage": 0})
        line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded packed-axon substrate, seeded walkers)",
                "config": {"workload": WORKLOAD, "walkers_per_gpu": N, "time_steps": run.nsteps,
                           "directions": int(dirs.shape[1]), "bvalues": bvals.tolist(),
                           "cell_um": tuning.cell, "steps_per_launch": tuning.steps_per_launch,
                           "rebin_coarsen": tuning.coarsen, "rebin_by_label": tuning.by_label,
                           "near_margin_um": tuning.near_margin, "lists": tuning.lists,
                           "near_shape": tuning.near_shape,
                           "near_list_entries": int(dsub.near[2].numel()) if dsub.near is not None else 0,
                           "spheres": sub.S, "cells": dsub.ncell,
                           "cell_list_entries": dsub.n_items, "l2": "256 MiB flush between timed steps",
                           "parallelism": f"walkers sharded over {world} GPU(s) by walker-id range; "
                                          "one all-reduce of the signal sums per step"},
                "e2e": None if e2e_value is None else {
                    "value": e2e_value, "unit": "walker-steps/s",
                    "h2d_bytes_per_step": int(x_host.numel() * x_host.element_size()
                                              + lab_host.numel() * lab_host.element_size()),
                    "d2h_bytes_per_step": int(out_bytes),
                    "call": "ShardedDwiRun.prepare(host positions, labels).walk().signal_sums(), eager"},
                "gpu_launches": launches_per_step * args.steps,
                "kernel": {"name": "walk_fused_kernel", "launches": n_walk, "avg_launch_ms": walk_launch_ms,
                           "walker_steps_per_launch": per_launch_ws, "kernel_walker_steps_per_s": kernel_ws_s,
                           "share_of_step": walk_ms / eager_ms, "eager_step_ms": eager_ms,
                           "timing": "value from CUDA-graph replays of the step; kernel figures from one eager "
                                     "step with events around each fused launch"},
                "cell_build": {"ms": cell_build_ms, "timing": "wall clock of one device_substrate build "
                               "(host preparation, cell and near lists, per-entry records), synchronised on "
                               "both sides; once per substrate, not part of value"},
                "roofline": roof_issue, "roofline_fp32": roof_fp32, "roofline_hbm": roof_hbm,
                "cpu_baseline": cpu, "clocks": clk,
                "signal_b0_mean": float(np.mean(np.abs(S[:, 0]))),
                "signal_mean_by_b": [float(np.mean(S[:, b].real)) for b in range(S.shape[1])]}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _tuning_from_args(args, base):
    if args.cell:
        base.cell = args.cell
    if args.steps_per_launch:
        base.steps_per_launch = args.steps_per_launch
    if args.coarsen:
        base.coarsen = args.coarsen
    if args.by_label is not None:
        base.by_label = bool(args.by_label)
    if args.near_margin is not None:
        base.near_margin = args.near_margin if args.near_margin > 0 else None
    if args.lists:
        base.lists = args.lists
    if args.near_shape:
        base.near_shape = args.near_shape
    if args.stage is not None:
        base.stage = args.stage
    return base


def plain_leg(specs, positions, sig_batched, every: int):
    """The plain per-substrate path on every `every`-th job, one job after
    another (1 um cells): (walker-steps/s, jobs timed, walker-steps timed,
    largest |S_plain - S_batched|)."""
    import torch
    from nozomi_b200.batch import SubstrateCache
    from nozomi_b200.plain import run_plain
    from nozomi_b200.simulate import Tuning
    stream = torch.cuda.current_stream()
    sel = list(range(0, len(specs), max(1, every)))
    ms, ws, err = 0.0, 0, 0.0
    tuning, cache = Tuning(), SubstrateCache()
    for i in sel:
        sp = specs[i]
        dsub = cache.get(sp.key, sp.substrate, sp.D, sp.T2, tuning)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = run_plain(dsub, sp, positions[i][0])
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        ws += sp.N * sp.nsteps
        o = out.cpu().numpy()
        err = max(err, float(np.abs((o[0] + 1j * o[1]) / sp.N - sig_batched[i]).max()))
    return ws / (ms * 1e-3), len(sel), ws, err


def serving_leg(pairs, tuning, threads, max_requests=None, max_backlog_s=None):
    """Poisson request streams (configs of the mixed workload's distribution,
    substrates reused with probability 0.7) through the continuous-batching
    server, one stream per (rate, window).  Returns per-rate statistics,
    substrate cache hits/misses and the host seconds spent generating the
    streams' substrates."""
    import torch
    from nozomi_b200.batch import SubstrateCache
    from nozomi_b200.serve import Server, latency_stats
    from nozomi_b200.workloads import request_stream
    cache = SubstrateCache()
    per_rate, done_all = [], []
    gen_s = 0.0
    for rate, window in pairs:
        t0 = time.perf_counter()
        reqs = request_stream(rate, window, seed=5, max_requests=max_requests)
        gen_s += time.perf_counter() - t0
        srv = Server(tuning=tuning, threads=threads, cache=cache, max_backlog_s=max_backlog_s)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = srv.serve(reqs)
        wall = time.perf_counter() - t0
        st = latency_stats(done)
        st.update({"rate_req_s": rate, "arrival_window_s": window, "requests": len(reqs),
                   "walker_steps": srv.walker_steps, "walker_steps_per_s": srv.walker_steps / wall, "wall_s": wall,
                   "rounds": srv.rounds, "failed": sum(t.error is not None and not t.shed for t in done),
                   "shed": sum(t.shed for t in done), "max_backlog_s": max_backlog_s})
        per_rate.append(st)
        done_all += done
    return per_rate, {"hits": cache.hits, "misses": cache.misses}, gen_s, done_all


def run_batched(args):
    import torch
    import torch.distributed as dist
    from nozomi_b200 import engine, _lib as L
    from nozomi_b200.batch import BatchRun, SubstrateCache, simulate_batch
    from nozomi_b200.shard import init_process_group, shard_jobs
    from nozomi_b200.simulate import Tuning
    from nozomi_b200.workloads import mixed_specs
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        init_process_group(args.dist_backend, timeout_s=180)
    engine.require_cuda()
    t0 = time.perf_counter()
    all_specs = mixed_specs(seed=4, n_jobs=args.jobs, walker_scale=args.walker_scale, axons=tuple(args.axons))
    gen_s = time.perf_counter() - t0
    # over several GPUs the jobs shard whole, longest first onto the least
    # loaded rank; no data crosses ranks (strong scaling of a fixed batch)
    mine = shard_jobs([sp.walker_steps for sp in all_specs], world)[rank] if world > 1 else range(len(all_specs))
    specs = [all_specs[i] for i in mine]
    tuning = _tuning_from_args(args, Tuning())
    tune_report = None
    threads = args.threads
    if not args.no_autotune:  # the launch shape from the autotuner's short trials (cached per GPU and workload)
        from nozomi_b200.autotune import autotune
        t0 = time.perf_counter()
        tuning, threads, tune_report = autotune(specs)
        tune_report["seconds"] = time.perf_counter() - t0
        tuning = _tuning_from_args(args, tuning)
    cache = SubstrateCache()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run = BatchRun(specs, tuning=tuning, threads=threads, cache=cache)
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    positions = run.seed_positions()
    run.positions = positions
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    lib = L.load()
    fp32_peak_tflops = fp32_peak(lib, L, stream, sms)
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(max(1, args.warmup)):
        run.step()
        flush.zero_()
    barrier()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        run.step()
    graph.replay()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    ms = 0.0
    for _ in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (outside the step's events)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        graph.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    barrier()
    clk = clocks.stop()
    del graph
    sig_batched = run.signals()

    # the same step launched eagerly with CUDA events around every batched
    # walk launch: the dominant kernel's average launch and its share
    ev = []
    flush.zero_()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.prepare().run(events=ev)
    e1.record(stream)
    torch.cuda.synchronize()
    eager_ms = e0.elapsed_time(e1)
    walk_ms = sum(a.elapsed_time(b) for a, b in ev)
    chunk_ws = [c["walker_steps"] for c in run.chunks]

    # end to end through the public call: positions from pinned host memory,
    # the batch planned, walked and reduced, the signals copied back
    host_pos = [(x.cpu().pin_memory(), lab.cpu().pin_memory()) for x, lab in positions]
    e2e_ms, io = 0.0, {}
    for i in range(args.e2e_steps + 1):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sig_e2e = simulate_batch(specs, positions=host_pos, tuning=tuning, threads=threads, cache=cache, stats=io)
        e1.record(stream)
        torch.cuda.synchronize()
        if i > 0:  # the first pass warms the path
            e2e_ms += e0.elapsed_time(e1)
    e2e_diff = max(float(np.abs(a - b).max()) for a, b in zip(sig_e2e, sig_batched))

    t_local = torch.tensor([ms, e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t_local, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t_local[0]), float(t_local[1])
    ws = sum(sp.walker_steps for sp in all_specs)
    value = ws * args.steps / (ms * 1e-3)
    e2e_value = ws * args.e2e_steps / (e2e_ms * 1e-3) if args.e2e_steps else None
    kernel_ws_s = sum(chunk_ws) / (walk_ms * 1e-3)
    wl = BATCH_WORKLOAD.format(jobs=len(all_specs), scale=args.walker_scale, a0=args.axons[0], a1=args.axons[1])
    config = {"workload": wl, "jobs": len(all_specs), "walker_steps_per_step": ws,
              "walkers": sum(sp.N for sp in all_specs), "threads": threads,
              "steps_per_launch": tuning.steps_per_launch, "near_margin_um": tuning.near_margin,
              "cell_um": tuning.cell, "rebin_coarsen": tuning.coarsen, "rebin_by_label": tuning.by_label,
              "lists": tuning.lists, "near_shape": tuning.near_shape, "stage_records": tuning.stage,
              "persistent_grid": run.grid, "chunks": len(run.chunks),
              "l2": "256 MiB flush between timed steps (the inputs, 64 substrates' cell lists and walker "
                    "state, are also larger than L2)",
              "parallelism": (f"jobs sharded whole over {world} GPUs, longest first" if world > 1 else "one GPU")}
    e2e = None if e2e_value is None else {
        "value": e2e_value, "unit": "walker-steps/s", "h2d_bytes_per_step": int(io.get("h2d_bytes", 0)),
        "d2h_bytes_per_step": int(io.get("d2h_bytes", 0)),
        "call": "nozomi_b200.batch.simulate_batch(specs, positions=pinned host arrays): protocol tables, job, "
                "item and re-binning tables built and uploaded, walkers packed, every chunk re-binned and walked "
                "(eager launches), signals reduced and copied back; cell lists from a warm substrate cache",
        "max_signal_diff_vs_graph": e2e_diff}
    launch_ms = walk_ms / max(len(ev), 1)
    ws_launch = sum(chunk_ws) / max(len(chunk_ws), 1)
    state_bytes = 128 * sum(c["sort_walkers"] for c in run.chunks) / max(len(run.chunks), 1)
    shape = {"cell": tuning.cell, "near_margin": tuning.near_margin, "coarsen": tuning.coarsen, "threads": threads,
             "lists": tuning.lists, "near_shape": tuning.near_shape, "stage": tuning.stage}
    if world > 1:
        if rank == 0:
            # the issue roofline of rank 0's own batched launches (the host-core
            # baseline and its work counts are measured at N=1 only)
            roof_issue = rooflines("batched", kernel_ws_s, ws_launch, launch_ms, state_bytes, clk, sms,
                                   fp32_peak_tflops, None, None, shape=shape)[0]
            print(json.dumps({"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                              "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                              "data": "synthetic (seeded substrates, protocols and walkers)", "config": config,
                              "e2e": e2e, "gpu_launches": run.launches() * args.steps,
                              "kernel": {"name": "walk_fused_kernel (batched form, nz_walk_batch), rank 0",
                                         "launches": len(ev), "avg_launch_ms": launch_ms,
                                         "kernel_walker_steps_per_s": kernel_ws_s},
                              "roofline": roof_issue, "cpu_baseline": None, "clocks": clk}), flush=True)
        dist.barrier()
        dist.destroy_process_group()
        return 0

    plain = None
    if not args.no_plain:
        pv, pjobs, pws, perr = plain_leg(specs, positions, sig_batched, args.plain_every)
        plain = {"value": pv, "unit": "walker-steps/s", "jobs_timed": pjobs, "every": args.plain_every,
                 "walker_steps_timed": pws, "cell_um": 1.0, "max_signal_diff_vs_batched": perr,
                 "launch": "one plain-kernel launch per waveform sample from the host, per-direction phase in "
                           "HBM, jobs one after another (every k-th job of the batch)"}
    serving = None
    if not args.no_serving:
        pairs = [tuple(float(v) for v in p.split(":")) for p in args.serve.split(",") if p]
        stune = Tuning(cell=args.serve_cell or tuning.cell, coarsen=args.serve_coarsen or tuning.coarsen,
                       near_margin=tuning.near_margin, by_label=tuning.by_label)
        per_rate, sc, sgen, _ = serving_leg(pairs, stune, threads, args.max_requests, args.serve_max_backlog)
        serving = {"per_rate": per_rate, "substrate_cache": sc, "substrate_generation_s": sgen,
                   "cell_um": stune.cell, "rebin_coarsen": stune.coarsen,
                   "rounds": "time-bounded (about 50 ms at the measured throughput, 100-4000 steps)",
                   "admission": "side stream, overlapping the running round"}
        if plain:
            for r in per_rate:
                r["speedup_vs_plain"] = r["walker_steps_per_s"] / plain["value"]
    cpu, wk_all = None, None
    if not args.no_cpu_baseline:
        cases, what = reference_cases("batched")
        try:
            v, cores, sample, _ = reference_cpu_sample(cases, args.cpu_seconds / 2)
            cpu = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "reference",
                   "sample": f"{what}: {sample}; {REF_CPU_KIND}"}
        except (FileNotFoundError, ValueError) as e:
            v, cores, sample = port_sample(cases, args.cpu_seconds / 2)
            cpu = {"value": v, "unit": "walker-steps/s", "cores": cores, "kind": "port",
                   "sample": f"{what}: {sample}; oracle/walk_oracle.c, OpenMP over walkers",
                   "reference_unavailable": str(e)}
        # algorithmic work per walker-step from the oracle's count mode on the
        # sampled jobs (the lists of the batch's cell size)
        works = [cpu_sample(sub, gw, dirs, tuning.cell, 0.5, work=True)[3] for _, sub, gw, dirs in cases]
        wk_all = {k: float(np.mean([w[k] for w in works])) for k in works[0]}
    ndir_mean = sum(sp.walker_steps * np.asarray(sp.dirs).shape[1] for sp in specs) / ws
    F_alg = None if wk_all is None else 10 * wk_all["spheres_in_reach"] + 36 * wk_all["solves_in_reach"] + 6 * ndir_mean
    roof_issue, roof_fp32, roof_hbm = rooflines(
        "batched", kernel_ws_s, ws_launch, launch_ms, state_bytes, clk, sms, fp32_peak_tflops, F_alg, wk_all,
        shape=shape)
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded substrates, protocols and walkers)", "config": config,
            "speedup_vs_plain": None if plain is None else value / plain["value"],
            "plain": plain, "serving": serving, "e2e": e2e,
            "gpu_launches": run.launches() * args.steps,
            "kernel": {"name": "walk_fused_kernel (batched form, nz_walk_batch)", "launches": len(ev),
                       "avg_launch_ms": launch_ms, "walker_steps_per_launch": ws_launch,
                       "kernel_walker_steps_per_s": kernel_ws_s, "share_of_step": walk_ms / eager_ms,
                       "eager_step_ms": eager_ms, "walker_steps_per_chunk": chunk_ws,
                       "timing": "value from CUDA-graph replays of the step; kernel figures from one eager "
                                 "step with events around each batched launch"},
            "setup": {"substrate_generation_s": gen_s, "device_substrates_s": build_s,
                      "timing": "host generation of the 64 seeded substrates and their one-time device cell "
                                "lists (wall clock); not part of value"},
            "autotune": None if tune_report is None else {
                "cached": tune_report["cached"], "choice": {"threads": threads, **dataclasses.asdict(tuning)},
                "trials": len(tune_report.get("trials", [])), "seconds": tune_report.get("seconds"),
                "trial_walker_steps_per_s": tune_report.get("trial_walker_steps_per_s")},
            "roofline": roof_issue, "roofline_fp32": roof_fp32, "roofline_hbm": roof_hbm,
            "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


def run_serving(args):
    """The request streams alone (--serve rate:window pairs), with the plain
    kernel timed on a sample of the served requests."""
    import torch
    if int(os.environ.get("RANK", "0")) != 0:  # a one-GPU request loop
        return 0
    from nozomi_b200 import engine
    from nozomi_b200.batch import SubstrateCache
    from nozomi_b200.plain import run_plain
    from nozomi_b200.simulate import Tuning
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    engine.require_cuda()
    tuning = _tuning_from_args(args, Tuning())
    if args.serve_cell:
        tuning.cell = args.serve_cell
    if args.serve_coarsen:
        tuning.coarsen = args.serve_coarsen
    pairs = [tuple(float(v) for v in p.split(":")) for p in args.serve.split(",") if p]
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    per_rate, sc, sgen, all_done = serving_leg(pairs, tuning, args.threads, args.max_requests, args.serve_max_backlog)
    clk = clocks.stop()
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
    value = sum(r["walker_steps"] for r in per_rate) / sum(r["wall_s"] for r in per_rate)
    line = {"metric": "walker-steps/s", "value": value, "unit": "walker-steps/s", "n_gpus": 1,
            "steps": len(per_rate), "warmup": 0, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded Poisson request streams)",
            "config": {"workload": "serving: Poisson arrivals per rate, substrates of 10-500 beaded axons reused "
                                   "with probability 0.7, 1e4-5e5 walkers, 2000-8000 steps at 5 us, 6-60 directions, "
                                   "b<=3 ms/um^2, seed 5", "rates_and_windows": args.serve,
                       "max_requests_per_rate": args.max_requests, "max_backlog_s": args.serve_max_backlog,
                       "threads": args.threads,
                       "cell_um": tuning.cell, "rebin_coarsen": tuning.coarsen},
            "per_rate": per_rate, "substrate_generation_s": sgen,
            "plain": {"value": plain_value, "unit": "walker-steps/s", "requests_timed": len(sample),
                      "launch": "one plain-kernel launch per step, requests one after another"},
            "speedup_vs_plain": value / plain_value, "substrate_cache": sc, "clocks": clk}
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
    sub, pg, dirs, bvals = workload_packed()
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


def main(argv=None):
    args = parse(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference_gpu":
        return run_reference_gpu(args)
    if args.workload == "packed":
        return run_packed(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "narrow":
        return run_narrow(args)
    return run_batched(args)


if __name__ == "__main__":
    sys.exit(main())
