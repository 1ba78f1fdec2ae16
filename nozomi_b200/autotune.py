"""Launch-shape autotuner for the batched walk.

Chooses walkers per CTA (``threads``), cell edge, near-list margin, steps per
launch and re-binning coarsening by timing short trials of the batch itself:
at most ``max_jobs`` jobs (the largest), each cut to ``max_walkers`` walkers
and its first ``trial_steps`` steps.  The search is coordinate descent from
the defaults (each restricted to the search space), one parameter at a
time, keeping a change only if it is faster by more than ``min_gain``.  Choices are cached per (GPU, workload signature)
in a JSON file so later runs of the same shape skip the search.
"""
from __future__ import annotations

import dataclasses
import fcntl
import hashlib
import json
import os
import threading
from pathlib import Path

import numpy as np
import torch

from .batch import BatchRun, SubstrateCache
from .simulate import Tuning
from .waveforms import ArbitraryWaveform

SPACE = {
    "threads": [64, 128, 256],
    "cell": [0.4, 0.5, 0.667, 1.0, 1.5],
    "near_margin": [0.4, 0.5, 0.6, None],
    "steps_per_launch": [500, 1000, 2000, 4000],
    "coarsen": [4, 8, 12, 16],
}
CACHE_FILE = Path(os.environ.get("NOZOMI_B200_CACHE", Path.home() / ".cache" / "nozomi_b200")) / "autotune.json"


def signature(specs) -> str:
    """Workload shape: job count, walker/step/direction/sphere-count histograms, dt."""
    N = np.array([s.N for s in specs])
    st = np.array([s.nsteps for s in specs])
    nd = np.array([np.asarray(s.dirs).shape[1] for s in specs])
    S = np.array([s.substrate.S for s in specs])
    dts = sorted({round(float(s.gwave.dt), 6) for s in specs})
    q = lambda a: np.percentile(a, [10, 50, 90]).round(-2 if a.max() > 1000 else 0).tolist()  # noqa: E731
    key = json.dumps({"n": len(specs), "N": q(N), "steps": q(st), "dirs": q(nd), "S": q(S), "dt": dts})
    gpu = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return hashlib.sha1((gpu + key).encode()).hexdigest()[:16]


def load_choices(path: Path) -> dict:
    """Cached choices by signature; an unreadable or corrupt file is empty."""
    try:
        data = json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}
    return data if isinstance(data, dict) else {}


def cached_choice(path: Path, sig: str):
    """(Tuning, threads, entry) cached for `sig`, or None (absent, or written
    by a version with other Tuning fields)."""
    saved = load_choices(path).get(sig)
    try:
        return Tuning(**saved["tuning"]), int(saved["threads"]), saved
    except (TypeError, KeyError, ValueError):
        return None


def store_choice(path: Path, sig: str, entry: dict):
    """Add one signature's choice.  The read-modify-write runs under an
    exclusive lock on a sidecar file, so processes storing different
    signatures at once keep every entry; the file is replaced atomically from
    a temporary of this process and thread, so a reader never sees it half
    written."""
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path.with_name(path.name + ".lock"), "a") as lk:
        fcntl.flock(lk.fileno(), fcntl.LOCK_EX)
        try:
            data = load_choices(path)
            data[sig] = entry
            tmp = path.with_name(f"{path.name}.{os.getpid()}.{threading.get_ident()}.tmp")
            tmp.write_text(json.dumps(data, indent=1))
            os.replace(tmp, path)
        finally:
            fcntl.flock(lk.fileno(), fcntl.LOCK_UN)


def _trial_specs(specs, max_jobs, max_walkers, trial_steps):
    big = sorted(specs, key=lambda s: -s.walker_steps)[:max_jobs]
    out = []
    for s in big:
        w = np.asarray(s.gwave.wave)[:trial_steps]
        gw = ArbitraryWaveform(w, s.gwave.dt)
        out.append(dataclasses.replace(s, gwave=gw, N=min(s.N, max_walkers)))
    return out


def _time(specs, tuning, threads, cache, reps=2) -> float:
    run = BatchRun(specs, tuning=tuning, threads=threads, cache=cache)
    run.step()  # warm-up: allocations, cell lists, scratch
    stream = torch.cuda.current_stream()
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run.step()
        e1.record(stream)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return run.walker_steps() / (best * 1e-3)


def autotune(specs, space=None, trial_steps: int = 2000, max_walkers: int = 50_000, max_jobs: int = 16,
             min_gain: float = 0.02, use_cache: bool = True, cache_file: Path = CACHE_FILE):
    """Returns (Tuning, threads, report)."""
    space = space or SPACE
    sig = signature(specs)
    if use_cache:
        hit = cached_choice(cache_file, sig)
        if hit is not None:
            t, threads, saved = hit
            return t, threads, {"cached": True, "signature": sig, **saved}
    trial = _trial_specs(specs, max_jobs, max_walkers, trial_steps)
    cache = SubstrateCache()
    # start from the defaults, or a space's first value where it lacks the default
    default = {"threads": 128, "cell": 1.0, "near_margin": 0.5, "steps_per_launch": 500, "coarsen": 4}
    cur = {k: (v if v in space[k] else space[k][0]) for k, v in default.items()}
    trials = []

    def measure(cfg):
        t = Tuning(cell=cfg["cell"], near_margin=cfg["near_margin"], steps_per_launch=cfg["steps_per_launch"],
                   coarsen=cfg["coarsen"])
        v = _time(trial, t, cfg["threads"], cache)
        trials.append({**cfg, "walker_steps_per_s": v})
        return v

    best = measure(cur)
    # the cell edge first (the best re-binning coarsening and near margin depend on it)
    for name in ["cell", "coarsen", "near_margin", "threads", "steps_per_launch"]:
        for val in space[name]:
            if val == cur[name]:
                continue
            cand = dict(cur, **{name: val})
            v = measure(cand)
            if v > best * (1 + min_gain):
                best, cur = v, cand
    tuning = Tuning(cell=cur["cell"], near_margin=cur["near_margin"], steps_per_launch=cur["steps_per_launch"],
                    coarsen=cur["coarsen"])
    report = {"cached": False, "signature": sig, "tuning": dataclasses.asdict(tuning), "threads": cur["threads"],
              "trial_walker_steps_per_s": best, "trials": trials}
    if use_cache:
        store_choice(cache_file, sig, {"tuning": report["tuning"], "threads": cur["threads"],
                                       "trial_walker_steps_per_s": best})
    return tuning, cur["threads"], report
