"""Synthetic mixed workloads (seeded): many beaded-axon substrates of uneven
size under per-substrate PGSE protocols.

* ``mixed_specs`` — the batched workload: substrates built like the single
  beaded axon (40 spheres at 1 um, radii U[0.5, 1.5], z-periodic) but with
  axon counts uniform in [10, 500] packed in a periodic box; walker counts
  log-uniform in [1e4, 1e6] (rounded to 1000); step counts uniform in
  [2000, 8000] at dt = 5 us with PGSE delta = te/3, Delta = 2 te/3; 6 to 60
  directions uniform on the sphere; b in {0, 1, 2, 3} ms/um^2.
* ``request_stream`` — the served workload: Poisson arrivals; each request
  draws a substrate from the same distribution (an earlier one again with
  probability 0.7), 1e4 to 5e5 walkers log-uniform, 6 to 60 directions,
  b up to 3 ms/um^2.
Substrates are cached on disk under ~/.cache/nozomi_b200 (they take seconds
to pack).
"""
from __future__ import annotations

import hashlib
import os
import pickle
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .batch import JobSpec
from .substrates import Substrate, axon_bundle
from .waveforms import PGDiffWaveform

CACHE = Path(os.environ.get("NOZOMI_B200_CACHE", Path.home() / ".cache" / "nozomi_b200"))
DT = 0.005


def packed_workload():
    """The packed-substrate workload: 200 beaded axons x 100 spheres in a
    periodic 40x40x80 um box (seed 2), PGSE 20/10/30 ms at dt = 5 us (6000
    steps), 30 directions uniform on the sphere (seed 2), b in {0,1,2,3}
    ms/um^2.  Returns (substrate, waveform, dirs [3,30], b-values)."""
    from . import substrates as sb
    sub = sb.packed_axons(seed=2)
    pg = PGDiffWaveform(20.0, 10.0, 30.0, time_step=0.005)
    rng = np.random.default_rng(2)
    dirs = rng.standard_normal((3, 30))
    dirs /= np.linalg.norm(dirs, axis=0)
    return sub, pg, dirs, np.array([0.0, 1.0, 2.0, 3.0])


def _store(path, obj):
    """Pickle obj to path through a file of this process's own, renamed into
    place: ranks that build the same cached substrate at once never see or
    rename one another's partial files."""
    tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp")
    with open(tmp, "wb") as f:
        pickle.dump(obj, f)
    os.replace(tmp, path)


def calibration_substrate() -> Substrate:
    """A stand-in for the reference's segment-calibration substrate
    (VF0.65_d1.68_OD200_bead1.0_500axons, docs/2_calibration.md:98-108):
    500 beaded axons, base diameter lognormal (mean 1.68 um, sd 0.45 um),
    beads of +20-50 % radius every 5.7 um, spheres every 0.5 um, packed
    parallel (no orientation dispersion) in a periodic 50 um cube to a
    volume fraction of 0.65 (seed 7).  About a minute to pack; cached."""
    from .substrates import packed_axons
    CACHE.mkdir(parents=True, exist_ok=True)
    path = CACHE / "calibration_500axons_v1.pkl"
    if path.exists():
        with open(path, "rb") as f:
            return pickle.load(f)
    s = packed_axons(n_axons=500, L=(50.0, 50.0, 50.0), spheres_per_axon=100, r_mean=0.84, r_sd=0.225,
                     bead_amp=(0.2, 0.5), bead_spacing=5.7, r_min=0.3, seed=7, max_iter=3000)
    _store(path, s)
    return s


def _bundle_key(n_axons: int, seed: int) -> str:
    return hashlib.sha1(f"axon_bundle-v2-{n_axons}-{seed}".encode()).hexdigest()[:16]


def bundle(n_axons: int, seed: int) -> Substrate:
    CACHE.mkdir(parents=True, exist_ok=True)
    path = CACHE / f"bundle_{_bundle_key(n_axons, seed)}.pkl"
    if path.exists():
        with open(path, "rb") as f:
            return pickle.load(f)
    s = axon_bundle(n_axons, seed)
    _store(path, s)
    return s


def pgse(steps: int, dt: float = DT) -> PGDiffWaveform:
    te = steps * dt
    return PGDiffWaveform(2 * te / 3, te / 3, te, time_step=dt)


def unit_directions(rng, n: int) -> np.ndarray:
    d = rng.standard_normal((3, n))
    return d / np.linalg.norm(d, axis=0)


def mixed_specs(seed: int = 4, n_jobs: int = 64, axons=(10, 500), walkers=(1e4, 1e6), steps=(2000, 8000),
                ndirs=(6, 60), bvalues=(0.0, 1.0, 2.0, 3.0), walker_scale: float = 1.0) -> list:
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_jobs):
        na = int(rng.integers(axons[0], axons[1] + 1))
        N = int(max(1000, round(np.exp(rng.uniform(np.log(walkers[0]), np.log(walkers[1]))) * walker_scale / 1000)
                    * 1000))
        nst = int(rng.integers(steps[0], steps[1] + 1))
        nd = int(rng.integers(ndirs[0], ndirs[1] + 1))
        gw = pgse(nst)
        dirs = unit_directions(rng, nd)
        amps = gw.amplitude_for_b(np.asarray(bvalues))
        specs.append(JobSpec(bundle(na, seed * 1000 + i), gw, dirs, amps, N, seed=seed * 100000 + i,
                             key=("bundle", na, seed * 1000 + i)))
    return specs


@dataclass
class Request:
    arrival: float       # seconds after the stream starts
    spec: JobSpec


def request_stream(rate: float, duration: float, seed: int = 5, reuse: float = 0.7, axons=(10, 500),
                   walkers=(1e4, 5e5), steps=(2000, 8000), ndirs=(6, 60), bmax: float = 3.0,
                   max_requests: int | None = None, workers: int | None = None) -> list:
    """Requests of a Poisson stream at `rate` per second over `duration`
    seconds (at most max_requests).  A request reuses an earlier request's
    substrate with probability `reuse`; requests of one substrate share one
    Substrate object.  Substrates not yet in the disk cache are generated
    first, by `workers` processes (default: up to 16 when more than 8 are
    missing); the stream is the same whatever the number of workers."""
    rng = np.random.default_rng(seed)
    t, drawn, seen = 0.0, [], []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and len(drawn) >= max_requests):
            break
        if seen and rng.uniform() < reuse:
            na, sseed = seen[int(rng.integers(len(seen)))]
        else:
            na, sseed = int(rng.integers(axons[0], axons[1] + 1)), int(rng.integers(1 << 30))
            seen.append((na, sseed))
        N = int(max(1000, round(np.exp(rng.uniform(np.log(walkers[0]), np.log(walkers[1]))) / 1000) * 1000))
        nst = int(rng.integers(steps[0], steps[1] + 1))
        nd = int(rng.integers(ndirs[0], ndirs[1] + 1))
        b = np.linspace(0.0, rng.uniform(1.0, bmax), 4)
        dirs = unit_directions(rng, nd)
        drawn.append((t, na, sseed, N, nst, dirs, b, int(rng.integers(1 << 31))))
    subs = bundles(seen, workers)
    out = []
    for t, na, sseed, N, nst, dirs, b, rseed in drawn:
        gw = pgse(nst)
        spec = JobSpec(subs[(na, sseed)], gw, dirs, gw.amplitude_for_b(b), N, seed=rseed, key=("bundle", na, sseed))
        out.append(Request(t, spec))
    return out


def _bundle_args(args):
    return bundle(*args)


def bundles(keys, workers: int | None = None) -> dict:
    """{(n_axons, seed): bundle(n_axons, seed)} for every key; the ones not
    in the disk cache are generated in `workers` spawned processes when
    there are more than 8 of them (workers None: up to 16)."""
    keys = list(dict.fromkeys(keys))
    missing = [k for k in keys if not (CACHE / f"bundle_{_bundle_key(*k)}.pkl").exists()]
    if workers is None:
        workers = min(16, os.cpu_count() or 1) if len(missing) > 8 else 1
    if workers > 1 and missing:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            list(ex.map(_bundle_args, missing, chunksize=4))  # written to the disk cache
    return {k: bundle(*k) for k in keys}
