"""The reference's own walk kernel on the GPU: a baseline, not the product.

nozomi runs its walk as CUDA through pycuda: DiffSim3d fills the %-template
of simulation_toolkit/simulation_engine/sim3d_kernel.cu with the run's
constants (diffsim3d.py:39, pars from :78-104 and :107-168), compiles it with
SourceModule's default options and launches one kernel per waveform sample
with block 1000 (:236-261).  pycuda is not installed here, so:

* ``build(name, pars)`` (needs the reference source tree; ``__graft_entry__.
  build()`` runs it where the tree is present) writes the substituted source
  to ``baseline/_ref/<name>.cu`` and compiles it with ``ref_gpu_harness.cu``
  (our launch shim) by nvcc for sm_100a with no optimisation flags beyond
  nvcc's defaults, like SourceModule, into ``baseline/_ref/<name>.so``, with
  ``<name>.json`` holding the pars.  ``baseline/_ref`` is git-ignored: the
  reference source never enters the repository.
* ``RefGpuWalk`` loads such a build and launches the unmodified kernels on
  device arrays the caller owns (torch tensors), with the reference's draws
  (cuRAND XORWOW states initialised by its ``initstates``).

``pars_for(...)`` forms the pars the way DiffSim3d does, from a substrate,
the walker count and the cell grid; the padded cell table comes from
nozomi_b200's ``nz_segments_fill`` (the reference's set_segments rule,
tested equal to it) and its K must equal the compiled ``nspheres_per_seg``.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the reference source tree: NOZOMI_REFERENCE_ROOT, else a folder named
# "reference" beside this repository
REFERENCE_ROOT = Path(os.environ.get("NOZOMI_REFERENCE_ROOT", HERE.parent.parent / "reference"))
KERNEL_REL = "simulation_toolkit/simulation_engine/sim3d_kernel.cu"
BLOCK = 1000  # DiffSim3d.set_block_grid (diffsim3d.py:170-172)


def reference_available() -> bool:
    return (REFERENCE_ROOT / KERNEL_REL).is_file()


def pars_for(sub, nspins: int, nseg, K: int, D: float = 2.0, T2: float = 100.0) -> dict:
    """Template constants as DiffSim3d.set_spins / set_geometry / set_segments
    form them (diffsim3d.py:78-104, 111-122, 166): python scalars, D and T2
    joined per structure with the box last."""
    Lx, Ly, Lz = (float(v) for v in sub.L)
    nx, ny, nz = (int(v) for v in nseg)
    ns = int(sub.nstructures)
    return {"nspins": int(nspins), "nspheres": int(sub.S), "nstructures": ns, "Lx": Lx, "Ly": Ly, "Lz": Lz,
            "dLx": Lx / nx, "dLy": Ly / ny, "dLz": Lz / nz, "nLx": nx, "nLy": ny, "nLz": nz,
            "D": ",".join(map(str, [float(D)] * (ns + 1))), "T2": ",".join(map(str, [float(T2)] * (ns + 1))),
            "nspheres_per_seg": int(K)}


def build(name: str, pars: dict, arch: str = "sm_100a") -> Path:
    """Substitute and compile; returns the .so path (rebuilt when the pars,
    the harness or the kernel source change)."""
    OUT.mkdir(parents=True, exist_ok=True)
    src = (REFERENCE_ROOT / KERNEL_REL).read_text() % pars
    harness = HERE / "ref_gpu_harness.cu"
    so = OUT / f"{name}.so"
    meta = OUT / f"{name}.json"
    stamp = {"pars": pars, "harness": harness.read_text(), "source_len": len(src), "arch": arch}
    if so.exists() and meta.exists():
        old = json.loads(meta.read_text())
        if old.get("stamp") == stamp:
            return so
    cu = OUT / f"{name}.cu"
    cu.write_text(src)
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    cmd = [nvcc, "-gencode", f"arch=compute_{arch[3:]},code={arch}", "-shared", "-Xcompiler", "-fPIC",
           f"-DNZ_REF_KERNEL_SOURCE=\"{cu}\"", "-o", str(so) + ".tmp", str(harness)]
    subprocess.run(cmd, check=True)
    os.replace(str(so) + ".tmp", so)
    meta.write_text(json.dumps({"pars": pars, "stamp": stamp}, indent=1))
    return so


def built(name: str):
    """(so path, pars) of a build in baseline/_ref, or None."""
    so, meta = OUT / f"{name}.so", OUT / f"{name}.json"
    if not (so.exists() and meta.exists()):
        return None
    return so, json.loads(meta.read_text())["pars"]


class RefGpuWalk:
    """The reference's randomWalk3d_phase_multidirr on device tensors."""

    def __init__(self, name: str):
        import torch
        b = built(name)
        if b is None:
            raise FileNotFoundError(f"baseline/_ref/{name}.so is not built (needs the reference source tree)")
        self.so, self.pars = b
        self.lib = ctypes.CDLL(str(self.so))
        P, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        self.lib.refgpu_last_error.restype = ctypes.c_char_p
        self.lib.refgpu_initstates.argtypes = [i, i, i, P]
        self.lib.refgpu_walk_multidir.argtypes = [f, P, P, P, P, P, f, f, P, i, i, i, P]
        self.lib.refgpu_walk.argtypes = [f, P, P, P, P, P, i, i, P]
        self.N = int(self.pars["nspins"])
        if self.N % BLOCK:
            raise ValueError("the reference's walk kernels need nspins to be a multiple of 1000")
        self.grid = self.N // BLOCK
        self.torch = torch

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _check(self, rc):
        if rc:
            raise RuntimeError(self.lib.refgpu_last_error().decode())

    def initstates(self, seed: int):
        self._check(self.lib.refgpu_initstates(int(seed), self.grid, BLOCK, self._stream()))

    def setup(self, spheres32, segments, K: int, positions, ndir: int, diffdir):
        """spheres32 [5,S] float32, segments [ncell*K] int32, positions [3,N]
        float32, diffdir [3,ndir] float32 (device tensors)."""
        if K != int(self.pars["nspheres_per_seg"]):
            raise ValueError(f"cell table K={K} but the build has nspheres_per_seg={self.pars['nspheres_per_seg']}")
        if positions.shape[1] != self.N or spheres32.shape[1] != int(self.pars["nspheres"]):
            raise ValueError("walker or sphere count differs from the build")
        t = self.torch
        self.spheres, self.segments = spheres32.contiguous(), segments.contiguous()
        self.spins = positions.clone().contiguous()
        self.spins0 = positions.clone().contiguous()
        self.ndir = int(ndir)
        self.diffdir = diffdir.contiguous()
        self.phase = t.zeros(self.ndir * self.N, dtype=t.float32, device=positions.device)
        return self

    def step(self, dt: float, G: float, Garea: float):
        p = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
        self._check(self.lib.refgpu_walk_multidir(dt, p(self.spheres), p(self.segments), p(self.spins),
                                                  p(self.spins0), p(self.phase), G, Garea, p(self.diffdir),
                                                  self.ndir, self.grid, BLOCK, self._stream()))


def member_counts(spheres64: np.ndarray, L, nseg, jump_tol: float = 1.0) -> np.ndarray:
    """Members per cell under set_segments' rule (diffsim3d.py:128-141:
    in_segment < jump_tol, float64, the reference's operation order),
    evaluated only on a window of cells around each sphere; cell id
    p*nx*ny + m*nx + n.  K is the maximum."""
    sx, sy, sz, sr = (np.asarray(spheres64[i], np.float64) for i in range(4))
    Lx, Ly, Lz = (float(v) for v in L)
    nx, ny, nz = (int(v) for v in nseg)
    dLx, dLy, dLz = Lx / nx, Ly / ny, Lz / nz
    counts = np.zeros(nx * ny * nz, np.int64)

    def window(c, r, d, Lh, n):
        lo = np.floor((c - r - jump_tol + Lh) / d).astype(np.int64) - 1
        return np.clip(lo, 0, n - 1)

    w = int(np.ceil((2 * sr.max() + 2 * jump_tol) / min(dLx, dLy, dLz))) + 3 if sr.size else 0
    x0, y0, z0 = window(sx, sr, dLx, Lx / 2, nx), window(sy, sr, dLy, Ly / 2, ny), window(sz, sr, dLz, Lz / 2, nz)
    for i in range(w):
        n = x0 + i
        inx = np.maximum(n * dLx - sr - sx - Lx / 2, sx - ((n + 1) * dLx + sr - Lx / 2))
        okx = n < nx
        for j in range(w):
            m = y0 + j
            iny = np.maximum(np.maximum(inx, m * dLy - sr - sy - Ly / 2), sy - ((m + 1) * dLy + sr - Ly / 2))
            oky = okx & (m < ny)
            for k in range(w):
                p = z0 + k
                v = np.maximum(np.maximum(iny, p * dLz - sr - sz - Lz / 2), sz - ((p + 1) * dLz + sr - Lz / 2))
                ok = oky & (p < nz) & (v < jump_tol)
                np.add.at(counts, (p * nx * ny + m * nx + n)[ok], 1)
    return counts


BUILDS = {  # name: what it is
    "packed_1e6": "packed axons (200 axons, 40x40x80 um), 1e6 walkers, 1 um cells",
    "single_axon_1e4": "single beaded axon (40 spheres + z images, 8x8x40 um), 1e4 walkers, cells (1, 1, 8)",
}


# jobs of the batched mixed workload (mixed_specs(seed=4), 64 jobs) whose
# substrates the reference arm of the batched benchmark walks: one of every 16
BATCH_SAMPLE_JOBS = (0, 16, 32, 48)


def workload_pars(name: str, nspins: int | None = None) -> dict:
    """Template pars of a named workload (walker count overridable):
    packed_1e6, single_axon_1e4, or batched_job<i> (job i of the batched
    mixed workload, 1 um cells)."""
    from nozomi_b200.substrates import beaded_axon, cell_grid
    if name == "packed_1e6":
        from nozomi_b200.workloads import packed_workload
        sub = packed_workload()[0]
        nseg, N = cell_grid(sub.L, 1.0), 1_000_000
    elif name == "single_axon_1e4":
        sub, nseg, N = beaded_axon(), (1, 1, 8), 10_000
    elif name.startswith("batched_job"):
        from nozomi_b200.workloads import mixed_specs
        sp = mixed_specs(seed=4, n_jobs=64)[int(name[len("batched_job"):])]
        sub, nseg, N = sp.substrate, cell_grid(sp.substrate.L, 1.0), sp.N
    else:
        raise KeyError(name)
    N = N if nspins is None else int(nspins)
    K = int(member_counts(sub.spheres(), sub.L, nseg).max())
    return pars_for(sub, N, nseg, K)


def build_all() -> list:
    """Build every baseline workload (only where the reference tree exists)."""
    if not reference_available():
        return []
    return [build(name, workload_pars(name)) for name in BUILDS]
