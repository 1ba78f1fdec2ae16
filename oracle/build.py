"""Oracle build recipes — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__`` and ``bench.py``'s CPU-baseline legs use the
oracle; the product never imports it.

* ``build_oracle()`` compiles the C restatement ``walk_oracle.c`` into
  ``oracle/liboracle.so`` (gcc, OpenMP, ``-ffp-contract=off`` so that the
  single-precision walk rounds every operation as the reference source reads).
* ``build_reference_kernel(code)`` compiles the reference's own kernel source
  (``simulation_toolkit/simulation_engine/sim3d_kernel.cu``), after the same
  ``%``-template substitution the reference performs at diffsim3d.py:39, as C++
  for the CPU with the host stand-ins in ``oracle/refshim`` and the launch
  emulation ``refshim/harness.cpp``.  Outputs go to ``oracle/_ref/`` only; the
  reference source is read where it lies and never copied into the repository.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
from pathlib import Path

ORACLE_DIR = Path(__file__).resolve().parent
REF_OUT = ORACLE_DIR / "_ref"
ORACLE_SO = ORACLE_DIR / "liboracle.so"
# the reference source tree: NOZOMI_REFERENCE_ROOT, else a folder named
# "reference" beside this repository
REFERENCE_ROOT = Path(os.environ.get("NOZOMI_REFERENCE_ROOT", ORACLE_DIR.parent.parent / "reference"))
REF_KERNEL_REL = "simulation_toolkit/simulation_engine/sim3d_kernel.cu"

_ORACLE_SRC = [ORACLE_DIR / "walk_oracle.c", ORACLE_DIR / "walk_step.inc", ORACLE_DIR / "oz_rng.h"]


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    """Compile oracle/liboracle.so if missing or older than its sources."""
    if force or _stale(ORACLE_SO, _ORACLE_SRC):
        cmd = ["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-Wall", "-o", str(ORACLE_SO), str(ORACLE_DIR / "walk_oracle.c"), "-lm"]
        subprocess.run(cmd, check=True)
    return ORACLE_SO


def reference_available() -> bool:
    return (REFERENCE_ROOT / REF_KERNEL_REL).is_file()


def substitute_reference(pars: dict) -> str:
    """The reference's kernel source with its template constants filled in,
    exactly as ``self.code % self.pars`` does (diffsim3d.py:39)."""
    return (REFERENCE_ROOT / REF_KERNEL_REL).read_text() % pars


def build_reference_kernel(code: str) -> Path:
    """Compile an already-substituted reference kernel source for the CPU."""
    REF_OUT.mkdir(parents=True, exist_ok=True)
    shim = ORACLE_DIR / "refshim"
    tag = hashlib.sha1((code + (shim / "harness.cpp").read_text() + (shim / "curand_kernel.h").read_text()
                        + (ORACLE_DIR / "oz_rng.h").read_text()).encode()).hexdigest()[:16]
    so = REF_OUT / f"ref_{tag}.so"
    if so.exists():
        return so
    src = REF_OUT / f"ref_{tag}.cpp"
    src.write_text(code)
    cmd = ["g++", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-w",
           "-I", str(shim), "-x", "c++", str(src), "-x", "c++", str(shim / "harness.cpp"),
           "-o", str(so) + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(str(so) + ".tmp", so)
    return so


REF_INDEX = REF_OUT / "index.json"

# named CPU builds of the reference kernel that bench.py's reference arm loads
# on a host without the reference tree: name -> (workload, walker count of the
# build).  The batched benchmark's reference arm walks jobs 0, 16, 32 and 48
# of the mixed workload with 8,000 walkers each.
BENCH_BUILDS = {"packed_cpu_16k": ("packed_1e6", 16_000),
                **{f"batched_job{i}_cpu_8k": (f"batched_job{i}", 8_000) for i in (0, 16, 32, 48)}}


def build_reference_named(name: str, pars: dict) -> Path:
    """build_reference_kernel for `pars`, recorded under `name` in
    oracle/_ref/index.json with its pars."""
    import json
    so = build_reference_kernel(substitute_reference(pars))
    idx = json.loads(REF_INDEX.read_text()) if REF_INDEX.exists() else {}
    idx[name] = {"so": so.name, "pars": pars}
    REF_INDEX.write_text(json.dumps(idx, indent=1))
    return so


def reference_named(name: str):
    """(so path, pars) of a named CPU build of the reference kernel, or None."""
    import json
    if not REF_INDEX.exists():
        return None
    e = json.loads(REF_INDEX.read_text()).get(name)
    if not e or not (REF_OUT / e["so"]).exists():
        return None
    return REF_OUT / e["so"], e["pars"]


def build_reference_bench() -> list:
    """The CPU builds of the reference kernel for bench.py's reference arms
    (the packed workload and a sample of the batched workload's jobs; 1 um
    cells; template constants as DiffSim3d forms them), where the reference
    tree is present."""
    if not reference_available():
        return []
    import sys
    sys.path.insert(0, str(ORACLE_DIR.parent))
    from baseline.reference_gpu import workload_pars
    return [build_reference_named(name, workload_pars(wl, nspins=n)) for name, (wl, n) in BENCH_BUILDS.items()]


if __name__ == "__main__":
    print(build_oracle(force=True))
