"""The product never routes through the oracle, and has no CPU path.

The oracle (oracle/) is test infrastructure.  The package nozomi_b200 must not
import it; bench.py may use it only in its CPU-baseline legs (the timed
restatement and the reference kernel's CPU build); the CUDA library exports no
oracle symbol; and without a GPU the product raises instead of computing."""
import ast
import ctypes
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _oracle_imports(tree):
    """(line, enclosing top-level name) of every import of the oracle package."""
    out = []
    for top in tree.body:
        for node in ast.walk(top):
            mods = []
            if isinstance(node, ast.Import):
                mods = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom) and node.level == 0:
                mods = [node.module or ""]
            for m in mods:
                if m == "oracle" or m.startswith("oracle."):
                    out.append((node.lineno, getattr(top, "name", None)))
    return out


def test_package_never_imports_the_oracle():
    files = sorted((ROOT / "nozomi_b200").rglob("*.py"))
    assert len(files) > 10
    for f in files:
        assert not _oracle_imports(ast.parse(f.read_text())), f"{f} imports the oracle"


def test_bench_uses_the_oracle_only_in_its_cpu_baseline_legs():
    found = _oracle_imports(ast.parse((ROOT / "bench.py").read_text()))
    assert found, "the CPU baseline legs import the oracle"
    legs = {"cpu_sample", "ReferenceCpu", "run_reference"}
    for line, owner in found:
        assert owner in legs, f"bench.py:{line} imports the oracle outside the CPU baseline legs ({owner})"


def test_library_exports_no_oracle_symbol():
    from nozomi_b200 import _lib
    lib = _lib.load()
    for name in ("oz_walk_f32", "oz_walk_f64", "oz_seed", "oz_philox_normals", "oz_segments", "oz_cells"):
        with pytest.raises(AttributeError):
            getattr(lib, name)
    assert isinstance(lib, ctypes.CDLL)


def test_no_cpu_path_without_a_gpu():
    """Every product entry point refuses on a machine without CUDA."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the refusal is tested on CPU-only machines")
    from nozomi_b200 import engine
    from nozomi_b200.diffsim3d import DiffSim3d
    from nozomi_b200.geometry import SimGeometry3D, Structure3D
    with pytest.raises(engine.NozomiError, match="CUDA device"):
        engine.require_cuda()
    sph = np.array([[0.0], [0.0], [0.0], [1.0], [0.0]])
    with pytest.raises(engine.NozomiError, match="CUDA device"):
        engine.DeviceSubstrate(sph, 1, (4.0, 4.0, 4.0), (1, 1, 1), [2.0, 2.0], [100.0, 100.0])
    g = SimGeometry3D(4.0, 4.0, 4.0, 2.0, 100, 1)
    g.add_structure(Structure3D(np.zeros(1), np.zeros(1), np.zeros(1), np.ones(1), 2.0, 100, 1))
    with pytest.raises(engine.NozomiError, match="CUDA device"):
        DiffSim3d(g, 1000)
