"""The C ABI library loads without a GPU and exports every function that
include/nozomi_b200.h declares, with a ctypes signature for each."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(nz_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    from nozomi_b200 import _lib
    lib = _lib.load()
    names = declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} not exported"
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"
    assert set(_lib.SIGNATURES) <= set(names)


def test_version_and_status_strings():
    from nozomi_b200 import _lib
    lib = _lib.load()
    assert lib.nz_version() == 1
    assert lib.nz_status_string(0) == b"ok"
    assert lib.nz_status_string(1) == b"invalid argument"


def test_argument_errors_without_gpu():
    """Argument checks run before any CUDA call: usable on a CPU machine."""
    from nozomi_b200 import _lib
    lib = _lib.load()
    rc = lib.nz_cells_count(None, 5, 1.0, 1.0, 1.0, 0, 1, 1, 1.0, None, None)
    assert rc == _lib.NZ_ERR_ARG
    assert b"nz_cells_count" in lib.nz_last_error()
    with pytest.raises(_lib.NozomiError):
        _lib.check(rc, "nz_cells_count")


def test_scratch_sizes_and_more_argument_errors_without_gpu():
    """Scratch-size arithmetic and argument checks of the later entry points,
    all decided on the host before any CUDA call."""
    import ctypes
    from nozomi_b200 import _lib
    lib = _lib.load()
    # re-binning: walker bins, histogram, cursor, and two tile arrays for the
    # many-CTA scan (one int per 8,192 keys), each padded to 256 bytes
    pad = lambda b: (b + 255) // 256 * 256  # noqa: E731
    for N, nb in ((1000, 100), (300_000, 16_000), (250_000, 384_000)):
        tiles = -(-nb // 8192)
        assert lib.nz_sort_scratch_bytes(N, nb) == pad(4 * N) + 2 * pad(4 * nb) + 2 * pad(4 * tiles)
    # narrow-pulse displacements: 12 bytes per walker-step
    assert lib.nz_walk_fused_moments_scratch_bytes(1000, 256) == 1000 * 256 * 12
    assert lib.nz_walk_fused_moments_scratch_bytes(0, 256) == 0
    # seeding a walker range that runs past 2^32 ids
    sub = _lib.Substrate()
    sub.S, sub.nstructures = 0, 0
    rc = lib.nz_seed_range(ctypes.byref(sub), None, 0xFFFFFF00, 1024, 1, 2, 1, 10, None, None, None, None)
    assert rc == _lib.NZ_ERR_ARG and b"nz_seed_range" in lib.nz_last_error()
    # the moments walk with no substrate lists
    rc = lib.nz_walk_fused_moments(ctypes.byref(sub), None, 0, 0.005, None, None, 0, 10, None, None, 0, None, None)
    assert rc == _lib.NZ_ERR_ARG
