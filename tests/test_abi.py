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
