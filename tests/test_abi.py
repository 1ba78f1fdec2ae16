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


FAKE = 0x7F0000000000  # a 16-byte-aligned address the host never dereferences


def _fused_substrate(_lib):
    sub = _lib.Substrate()
    sub.grid = _lib.Grid(8.0, 8.0, 8.0, 1.0, 1.0, 1.0, 8, 8, 8)
    sub.nstructures, sub.S = 1, 4
    for f in ("spheres", "cell_start", "cell_count", "cell_items", "cell_sph4", "cell_sid", "D", "T2"):
        setattr(sub, f, FAKE)
    return sub


def _state(_lib, N, base=FAKE):
    return _lib.State(N, base, base + 0x1000, base + 0x2000, base + 0x3000)


def test_empty_inputs_return_ok_without_gpu():
    """Zero walkers, zero items or an empty step range: every entry point
    returns ok before any CUDA call, and null arrays are accepted where they
    would hold nothing."""
    import ctypes
    from nozomi_b200 import _lib
    lib = _lib.load()
    by = ctypes.byref
    sub = _fused_substrate(_lib)
    draws = _lib.Draws(None, 0, 0, 1, 2, 0)
    empty = _lib.State(0, None, None, None, None)
    wk0 = _lib.Walkers()
    wk0.N = 0
    for mode in (0, _lib.MODE_SIG, _lib.MODE_PHI):
        assert lib.nz_walk_step(by(sub), by(wk0), mode, 0.01, 0.0, 0.0, 0, by(draws), None) == 0
    wk0.ndir = 3
    assert lib.nz_walk_step(by(sub), by(wk0), _lib.MODE_PHASE, 0.01, 0.0, 0.0, 0, by(draws), None) == 0
    assert lib.nz_state_pack(by(wk0), None, by(empty), None) == 0
    assert lib.nz_state_unpack(by(empty), by(wk0), None) == 0
    assert lib.nz_state_unpack_by_id(by(empty), by(wk0), None, None) == 0
    assert lib.nz_walk_fused(by(sub), by(empty), _lib.MODE_PHI, 0.01, FAKE, FAKE, 0, 100, by(draws), None, None) == 0
    # a non-empty state over an empty step range
    st = _state(_lib, 1000)
    assert lib.nz_walk_fused(by(sub), by(st), _lib.MODE_PHI, 0.01, FAKE, FAKE, 50, 50, by(draws), None, None) == 0
    assert lib.nz_walk_fused_moments(by(sub), by(empty), 0, 0.01, None, None, 0, 100, by(draws), None, 0, FAKE,
                                     None) == 0
    assert lib.nz_walk_batch(FAKE, 3, FAKE, 0, _lib.MODE_PHI, 0, 100, FAKE, 148, 128, None) == 0
    assert lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_PHI, 7, 7, FAKE, 148, 128, None) == 0
    assert lib.nz_signal_phi(by(empty), FAKE, 6, FAKE, 4, FAKE, None) == 0
    assert lib.nz_signal_phase(FAKE, 6, 0, FAKE, 4, FAKE, None) == 0
    assert lib.nz_phase_from_phi(by(empty), FAKE, 6, None, None) == 0
    assert lib.nz_moments(FAKE, FAKE, 0, FAKE, None) == 0
    assert lib.nz_cells_gather(FAKE, 4, None, 0, None, None, 512, FAKE, None, None) == 0
    assert lib.nz_batch_sort(FAKE, 3, 0, 0, None, 0, None) == 0  # no walkers: nothing to do
    grid = sub.grid
    need = lib.nz_sort_scratch_bytes(0, 8 * 8 * 8)  # the histogram of the 8x8x8 grid's bins
    assert need > 0
    assert lib.nz_state_sort(by(empty), by(grid), 1, by(_lib.State(0, None, None, None, None)), FAKE, need, None) == 0


def test_invalid_arguments_rejected_without_gpu():
    """Malformed calls that would otherwise launch a kernel on bad memory are
    refused on the host with NZ_ERR_ARG (or NZ_ERR_CAPACITY) and a message."""
    import ctypes
    from nozomi_b200 import _lib
    lib = _lib.load()
    by = ctypes.byref
    sub = _fused_substrate(_lib)
    draws = _lib.Draws(None, 0, 0, 1, 2, 0)
    N = 1000
    a, b = _state(_lib, N), _state(_lib, N, FAKE + 0x100000)

    def refused(rc, who, status=_lib.NZ_ERR_ARG):
        assert rc == status, (who, rc)
        assert who.encode() in lib.nz_last_error(), lib.nz_last_error()

    grid = sub.grid
    nb = 8 * 8 * 8
    need = lib.nz_sort_scratch_bytes(N, nb)
    assert lib.nz_state_sort_keyed(by(a), by(grid), 1, 0, by(b), FAKE, need - 4, None) == _lib.NZ_ERR_CAPACITY
    bad_grid = _lib.Grid(8.0, 8.0, 8.0, 1.0, 1.0, 1.0, 8, 0, 8)
    refused(lib.nz_state_sort(by(a), by(bad_grid), 1, by(b), FAKE, need, None), "nz_state_sort")
    refused(lib.nz_state_sort_static(by(a), by(bad_grid), 1, by(b), None), "nz_state_sort_static")
    refused(lib.nz_state_sort(by(a), by(grid), 1, by(a), FAKE, need, None), "nz_state_sort")  # in place
    refused(lib.nz_state_sort(by(a), by(grid), 1, by(_state(_lib, N - 1, FAKE + 0x100000)), FAKE, need, None),
            "nz_state_sort")
    refused(lib.nz_state_sort(by(_state(_lib, N, FAKE + 8)), by(grid), 1, by(b), FAKE, need, None), "nz_state_sort")
    refused(lib.nz_state_sort(by(_lib.State(N, FAKE, None, FAKE, FAKE)), by(grid), 1, by(b), FAKE, need, None),
            "nz_state_sort")
    refused(lib.nz_signal_phi(by(_lib.State(N, FAKE, FAKE, None, FAKE)), FAKE, 6, FAKE, 4, FAKE, None),
            "nz_signal_phi")
    refused(lib.nz_phase_from_phi(by(a), FAKE, 6, None, None), "nz_phase_from_phi")
    refused(lib.nz_cells_gather(FAKE, 4, FAKE, 10, FAKE, FAKE, 0, FAKE, FAKE, None), "nz_cells_gather")
    refused(lib.nz_cells_gather(FAKE, 4, FAKE, 10, FAKE, FAKE, 8, FAKE + 4, FAKE, None), "nz_cells_gather")
    # batched re-binning: key counts per job, scratch, walkers without keys or jobs
    assert lib.nz_sort_job_keys(by(grid), 1, 0) == 512 and lib.nz_sort_job_keys(by(grid), 3, 5) == 27 * 5
    assert lib.nz_sort_job_keys(by(bad_grid), 1, 0) == -1 and lib.nz_sort_job_keys(by(grid), 0, 0) == -1
    assert lib.nz_batch_sort_scratch_bytes(N, 3 * nb) == lib.nz_sort_scratch_bytes(N, 3 * nb)
    bneed = lib.nz_batch_sort_scratch_bytes(N, 3 * nb)
    refused(lib.nz_batch_sort(FAKE, 3, N, 3 * nb, FAKE, bneed - 4, None), "nz_batch_sort", _lib.NZ_ERR_CAPACITY)
    refused(lib.nz_batch_sort(FAKE, 3, N, 0, FAKE, bneed, None), "nz_batch_sort")
    refused(lib.nz_batch_sort(FAKE, 0, N, 3 * nb, FAKE, bneed, None), "nz_batch_sort")
    refused(lib.nz_batch_sort(None, 3, N, 3 * nb, FAKE, bneed, None), "nz_batch_sort")
    refused(lib.nz_batch_sort(FAKE, 3, -1, 3 * nb, FAKE, bneed, None), "nz_batch_sort")
    # fused walk: draw table, step range, moments limits, misaligned cell records
    refused(lib.nz_walk_fused(by(sub), by(a), _lib.MODE_PHI, 0.01, FAKE, FAKE, 0, 10,
                              by(_lib.Draws(FAKE, 10, 4, 1, 2, 0)), None, None), "nz_walk_fused")
    refused(lib.nz_walk_fused(by(sub), by(a), _lib.MODE_PHI, 0.01, FAKE, FAKE, 10, 5, by(draws), None, None),
            "nz_walk_fused")
    refused(lib.nz_walk_fused(by(sub), by(a), _lib.MODE_MOMENTS, 0.01, None, None, 0, _lib.MOMENT_STEPS + 1,
                              by(draws), FAKE, None), "nz_walk_fused")
    refused(lib.nz_walk_fused(by(sub), by(a), _lib.MODE_PHI, 0.01, None, FAKE, 0, 10, by(draws), None, None),
            "nz_walk_fused")
    mis = _fused_substrate(_lib)
    mis.cell_sph4 = FAKE + 4
    refused(lib.nz_walk_fused(by(mis), by(a), 0, 0.01, None, None, 0, 10, by(draws), None, None), "nz_walk_fused")
    near = _fused_substrate(_lib)
    near.near_sph4, near.near_margin = FAKE, 0.5  # near records without their index arrays
    refused(lib.nz_walk_fused(by(near), by(a), 0, 0.01, None, None, 0, 10, by(draws), None, None), "nz_walk_fused")
    # index lists: a width other than 2 or 4, 16 bits for too many spheres, a
    # missing record array, misaligned records, near entries without offsets
    ix = _fused_substrate(_lib)
    ix.cell_sph4 = ix.cell_sid = None
    ix.idx_bytes, ix.cell_idx, ix.rec4, ix.rec_sid, ix.sid_start = 2, FAKE, FAKE, FAKE, FAKE
    for field, value in (("idx_bytes", 3), ("S", 70000), ("rec4", None), ("rec4", FAKE + 8), ("sid_start", None),
                         ("near_idx", FAKE)):
        bad = _fused_substrate(_lib)
        ctypes.pointer(bad)[0] = ix
        setattr(bad, field, value)
        refused(lib.nz_walk_fused(by(bad), by(a), 0, 0.01, None, None, 0, 10, by(draws), None, None),
                "nz_walk_fused")
    assert lib.nz_walk_fused(by(ix), by(empty_state := _lib.State(0, None, None, None, None)), 0, 0.01, None, None,
                             0, 10, by(draws), None, None) == 0
    ix.S = 70000
    ix.idx_bytes = 4  # 32-bit entries take any sphere count
    assert lib.nz_walk_fused(by(ix), by(empty_state), 0, 0.01, None, None, 0, 10, by(draws), None, None) == 0
    refused(lib.nz_cells_index(FAKE, 10, None, 70000, FAKE, FAKE, 8, FAKE, 2, None), "nz_cells_index")
    refused(lib.nz_cells_index(FAKE, 10, None, 100, FAKE, FAKE, 8, FAKE, 3, None), "nz_cells_index")
    refused(lib.nz_cells_index(FAKE, 10, None, 100, FAKE, FAKE, 0, FAKE, 2, None), "nz_cells_index")
    assert lib.nz_cells_index(None, 0, None, 100, None, None, 8, None, 2, None) == 0
    refused(lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_PHI | _lib.LIST_IDX16 | _lib.LIST_IDX32, 0, 100, FAKE, 148,
                              128, None), "nz_walk_batch")
    occ = ctypes.c_int(0)
    refused(lib.nz_batch_occupancy(_lib.MODE_PHI | _lib.LIST_IDX16 | _lib.LIST_IDX32, 128, ctypes.byref(occ)),
            "nz_batch_occupancy")
    # collision detection: grid checks, scratch, capacities
    cg = _lib.Grid(60.0, 60.0, 40.0, 6.0, 6.0, 5.7142857, 10, 10, 7)
    cneed = lib.nz_collide_scratch_bytes(1000, by(cg))
    assert cneed > 0 and lib.nz_collide_scratch_bytes(-1, by(cg)) == 0
    refused(lib.nz_collide_cells(FAKE, FAKE, 1000, by(cg), FAKE, FAKE, cneed - 1, None), "nz_collide_cells",
            _lib.NZ_ERR_CAPACITY)
    refused(lib.nz_collide_cells(FAKE, FAKE, 1000, by(_lib.Grid(60.0, 60.0, 40.0, 6.0, 0.0, 5.7, 10, 10, 7)), FAKE,
                                 FAKE, cneed, None), "nz_collide_cells")
    refused(lib.nz_collide_pairs(FAKE, FAKE, None, 1000, by(cg), 0.0, FAKE, 50, FAKE, 10, FAKE, FAKE, cneed, None),
            "nz_collide_pairs")
    refused(lib.nz_collide_pairs(FAKE, FAKE, FAKE, 1000, by(cg), 0.0, FAKE, 50, None, 10, FAKE, FAKE, cneed, None),
            "nz_collide_pairs")
    refused(lib.nz_pairs_sort(FAKE, 10, 0, FAKE, FAKE, 1 << 20, None), "nz_pairs_sort")
    refused(lib.nz_pairs_sort(FAKE, 10, 1000, FAKE, FAKE, 16, None), "nz_pairs_sort", _lib.NZ_ERR_CAPACITY)
    assert lib.nz_pairs_sort(None, 0, 1000, None, None, 0, None) == 0
    # ingestion: scratch sizes, small scratch, odd pads, missing arrays
    pad = lambda b: (b + 255) // 256 * 256  # noqa: E731
    assert lib.nz_ingest_scratch_bytes(100_000) == 2 * pad(400_000) + 2 * pad(4 * 13)
    need = lib.nz_ingest_scratch_bytes(1000)
    refused(lib.nz_ingest_split(FAKE, 1000, 10.0, FAKE, FAKE, FAKE, need - 1, None), "nz_ingest_split",
            _lib.NZ_ERR_CAPACITY)
    refused(lib.nz_ingest_split(None, 1000, 10.0, FAKE, FAKE, FAKE, need, None), "nz_ingest_split")
    refused(lib.nz_ingest_plan(FAKE, FAKE, 10, 49, FAKE, FAKE, FAKE, FAKE, FAKE, need, None), "nz_ingest_plan")
    refused(lib.nz_ingest_plan(FAKE, FAKE, 1000, 50, FAKE, FAKE, FAKE, FAKE, FAKE, 16, None), "nz_ingest_plan",
            _lib.NZ_ERR_CAPACITY)
    refused(lib.nz_ingest_write(FAKE, FAKE, 0, FAKE, FAKE, 10, 10.0, 50, FAKE, None, None), "nz_ingest_write")
    assert lib.nz_ingest_write(None, None, 0, None, None, 0, 10.0, 50, None, None, None) == 0
    # moments walk: scratch below [steps][3][N] floats, or an unsupported mode
    small = lib.nz_walk_fused_moments_scratch_bytes(N, 100) - 4
    refused(lib.nz_walk_fused_moments(by(sub), by(a), 0, 0.01, None, None, 0, 100, by(draws), FAKE, small, FAKE,
                                      None), "nz_walk_fused_moments")
    refused(lib.nz_walk_fused_moments(by(sub), by(a), _lib.MODE_PHI, 0.01, FAKE, FAKE, 0, 100, by(draws), FAKE,
                                      small + 4, FAKE, None), "nz_walk_fused_moments")
    # batched walk: CTA shape, persistent grid without a queue, moments
    refused(lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_PHI, 0, 100, FAKE, 148, 48, None), "nz_walk_batch")
    refused(lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_PHI, 0, 100, FAKE, 148, 512, None), "nz_walk_batch")
    refused(lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_PHI, 0, 100, None, 148, 128, None), "nz_walk_batch")
    refused(lib.nz_walk_batch(FAKE, 3, FAKE, 10, _lib.MODE_MOMENTS, 0, 100, FAKE, 148, 128, None), "nz_walk_batch")
    # staged batched walk: record lists, capacity out of range, the same shape checks
    staged = "nz_walk_batch_staged"
    idx = _lib.MODE_PHI | _lib.LIST_IDX16
    refused(lib.nz_walk_batch_staged(FAKE, 3, FAKE, 10, _lib.MODE_PHI, 0, 100, FAKE, 148, 128, 1024, None), staged)
    refused(lib.nz_walk_batch_staged(FAKE, 3, FAKE, 10, idx, 0, 100, FAKE, 148, 128, -1, None), staged)
    refused(lib.nz_walk_batch_staged(FAKE, 3, FAKE, 10, idx, 0, 100, FAKE, 148, 128, _lib.MAX_STAGE_RECORDS + 1,
                                     None), staged)
    refused(lib.nz_walk_batch_staged(FAKE, 3, FAKE, 10, idx, 0, 100, FAKE, 148, 48, 1024, None), staged)
    refused(lib.nz_walk_batch_staged(FAKE, 3, FAKE, 10, idx, 0, 100, None, 148, 128, 1024, None), staged)
    assert lib.nz_walk_batch_staged(FAKE, 3, FAKE, 0, idx, 0, 100, FAKE, 148, 128, 1024, None) == 0
    # plain step: unknown mode bits, phase without directions, null positions
    wk = _lib.Walkers()
    wk.N, wk.spins, wk.spins0 = N, FAKE, FAKE
    refused(lib.nz_walk_step(by(sub), by(wk), 64, 0.01, 0.0, 0.0, 0, by(draws), None), "nz_walk_step")
    refused(lib.nz_walk_step(by(sub), by(wk), _lib.MODE_PHASE, 0.01, 0.0, 0.0, 0, by(draws), None), "nz_walk_step")
    wk.spins = None
    refused(lib.nz_walk_step(by(sub), by(wk), 0, 0.01, 0.0, 0.0, 0, by(draws), None), "nz_walk_step")
    # packing: walker count mismatch
    wk.spins, wk.N = FAKE, N + 1
    refused(lib.nz_state_pack(by(wk), None, by(a), None), "nz_state_pack")


def test_protocol_tables_and_moment_rows_checked_without_gpu():
    """The fused walk reads G / Garea and writes moment rows by global step;
    the Python wrappers refuse tables or moment buffers that do not reach
    step1 (or have the wrong type) before any call into the library."""
    import torch
    from nozomi_b200 import _lib as L
    from nozomi_b200.engine import NozomiError, _check_tables
    G = torch.zeros(100, dtype=torch.float32)
    _check_tables("w", 100, L.MODE_PHI, G, G)
    _check_tables("w", 100, 0)  # no phase: no tables needed
    for bad in (torch.zeros(99, dtype=torch.float32), torch.zeros(100, dtype=torch.float64), None):
        with pytest.raises(NozomiError, match="steps to 100"):
            _check_tables("w", 100, L.MODE_PHI, G, bad)
    m = torch.zeros((100, 6), dtype=torch.float64)
    _check_tables("w", 100, 0, moments=m)
    with pytest.raises(NozomiError, match="rows of 6"):
        _check_tables("w", 101, 0, moments=m)
    with pytest.raises(NozomiError, match="rows of 6"):
        _check_tables("w", 10, 0, moments=m.float())
