"""ctypes binding of libnozomi_b200.so (the C ABI declared in include/nozomi_b200.h).

The library is the only compute path: loading fails loudly when it is missing
or when no CUDA device is present; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import os

# NOZOMI_B200_DEBUG_BOUNDS=1 loads the bounds-checked build instead: every
# cell index, list range and sphere index is checked before use, and a miss
# sets FLAG_BOUNDS on the walker (its access skipped) rather than reading
# out of range.  For tests and debugging; it is slower.
DEBUG_BOUNDS = os.environ.get("NOZOMI_B200_DEBUG_BOUNDS", "") not in ("", "0")
LIB_PATH = Path(__file__).resolve().parent / ("libnozomi_b200_debug.so" if DEBUG_BOUNDS else "libnozomi_b200.so")

NZ_OK, NZ_ERR_ARG, NZ_ERR_CUDA, NZ_ERR_CAPACITY, NZ_ERR_UNSEEDED = 0, 1, 2, 3, 4
MODE_SIG, MODE_PHASE, MODE_PHI, MODE_MOMENTS, MODE_TANGENT64 = 1, 2, 4, 8, 16
LIST_IDX16, LIST_IDX32 = 64, 128  # nz_walk_batch: the jobs' list format (none: per-entry records)
FLAG_DRAWS_EXHAUSTED, FLAG_ITER_CAP, FLAG_UNSEEDED, FLAG_BOUNDS, FLAG_STAGE_TIMEOUT = 1, 2, 4, 8, 16
MAX_STAGE_RECORDS = 12288  # nz_walk_batch_staged: records a CTA stages in shared memory at most
FUSED_THREADS = 128       # walkers per CTA / per work item of the fused and batched walks
MOMENT_STEPS = 256        # steps per launch when the fused walk accumulates moments
SCAN_SINGLE_KEYS = 32768  # nz_state_sort scans up to this many bins in one kernel, beyond it in three

_P = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_u = ctypes.c_uint32


class Grid(ctypes.Structure):
    _fields_ = [("Lx", _f), ("Ly", _f), ("Lz", _f), ("dLx", _f), ("dLy", _f), ("dLz", _f),
                ("nx", _i), ("ny", _i), ("nz", _i)]


class Substrate(ctypes.Structure):
    _fields_ = [("grid", Grid), ("nstructures", _i), ("S", _i), ("spheres", _P), ("cell_start", _P),
                ("cell_count", _P), ("cell_items", _P), ("cell_sph4", _P), ("cell_sid", _P), ("D", _P),
                ("T2", _P), ("near_margin", _f), ("near_start", _P), ("near_count", _P), ("near_sph4", _P),
                ("near_sid", _P), ("idx_bytes", _i), ("cell_idx", _P), ("near_idx", _P), ("rec4", _P),
                ("rec_sid", _P), ("sid_start", _P), ("n_items", _i), ("near_items", _i)]


class Draws(ctypes.Structure):
    _fields_ = [("table", _P), ("nsteps", _i), ("maxk", _i), ("key0", _u), ("key1", _u), ("stream", _u)]


class Walkers(ctypes.Structure):
    _fields_ = [("N", _i), ("spins", _P), ("spins0", _P), ("phase", _P), ("diffdir", _P), ("ndir", _i),
                ("sig", _P), ("phi", _P), ("label", _P), ("n_iter", _P), ("n_scatter", _P), ("flags", _P)]


class State(ctypes.Structure):
    _fields_ = [("N", _i), ("pos", _P), ("org", _P), ("phi", _P), ("comp", _P)]


class Job(ctypes.Structure):
    _fields_ = [("sub", Substrate), ("G", _P), ("Garea", _P), ("nsteps", _i), ("dt", _f), ("draws", Draws),
                ("mode", _i), ("state", State), ("moments", _P), ("step_offset", _i)]


class Item(ctypes.Structure):
    _fields_ = [("job", _i), ("first", _i), ("count", _i)]


class SortJob(ctypes.Structure):
    _fields_ = [("inp", State), ("out", State), ("grid", Grid), ("coarsen", _i), ("nlabels", _i),
                ("walker_offset", _i), ("key_offset", _i)]


# name -> (restype, argtypes); every symbol of include/nozomi_b200.h
SIGNATURES = {
    "nz_version": (_i, []),
    "nz_status_string": (ctypes.c_char_p, [_i]),
    "nz_last_error": (ctypes.c_char_p, []),
    "nz_device_sm_count": (_i, [_P]),
    "nz_cells_count": (_i, [_P, _i, _d, _d, _d, _i, _i, _i, _d, _P, _P]),
    "nz_exclusive_scan_i32": (_i, [_P, _P, _i, _P, _P]),
    "nz_cells_fill": (_i, [_P, _i, _d, _d, _d, _i, _i, _i, _d, _P, _P, _P, _P, _P]),
    "nz_cells_count_round": (_i, [_P, _i, _d, _d, _d, _i, _i, _i, _d, _P, _P]),
    "nz_cells_fill_round": (_i, [_P, _i, _d, _d, _d, _i, _i, _i, _d, _P, _P, _P, _P, _P]),
    "nz_segments_fill": (_i, [_P, _i, _d, _d, _d, _i, _i, _i, _i, _P, _P]),
    "nz_cells_gather": (_i, [_P, _i, _P, _i, _P, _P, _i, _P, _P, _P]),
    "nz_cells_index": (_i, [_P, _i, _P, _i, _P, _P, _i, _P, _i, _P]),
    "nz_collide_scratch_bytes": (ctypes.c_size_t, [_i, _P]),
    "nz_collide_cells": (_i, [_P, _P, _i, _P, _P, _P, ctypes.c_size_t, _P]),
    "nz_collide_pairs": (_i, [_P, _P, _P, _i, _P, _f, _P, _i, _P, _i, _P, _P, ctypes.c_size_t, _P]),
    "nz_pairs_sort_scratch_bytes": (ctypes.c_size_t, [_i]),
    "nz_pairs_sort": (_i, [_P, _i, _i, _P, _P, ctypes.c_size_t, _P]),
    "nz_ingest_scratch_bytes": (ctypes.c_size_t, [_i]),
    "nz_ingest_split": (_i, [_P, _i, _d, _P, _P, _P, ctypes.c_size_t, _P]),
    "nz_ingest_plan": (_i, [_P, _P, _i, _i, _P, _P, _P, _P, _P, ctypes.c_size_t, _P]),
    "nz_ingest_write": (_i, [_P, _P, _i, _P, _P, _i, _d, _i, _P, _P, _P]),
    "nz_seed": (_i, [_P, _P, _i, _u, _u, _u, _i, _P, _P, _P, _P]),
    "nz_seed_range": (_i, [_P, _P, _u, _i, _u, _u, _u, _i, _P, _P, _P, _P]),
    "nz_walk_step": (_i, [_P, _P, _i, _f, _f, _f, _i, _P, _P]),
    "nz_state_pack": (_i, [_P, _P, _P, _P]),
    "nz_state_unpack": (_i, [_P, _P, _P]),
    "nz_state_unpack_by_id": (_i, [_P, _P, _P, _P]),
    "nz_walk_fused": (_i, [_P, _P, _i, _f, _P, _P, _i, _i, _P, _P, _P]),
    "nz_walk_fused_moments_scratch_bytes": (ctypes.c_size_t, [_i, _i]),
    "nz_walk_fused_moments": (_i, [_P, _P, _i, _f, _P, _P, _i, _i, _P, _P, ctypes.c_size_t, _P, _P]),
    "nz_walk_batch": (_i, [_P, _i, _P, _i, _i, _i, _i, _P, _i, _i, _P]),
    "nz_batch_occupancy": (_i, [_i, _i, _P]),
    "nz_walk_batch_staged": (_i, [_P, _i, _P, _i, _i, _i, _i, _P, _i, _i, _i, _P]),
    "nz_batch_occupancy_staged": (_i, [_i, _i, _i, _P]),
    "nz_sort_scratch_bytes": (ctypes.c_size_t, [_i, _i]),
    "nz_state_sort": (_i, [_P, _P, _i, _P, _P, ctypes.c_size_t, _P]),
    "nz_state_sort_keyed": (_i, [_P, _P, _i, _i, _P, _P, ctypes.c_size_t, _P]),
    "nz_sort_job_keys": (ctypes.c_longlong, [_P, _i, _i]),
    "nz_batch_sort_scratch_bytes": (ctypes.c_size_t, [_i, _i]),
    "nz_batch_sort": (_i, [_P, _i, _i, _i, _P, ctypes.c_size_t, _P]),
    "nz_state_sort_static_capacity": (ctypes.c_size_t, []),
    "nz_state_sort_static": (_i, [_P, _P, _i, _P, _P]),
    "nz_signal_phi": (_i, [_P, _P, _i, _P, _i, _P, _P]),
    "nz_phase_from_phi": (_i, [_P, _P, _i, _P, _P]),
    "nz_signal_phase": (_i, [_P, _i, _i, _P, _i, _P, _P]),
    "nz_moments": (_i, [_P, _P, _i, _P, _P]),
    "nz_probe_fma": (_i, [_i, _i, _P, _P]),
}

_lib = None


class NozomiError(RuntimeError):
    pass


def load(require_built: bool = True) -> ctypes.CDLL:
    """Load the library (no GPU needed to load it)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise NozomiError(f"{LIB_PATH} is missing: build it with `python -m nozomi_b200.build`"
                              + (" --debug" if DEBUG_BOUNDS else ""))
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(rc: int, what: str = ""):
    if rc != NZ_OK:
        lib = load()
        msg = lib.nz_last_error().decode(errors="replace")
        raise NozomiError(f"{what or 'nozomi_b200'}: {lib.nz_status_string(rc).decode()} ({msg})")


def byref(s):
    return ctypes.byref(s)
