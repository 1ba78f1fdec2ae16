"""The allocation-free re-binning entry point (nz_state_sort_static).

It serves hosts that cannot give this library device memory: their memory
manager owns all of it from start-up, or an allocation's implicit
synchronisation would stall their other work.  Its scratch is a fixed array
inside the library.  Here it is called through the C ABI and must give the same
result as nz_state_sort with a caller-provided buffer, on two calls in a row
(the second call reuses the array the first one left behind).

Within one bin the sort's order depends on atomics, so results are compared
as: the same bin sequence over the output slots, and the same walker records
once ordered by walker id (exact equality).

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _state(N, rng):
    from nozomi_b200 import engine
    pos = np.stack([rng.uniform(-20, 20, N), rng.uniform(-20, 20, N), rng.uniform(-40, 40, N)]).astype(np.float32)
    x = torch.from_numpy(pos).cuda()
    wk = engine.Walkers(x, x + 0.5, phi=torch.from_numpy(rng.normal(0, 1, (6, N)).astype(np.float32)).cuda(),
                        sig=torch.from_numpy(rng.uniform(0, 1, N).astype(np.float32)).cuda())
    return engine.FusedState.from_walkers(wk)


def _canonical(st, grid, coarsen):
    pos = st.pos.cpu().numpy()
    ids = st.org.cpu().numpy()[:, 3].view(np.int32)
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    ix = np.clip(np.floor((pos[:, 0] + grid.Lx / 2) / grid.dLx), 0, nx - 1).astype(int) // coarsen
    iy = np.clip(np.floor((pos[:, 1] + grid.Ly / 2) / grid.dLy), 0, ny - 1).astype(int) // coarsen
    iz = np.clip(np.floor((pos[:, 2] + grid.Lz / 2) / grid.dLz), 0, nz - 1).astype(int) // coarsen
    bx, by = -(-nx // coarsen), -(-ny // coarsen)
    bins = (iz * by + iy) * bx + ix
    order = np.argsort(ids)
    rec = np.concatenate([getattr(st, t).cpu().numpy()[order] for t in ("pos", "org", "phi", "comp")], axis=1)
    return bins, rec


def test_static_scratch_sort_matches_buffered_sort_twice():
    from nozomi_b200 import engine, _lib as L
    engine.require_cuda()
    lib = L.load()
    rng = np.random.default_rng(12)
    N = 300_000
    grid = engine.box_grid((40.0, 40.0, 80.0), (40, 40, 80))
    coarsen = 2
    src = _state(N, rng)
    ref = engine.FusedState(N)
    src.sort_into(ref, grid, coarsen)  # nz_state_sort with a torch-allocated buffer
    ref_bins, ref_rec = _canonical(ref, grid, coarsen)
    assert np.all(np.diff(ref_bins) >= 0)
    nbins = 20 * 20 * 40
    assert lib.nz_sort_scratch_bytes(N, nbins) <= lib.nz_state_sort_static_capacity()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        out = engine.FusedState(N)
        a, b = src.struct(), out.struct()
        rc = lib.nz_state_sort_static(ctypes.byref(a), ctypes.byref(grid), coarsen, ctypes.byref(b), stream)
        L.check(rc, "nz_state_sort_static")
        torch.cuda.synchronize()
        bins, rec = _canonical(out, grid, coarsen)
        np.testing.assert_array_equal(bins, ref_bins)
        np.testing.assert_array_equal(rec, ref_rec)


def test_static_scratch_sort_rejects_oversize():
    from nozomi_b200 import engine, _lib as L
    engine.require_cuda()
    lib = L.load()
    cap = lib.nz_state_sort_static_capacity()
    N = int(cap // 4) + 1024  # the walker bin array alone exceeds the fixed scratch
    st = engine.FusedState(N)
    out = engine.FusedState(N)
    grid = engine.box_grid((10.0, 10.0, 10.0), (10, 10, 10))
    a, b = st.struct(), out.struct()
    rc = lib.nz_state_sort_static(ctypes.byref(a), ctypes.byref(grid), 1, ctypes.byref(b),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == L.NZ_ERR_CAPACITY
    assert b"more than the fixed" in lib.nz_last_error()
