"""The bounds-checked build (libnozomi_b200_debug.so, -DNZ_DEBUG_BOUNDS=1),
standing in for compute-sanitizer: every cell index, list range and
sphere / record index is checked before use; an index out of range sets
NZ_FLAG_BOUNDS on the walker and its access is skipped (nothing traps).

* The small parity cases (plain and fused walks, every list form, near
  lists, edge starts, batched walks) run in a child process on that build:
  they stay bit-exact against the oracle, whose flags never carry the
  bounds bit, so no access of theirs was out of range.
* Planted out-of-range indices (a sphere index past S in a plain cell list,
  a record index past S in an index list, a cell count running past the
  list) are caught: the walkers that meet them are flagged, the others walk
  as before.  These run only in the child process on the checked build.
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
ROOT = Path(__file__).resolve().parents[1]

PARITY = ("test_plain_dwi_matches_reference or test_plain_narrow_matches_reference or "
          "test_fused_matches_oracle_and_reference or test_fused_near_lists_match_full_lists or "
          "test_index_lists_with_shuffled_sphere_order or test_batch_positions_match_oracle or "
          "test_planted")


def test_parity_cases_on_the_bounds_checked_build():
    from nozomi_b200.build import DEBUG_LIB
    if not DEBUG_LIB.exists():
        pytest.fail(f"{DEBUG_LIB} is missing: build it with `python -m nozomi_b200.build --debug`")
    env = dict(os.environ, NOZOMI_B200_DEBUG_BOUNDS="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-k", PARITY,
                        "tests/test_gpu_parity.py", "tests/test_batch.py", "tests/test_debug_bounds.py"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1500)
    print(r.stdout[-3000:])
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "skipped" not in r.stdout.splitlines()[-1]


def _checked():
    from nozomi_b200 import _lib as L
    if not L.DEBUG_BOUNDS:
        pytest.skip("runs on the bounds-checked build (NOZOMI_B200_DEBUG_BOUNDS=1)")
    return L


@pytest.mark.parametrize("what", ["plain_item", "index_entry", "count"])
def test_planted_out_of_range_indices_are_flagged(what):
    """One cell of the overlap fixture's lists gets an out-of-range index (or
    a count past the end of the lists); walkers that meet it carry
    NZ_FLAG_BOUNDS and no access leaves the arrays."""
    L = _checked()
    from nozomi_b200 import engine
    from tests._fixtures import load
    c = load("dwi_overlap")
    sph, L3, nseg = c["spheres"], tuple(c["L"]), tuple(int(v) for v in c["nseg"])
    sub = engine.DeviceSubstrate(sph, int(c["nstructures"]), L3, nseg, c["D"], c["T2"],
                                 idx_bytes=0 if what == "plain_item" else 2)
    N, nt, dt = int(c["N"]), 5, float(c["dt"])  # 97 walkers start in the planted cell, most never reach it
    x0 = torch.from_numpy(c["x0"].astype(np.float32)).cuda()
    counts = sub.cell_count.cpu().numpy()
    busy = int(np.argmax(counts))  # the cell with the longest list
    first = int(sub.cell_start[busy].item())
    if what == "plain_item":
        sub.cell_items[first] = sub.S + 5
    elif what == "index_entry":
        sub.cell_idx[first] = sub.S + 5
    else:
        sub.cell_count[busy] = sub.n_items + 10
    draws = engine.philox_draws(3)
    if what == "plain_item" or what == "count":
        wk = engine.Walkers.with_counters(x0.clone(), x0.clone())
        for s in range(nt):
            engine.walk_step(sub, wk, 0, dt, 0.0, 0.0, s, draws)
        flags = wk.flags.cpu().numpy()
    if what != "plain_item":
        w = engine.Walkers(x0.clone(), x0.clone(), phi=torch.zeros((6, N), device="cuda"),
                           flags=torch.zeros(N, dtype=torch.int32, device="cuda"))
        st = engine.FusedState.from_walkers(w)
        z = torch.zeros(nt, device="cuda")
        engine.walk_fused(sub, st, 0, dt, z, z, 0, nt, draws)
        st.to_walkers(w)
        flags = w.flags.cpu().numpy() if what == "index_entry" else flags | w.flags.cpu().numpy()
    torch.cuda.synchronize()
    hit = (flags & L.FLAG_BOUNDS) != 0
    assert hit.any() and not hit.all()
