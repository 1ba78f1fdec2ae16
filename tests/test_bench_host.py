"""bench.py's host-side pieces that need no GPU: the clock-record summary
the timing rules rest on (a run that saw a slowdown reason is re-measured),
and the reference arm's CPU build of the reference kernel on a short sample
(where that build exists)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def test_clock_summary():
    import bench
    idle = "0, 1965, 1965, 300.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active"
    load = "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active"
    hot = "0, 1500, 1965, 1000.0, 0x0000000000000040, Not Active, Active, Not Active, Not Active"
    c = bench.Clocks.summarise("\n".join([idle, load, load, load]))
    assert c == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 4}
    c = bench.Clocks.summarise("\n".join([load, hot]))
    assert c["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert bench.Clocks.summarise("") is None
    assert bench.Clocks.summarise("0, [N/A], [N/A]")["sm_mhz"] is None


def test_reference_cpu_arm_runs_a_short_sample():
    """The reference arm's build (the reference's own kernel source compiled
    for the CPU, oracle/_ref) walks the packed workload's first walkers; all
    positions stay finite and inside the periodic box."""
    import bench
    from oracle.build import reference_named
    if reference_named(bench.REF_CPU_BUILD) is None:
        pytest.skip("oracle/_ref reference build absent (the reference tree was absent at build)")
    sub, pg, dirs, bvals = bench.workload()
    r = bench.ReferenceCpu(sub, pg, dirs)
    x0 = r.spins.copy()
    r.run(3)
    x = r.spins.reshape(3, r.N)
    assert np.isfinite(x).all() and not np.array_equal(r.spins, x0)
    L = np.array(sub.L)[:, None]
    assert np.all(np.abs(x) <= L / 2 + 1e-4)
