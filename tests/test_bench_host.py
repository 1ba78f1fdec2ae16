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


def test_clock_summary_keeps_this_gpus_rows():
    """All GPUs are sampled; the rows kept are this CUDA device's, found by
    UUID (any case, with or without nvidia-smi's GPU- prefix), else PCI bus,
    else nvidia-smi index."""
    import bench
    tail = ", Not Active, Not Active, Not Active"
    ours = f"3, 1950, 1965, 900.0, 0x4{tail}, Active, GPU-8d3a1c2e-aaaa-bbbb-cccc-0123456789ab, 00000000:1B:00.0"
    other = f"0, 1200, 1965, 700.0, 0x40, Not Active, Active, Not Active, Not Active, GPU-11111111-2222-3333-4444-555555555555, 00000000:0A:00.0"
    text = "\n".join([ours, other, ours, other, ours])
    by_uuid = bench.Clocks.summarise(text, uuid="8D3A1C2E-AAAA-BBBB-CCCC-0123456789AB", bus=99, index=0)
    assert by_uuid == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    assert bench.Clocks.summarise(text, uuid=None, bus=0x1B, index=0)["samples"] == 3
    by_index = bench.Clocks.summarise(text, index=0)
    assert by_index["samples"] == 2 and by_index["reasons"] == ["hw_thermal_slowdown"]
    assert bench.Clocks.summarise(text)["samples"] == 5  # nothing identifies the GPU: every row


def test_reference_cpu_arm_runs_a_short_sample():
    """The reference arm's builds (the reference's own kernel source compiled
    for the CPU, oracle/_ref) walk the first walkers of the packed workload
    and of a sampled job of the batched workload; all positions stay finite
    and inside the periodic box."""
    import bench
    for workload in ("packed", "batched"):
        cases, _ = bench.reference_cases(workload)
        build, sub, gw, dirs = cases[0]
        try:
            r = bench.ReferenceCpu(build, sub, gw, dirs)
        except FileNotFoundError:
            pytest.skip("oracle/_ref reference build absent (the reference tree was absent at build)")
        x0 = r.spins.copy()
        r.run(3)
        x = r.spins.reshape(3, r.N)
        assert np.isfinite(x).all() and not np.array_equal(r.spins, x0)
        L = np.array(sub.L)[:, None]
        assert np.all(np.abs(x) <= L / 2 + 1e-4)


def _reference_line(*extra):
    import json
    import subprocess
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--cpu-seconds", "1", *extra], cwd=ROOT, capture_output=True, text=True,
                         timeout=900, check=True).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    return json.loads(lines[0])


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` runs on the host cores alone (no GPU) and
    prints one JSON line with the base contract's keys, its cpu_baseline and
    an e2e without transfers; the same metric, unit and workload as the GPU
    arm: the batched workload by default (its sampled jobs), the packed one
    with --workload packed."""
    import bench
    from oracle.build import reference_named
    if reference_named("batched_job0_cpu_8k") is None or reference_named("packed_cpu_16k") is None:
        pytest.skip("oracle/_ref reference build absent (the reference tree was absent at build)")
    for extra, wl in (((), bench.BATCH_WORKLOAD.format(jobs=64, scale=1.0, a0=10, a1=500)),
                      (("--workload", "packed"), bench.WORKLOAD)):
        d = _reference_line(*extra)
        for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                  "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
            assert k in d, k
        assert d["impl"] == "reference" and d["metric"] == "walker-steps/s" and d["unit"] == "walker-steps/s"
        assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1
        assert d["config"]["workload"] == wl
        assert d["value"] > 0 and d["ms_per_step"] > 0
        cb = d["cpu_baseline"]
        assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
        assert d["e2e"] == {"value": d["value"], "unit": "walker-steps/s", "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}


def test_roofline_counts_are_tied_to_the_kernel_source():
    """The issue roofline multiplies ncu-counted warp instructions per
    walker-step by the kernel's walker-steps/s over 4 issue slots x SMs x
    clock; counts taken on other kernel sources are marked stale."""
    import bench
    saved = dict(bench.PROFILED["batched"])
    try:
        bench.PROFILED["batched"].update(kernel_sha=bench.kernel_sha(), warp_inst_per_walker_step=50.0,
                                         dram_bytes_per_walker_step=2.0, capture="test")
        clk = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": []}
        issue, fp32, hbm = bench.rooflines("batched", 1e10, 4e9, 300.0, 1e9, clk, 148, 70.0, 250.0)
        assert issue["bound"] == "issue" and not issue["stale"]
        assert abs(issue["frac"] - 50.0 * 1e10 / (148 * 4 * 1965e6)) < 1e-12
        assert issue["traffic"] == 2.0 * 4e9
        assert abs(fp32["frac"] - 1e10 * 250.0 / 1e12 / 70.0) < 1e-12
        assert abs(hbm["achieved"] - 1e9 / 0.3 / 1e9) < 1e-9
        bench.PROFILED["batched"]["kernel_sha"] = "0" * 16
        assert bench.rooflines("batched", 1e10, 4e9, 300.0, 1e9, clk, 148, 70.0, None)[0]["stale"]
    finally:
        bench.PROFILED["batched"].clear()
        bench.PROFILED["batched"].update(saved)


def test_committed_counts_match_the_committed_kernel():
    """The instruction and DRAM counts the bench line uses were captured on
    the kernel and list sources in the tree (a kernel change needs a new
    capture), and on the default list form."""
    import bench
    for name, prof in bench.PROFILED.items():
        assert prof["kernel_sha"] == bench.kernel_sha(), name
        assert prof["shape"]["lists"] == "index" and prof["shape"]["near_shape"] == "round", name
        assert prof["shape"]["stage"] == 0, name  # captured on the unstaged kernel
