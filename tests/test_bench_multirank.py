"""bench.py's multi-rank path (what `--gpus N` runs under torchrun) with two
ranks on one GPU over gloo: both ranks exit 0, rank 0 alone prints one line
whose value counts every rank's walker-steps, and the line carries the keys of
the single-GPU line.  The two ranks share the GPU, so the numbers say nothing
about scaling; the test covers the control flow (sharding, barriers, the
timing all-reduce, the sharded signal all-reduce, teardown)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _two_ranks(*args):
    port = _free_port()
    procs = []
    for rank in (1, 0):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                   LOCAL_RANK="0")
        procs.append(subprocess.Popen([sys.executable, "bench.py", "--gpus", "2", "--dist-backend", "gloo", *args],
                                      cwd=ROOT, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=600) for p in procs]
    for p, (out, err) in zip(procs, outs):
        assert p.returncode == 0, out[-2000:] + err[-3000:]
    r1, r0 = (o for o, _ in outs)
    assert not any(l.startswith("{") for l in r1.splitlines())
    lines = [json.loads(l) for l in r0.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    return lines[0]


def test_batched_two_ranks():
    d = _two_ranks("--jobs", "6", "--walker-scale", "0.02", "--steps", "1", "--warmup", "3", "--no-autotune",
                   "--e2e-steps", "1")
    assert d["n_gpus"] == 2 and d["scaling"] == "strong" and d["value"] > 0
    assert d["e2e"]["value"] > 0 and d["roofline"]["bound"] == "issue"
    assert d["config"]["jobs"] == 6 and "2 GPUs" in d["config"]["parallelism"]


def test_packed_two_ranks():
    d = _two_ranks("--workload", "packed", "--walkers", "20000", "--steps", "1", "--warmup", "3",
                   "--e2e-steps", "1")
    assert d["n_gpus"] == 2 and d["scaling"] == "weak" and d["value"] > 0
    assert d["e2e"]["value"] > 0 and d["cpu_baseline"] is None
    # both ranks' walkers in the sums: the b = 0 signal is exactly 1
    assert abs(d["signal_b0_mean"] - 1.0) < 1e-12
