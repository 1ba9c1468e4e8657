"""bench.py's GPU arm on a short run: the one JSON line the driver reads,
with the keys it checks (roofline, cpu_baseline, e2e with its copies,
clocks, the kernel count)."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpu_arm_line_contract():
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--steps", "200", "--warmup", "3", "--relax", "200",
           "--cpu-steps", "2", "--e2e-reps", "2", "--one-step-launches", "5", "--no-l256", "--no-batched",
           "--no-served", "--no-gpu-reference"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["metric"] == "attempted monomer moves/s" and d["unit"] == "moves/s" and d["value"] > 0
    assert d["n_gpus"] == 1 and d["steps"] == 200 and d["warmup"] == 3 and d["higher_is_better"] is True
    assert d["scaling"] == "weak" and d["vs_baseline"] is None and d["dtype"] == "u32"
    assert d["config"]["L"] == 128 and d["config"]["P"] == 2517 and d["config"]["relax_steps"] == 200
    # the headline launches of 100 steps: two timed launches, each a graph replay of the sweep and the
    # step-counter update
    assert d["timed_launches"] == 2 and d["gpu_launches"] == 4
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0 and 0 < r["frac"] < 1
    assert abs(r["achieved"] / r["peak"] - r["frac"]) < 1e-9 and r["traffic"] > 0
    assert d["issue_roofline"]["frac"] > 0
    c = d["cpu_baseline"]
    assert c["value"] > 0 and c["cores"] == 1 and c["kind"] in ("reference", "port") and c["sample"]
    e = d["e2e"]
    assert e["value"] > 0 and e["unit"] == "moves/s"
    assert e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    if "clocks" in d:
        assert d["clocks"]["sm_max_mhz"] > 0
