"""bench.py's reference arm on the host cores (no GPU needed): the JSON line
the driver reads, alone and launched as two ranks (rank 0 alone prints)."""
import json
import os
import socket
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def check_line(line, n):
    d = json.loads(line)
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["n_gpus"] == n and d["steps"] == 1 and d["warmup"] == 3
    assert d["metric"] == "attempted monomer moves/s" and d["unit"] == "moves/s" and d["value"] > 0
    assert d["higher_is_better"] is True and d["vs_baseline"] is None
    assert d["cpu_baseline"]["kind"] in ("reference", "port") and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["L"] == 128 and d["config"]["N"] == 1000 and d["config"]["P"] == 2517


def test_reference_arm_prints_one_line():
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--ref-steps", "1"], capture_output=True, text=True, timeout=300, cwd=REPO)
    assert out.returncode == 0, out.stderr
    lines = [x for x in out.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    check_line(lines[0], 1)


def test_reference_arm_under_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), os.path.join(REPO, "bench.py"), "--gpus", "2", "--impl",
           "reference", "--steps", "1", "--warmup", "3", "--ref-steps", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.strip().startswith("{")]
    assert len(lines) == 1
    check_line(lines[0], 2)


def test_cpu_ensemble_leg_runs_the_power_of_two_members():
    sys.path.insert(0, REPO)
    import bench
    mix = bench.ensemble_mix(64)
    out = bench.cpu_ensemble(mix, target_moves=2e5, max_procs=4)
    assert out["unit"] == "moves/s" and out["value"] > 0
    assert out["kind"] in ("reference", "port") and 1 <= out["cores"] <= 4
    assert all(m["L"] in (16, 24, 32, 48, 64) for m in mix)
    assert sum(1 for m in mix if m["L"] in (16, 32, 64)) >= out["cores"]
