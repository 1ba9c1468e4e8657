"""The N > 1 path of bench.py on CPU: replicas only.

Each rank runs an independent melt (seed + rank) and the ranks exchange
nothing but a barrier and the max of their timings, over gloo.  These tests
run that plumbing with world_size 2 on the host, and the reference arm
under torch.distributed.run, where rank 0 alone times the CPU efpol and
prints the one JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        # rank r "took" 10 + r ms: the job time is the slowest replica's
        t = bench.max_over_ranks(10.0 + rank, world)
        seed = bench.replica_seed(bench.WORKLOADS["L128"], rank)
        bench.barrier(world)
        q.put((rank, t, seed))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [11.0, 11.0]
    assert [g[2] for g in got] == [7, 8]   # L128 melt seed 7, replica r runs seed 7 + r


def test_single_rank_helpers_need_no_process_group():
    sys.path.insert(0, REPO)
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(3.5, 1) == 3.5


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_world2():
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()),
           os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2", "--workload", "L32",
           "--steps", "1", "--warmup", "3", "--ref-steps", "1"]
    r = subprocess.run(cmd, cwd=REPO, env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
