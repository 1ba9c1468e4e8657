"""The serving loop: jobs admitted while others run give the same bits as
the same job alone and as the single-melt API; dumps are the TUV files the
single-melt API writes at those steps."""
import os
import time

import numpy as np
import pytest

import elp

pytestmark = pytest.mark.gpu

JOBS = [dict(L=16, N=50, seed=11), dict(L=32, N=100, seed=12), dict(L=64, N=500, seed=13),
        dict(L=24, N=60, seed=14), dict(L=48, N=200, seed=15), dict(L=16, N=80, seed=16)]


def plain_checksum(kw, steps):
    m = elp.Melt(steps_per_launch=50, **kw)
    m.init_melt()
    m.run(steps)
    return elp.ring_checksum(*m.fetch())


def test_jobs_same_alone_in_mix_and_plain(tmp_path):
    steps = 200
    srv = elp.Server(quantum=50)
    alone = {}
    for kw in JOBS[:3]:
        jid = srv.submit(steps, **kw)
        srv.drain(300)
        r = srv.poll()
        assert len(r) == 1 and r[0]["id"] == jid and r[0]["status"] == 0 and r[0]["integrity"] == 0
        alone[kw["seed"]] = r[0]["checksum"]
    # the mix: staggered submissions join while others run
    ids = {}
    for i, kw in enumerate(JOBS):
        ids[srv.submit(steps, dump_interval=100, dump_dir=str(tmp_path / f"job{kw['seed']}"), **kw)] = kw
        time.sleep(0.01 * i)
    srv.drain(300)
    res = srv.poll()
    assert len(res) == len(JOBS)
    for r in res:
        kw = ids[r["id"]]
        assert r["status"] == 0 and r["integrity"] == 0
        assert r["steps"] == steps and r["dumps"] == 2
        want = plain_checksum(kw, steps)
        assert r["checksum"] == want, f"job {kw} differs from its single-melt run"
        if kw["seed"] in alone:
            assert r["checksum"] == alone[kw["seed"]]
    srv.close()
    # a dump equals the single-melt API's TUV at that step
    kw = JOBS[2]
    m = elp.Melt(**kw)
    m.init_melt()
    m.run(100)
    p = str(tmp_path / "plain.res")
    m.write_tuv(p)
    assert open(str(tmp_path / f"job{kw['seed']}" / "t=100_dev=0.res")).read() == open(p).read()


def test_admission_respects_the_budget():
    # budget for about two L=32 jobs: the rest wait in the queue and still finish
    one = 2 * (32 ** 3 * 4 + 393 * 16)
    srv = elp.Server(quantum=50, hbm_budget=int(2.5 * one))
    for i in range(6):
        srv.submit(100, L=32, N=100, seed=100 + i)
    peak = 0
    t0 = time.time()
    while time.time() - t0 < 120:
        st = srv.stats()
        peak = max(peak, st["resident"])
        if st["completed"] == 6:
            break
        time.sleep(0.002)
    srv.drain(120)
    res = srv.poll()
    assert len(res) == 6 and all(r["status"] == 0 for r in res)
    assert peak <= 2
    srv.close()


def test_rejects_bad_job_arguments():
    srv = elp.Server(quantum=50)
    with pytest.raises(elp.ElpError):
        srv.submit(75, L=16, N=50)           # not a multiple of the quantum
    with pytest.raises(elp.ElpError):
        srv.submit(100, dump_interval=30, L=16, N=50)
    srv.close()


def test_linear_chain_jobs_same_in_mix_and_plain(tmp_path):
    """Linear-chain jobs (efpol_lin) share the server with rings in their own
    groups and give the single-melt API's chains; a box without a
    specialised kernel shape refuses them."""
    lin = [dict(L=16, N=50, seed=21, linear=1), dict(L=64, N=200, seed=22, linear=1),
           dict(L=48, N=100, seed=23, linear=1)]
    steps = 200
    srv = elp.Server(quantum=50)
    ids = {}
    for i, kw in enumerate(lin + JOBS[:2]):
        ids[srv.submit(steps, dump_interval=100, dump_dir=str(tmp_path / f"j{i}"), **kw)] = kw
        time.sleep(0.005)
    bad = srv.submit(100, L=40, N=100, seed=24, linear=1)   # 40x20x20 tiles: generic kernel only
    srv.drain(300)
    res = {r["id"]: r for r in srv.poll()}
    assert len(res) == len(ids) + 1
    assert res[bad]["status"] == elp.ERR_ARG
    for jid, kw in ids.items():
        r = res[jid]
        assert r["status"] == 0 and r["integrity"] == 0 and r["dumps"] == 2
        assert r["checksum"] == plain_checksum(kw, steps), f"job {kw} differs from its single-melt run"
    srv.close()


def test_dump_write_failure_fails_the_job(tmp_path):
    """A dump that cannot be written ends its job with ELP_ERR_IO (the
    directory is a regular file, so every open fails, also for root)."""
    blocker = tmp_path / "not_a_dir"
    blocker.write_text("x")
    srv = elp.Server(quantum=50)
    bad = srv.submit(300, dump_interval=100, dump_dir=str(blocker), L=16, N=50, seed=31)
    good = srv.submit(300, dump_interval=100, dump_dir=str(tmp_path / "ok"), L=16, N=50, seed=32)
    srv.drain(120)
    res = {r["id"]: r for r in srv.poll()}
    assert res[bad]["status"] == elp.ERR_IO
    assert res[good]["status"] == 0 and res[good]["integrity"] == 0
    assert sorted(os.listdir(tmp_path / "ok")) == ["t=100_dev=0.res", "t=200_dev=0.res", "t=300_dev=0.res"]
    srv.close()


def test_small_jobs_pass_a_job_waiting_for_memory():
    """A job that does not fit the budget waits; smaller jobs queued behind it
    start before it (no head-of-line blocking), and it still runs once the
    memory frees up."""
    big = 2 * (64 ** 3 * 4 + 1573 * 16)
    srv = elp.Server(quantum=50, hbm_budget=int(1.5 * big))
    first = srv.submit(50000, L=64, N=200, seed=41)           # resident for about a second
    time.sleep(0.05)
    waiting = srv.submit(100, L=64, N=200, seed=42)           # does not fit beside it
    small = [srv.submit(100, L=16, N=50, seed=43 + i) for i in range(4)]
    srv.drain(300)
    res = {r["id"]: r for r in srv.poll()}
    assert all(r["status"] == 0 for r in res.values())
    assert all(res[s]["t_start"] < res[first]["t_done"] for s in small), "the resident job ended too early"
    assert all(res[s]["t_start"] < res[waiting]["t_start"] for s in small)
    assert res[waiting]["t_start"] >= res[first]["t_done"] - 0.05
    srv.close()
