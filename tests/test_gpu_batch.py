"""The batched engine: every melt of a batch follows exactly the trajectory it
follows alone (same spec -> same bits), whatever else shares the GPU."""
import numpy as np
import pytest

import elp

pytestmark = pytest.mark.gpu

MIX = [
    dict(L=16, N=50, seed=1000, steps_per_launch=7),
    dict(L=16, N=64, seed=1001, steps_per_launch=7),
    dict(L=24, N=120, seed=1002, steps_per_launch=7),
    dict(L=32, N=200, seed=1003, steps_per_launch=7),
    dict(L=48, N=300, seed=1004),
    dict(L=64, N=500, seed=1005),
    dict(L=64, N=90, seed=1006, periodic=0, tile=(32, 32, 16)),
    dict(L=32, N=100, seed=1007, periodic=0, tile=(32, 16, 8)),   # generic kernel
    dict(L=64, N=300, seed=1008, steps_per_launch=10),            # tiled, 10 steps per launch
    dict(L=48, N=100, seed=1009, steps_per_launch=4),             # tiled, 4 steps per launch
]


def test_batch_members_equal_single_runs():
    b = elp.Batch(MIX)
    b.init_melts()
    b.run(130)                     # tiled groups: one 100-step graph + 30 launches
    b.sync()
    for j, kw in enumerate(MIX):
        m = elp.Melt(**kw)
        m.init_melt()
        m.run(130)
        wa, ra = b.state(j)
        wb, rb = m.state()
        assert np.array_equal(wa, wb) and np.array_equal(ra, rb), f"melt {j} differs from its single run"
        assert b.accepted(j) == m.accepted()
        assert b.check(j) == 0
        assert b.info(j).step == 130


def test_batch_graph_replays_continue_the_stream():
    kw = dict(L=64, N=500, seed=77)
    b = elp.Batch([kw, dict(L=16, N=50, seed=78)])
    b.init_melts()
    for n in (100, 100, 7, 200):   # graph, replay, single launches, two replays
        b.run(n)
    m = elp.Melt(**kw)
    m.init_melt()
    m.run(407)
    wa, ra = b.state(0)
    wb, rb = m.state()
    assert np.array_equal(wa, wb) and np.array_equal(ra, rb)


def test_batch_load_and_fetch_roundtrip():
    b = elp.Batch([dict(L=16, N=50, seed=5), dict(L=24, N=60, seed=6)])
    b.init_melts()
    b.run(20)
    s0, b0 = b.fetch(0)
    b.load_chains(0, s0, b0, step=20)
    s1, b1 = b.fetch(0)
    assert np.array_equal(s0, s1) and np.array_equal(b0, b1)
    assert b.info(0).step == 20
