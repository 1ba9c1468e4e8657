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


def test_several_tiles_per_cta_give_the_same_bits():
    """A group with more tiles than resident CTAs (12 melts x 16 tiles of
    32x32x16 > 148) sweeps several tiles per CTA and step; every member still
    equals its single run (16 tiles, one per CTA)."""
    specs = [dict(L=64, N=200, seed=3000 + i, periodic=0, tile=(32, 32, 16)) for i in range(12)]
    b = elp.Batch(specs)
    b.init_melts()
    b.run(12)
    b.sync()
    for j in (0, 5, 11):
        m = elp.Melt(**specs[j])
        m.init_melt()
        m.run(12)
        wa, ra = b.state(j)
        wb, rb = m.state()
        assert np.array_equal(wa, wb) and np.array_equal(ra, rb), f"member {j} differs from its single run"
        assert b.check(j) == 0


@pytest.mark.parametrize("L,N", [(32, 100), (64, 200)])
def test_autotune_returns_a_geometry_with_a_known_clock(L, N):
    """The autotuner ranks candidates by time per efpol-equivalent step, so
    its choice always has a measured clock factor, and the returned spec
    runs and gives the same bits alone and batched."""
    sp, ms = elp.autotune(copies=4, steps=10, L=L, N=N, seed=9)
    assert ms > 0
    f = 1.0 if sp["periodic"] == 1 else elp.time_factor(0, *sp["tile"])
    assert 0 < f <= 1
    m = elp.Melt(**sp)
    m.init_melt()
    m.run(10)
    b = elp.Batch([sp, dict(sp, seed=10)])
    b.init_melts()
    b.run(10)
    w, r = m.state()
    wb, rb = b.state(0)
    assert np.array_equal(w, wb) and np.array_equal(r, rb)
