"""Bit-exact parity of the sweep kernels with the host replay on RELAXED melts.

The initial melt of the reference's CreatePolymers holds each ring on two
sites, so a few steps from it exercise almost none of the dense-melt cases:
kinks and crankshafts next to occupied sites, a monomer joining a neighbour
run, monomer 0 moving between runs, many label slots in one tile.  These
tests start where a production run spends its time, from states that are
already relaxed:

* the reference efpol's own dumps after 100 and 200 steps (rings and linear
  chains), loaded into the kernel and into the replay from their chains;
* melts relaxed on the GPU for thousands of steps (every specialised tiled
  shape, the bench's L=128 and L=256 melts), handed to the replay as they
  stand (site words and records);
* short rings (N = 14 to 40), whose many monomer-0 runs fill the
  shared-memory label slots close to their capacity, and beyond it in the
  tiles that CreatePolymers' slab of rings crowds (those tiles take the
  general move, with monomer 0's bookkeeping in the chain records).

The replay (oracle/replay.c) applies the same schedule, anchors and Philox
counters on the CPU; after every compared step the site words, the ring
records and the accepted-move count must be equal.  The move set itself is
the reference's DoStep (cpupol/efpol_lib.c:132-207).
"""
import os

import numpy as np
import pytest

import elp
import observables as obs
from oracle_binding import Replay

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(REPO, "tests", "golden")


def replay_like(m: elp.Melt, seed, linear=False):
    i = m.info()
    return Replay(i.L, i.N, i.P, seed=seed, periodic=bool(i.periodic), tile=tuple(i.tile), ncol=i.ncol,
                  linear=linear)


def occupied_fraction(words):
    return float(np.count_nonzero(words)) / words.size


def compare_run(m, r, steps, every, what):
    """Advance the kernel and the replay side by side, comparing every
    `every` steps; returns the accepted moves of the window."""
    a0, r0 = m.accepted(), r.accepted
    done = 0
    while done < steps:
        k = min(every, steps - done)
        m.run(k)
        r.steps(k)
        done += k
        w, rec = m.state()
        assert np.array_equal(w, r.lattice()), f"{what}: site words differ {done} steps into the window"
        assert np.array_equal(rec, r.records()), f"{what}: records differ {done} steps into the window"
        assert m.accepted() - a0 == r.accepted - r0, f"{what}: accepted moves differ after {done} steps"
    assert m.check() == 0
    return r.accepted - r0


REF_DUMPS = [
    # (golden dump, L, N, linear, geometry, steps)
    ("efpol_L32_N100_s1_t200", 32, 100, 0, dict(), 60),                                # whole box on chip
    ("efpol_L32_N100_s1_t200", 32, 100, 0, dict(periodic=0, tile=(16, 16, 16)), 60),   # tiled, 4 CTAs per SM
    ("efpol_L32_N100_s1_t200", 32, 100, 0, dict(periodic=0, tile=(32, 16, 8)), 60),    # generic kernel
    ("efpol_L32_N100_s1_t200", 32, 100, 0, dict(kernel=1), 60),                        # generic, whole box
    ("efpol_L16_N50_s3_t100", 16, 50, 0, dict(), 80),
    ("efpol_L16_N50_s3_t100", 16, 50, 0, dict(kernel=1), 80),
    ("efpol_lin_L32_N100_s1_t200", 32, 100, 1, dict(), 60),
    ("efpol_lin_L32_N100_s1_t200", 32, 100, 1, dict(periodic=0, tile=(16, 16, 16)), 60),
    ("efpol_lin_L16_N50_s3_t100", 16, 50, 1, dict(), 80),
]


@pytest.mark.parametrize("name,L,N,linear,kw,steps", REF_DUMPS)
def test_reference_dumps_step_like_the_replay(name, L, N, linear, kw, steps):
    """The reference efpol's relaxed dumps, stepped every step against the replay."""
    _, start, bonds = obs.read_tuv(os.path.join(GOLD, name + ".res.gz"))
    seed = 4000 + L + N + linear
    m = elp.Melt(L=L, N=N, seed=seed, linear=linear, **kw)
    m.load_chains(start, bonds, 200)
    r = replay_like(m, seed, linear=bool(linear))
    assert r.load(start, bonds) == 0
    r.set_state(r.lattice(), r.records(), 200)
    w, rec = m.state()
    assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())
    assert occupied_fraction(w) > 0.3, "the dump is not a relaxed melt"
    acc = compare_run(m, r, steps, 1, name)
    assert acc > 0


GPU_RELAXED = [
    # (L, N, geometry, relax steps, steps per launch, compared steps, compare every)
    (64, 200, dict(periodic=0, tile=(32, 32, 32)), 2000, 10, 50, 10),
    (64, 200, dict(periodic=0, tile=(32, 32, 16)), 2000, 10, 50, 10),
    (64, 200, dict(periodic=0, tile=(32, 16, 16)), 2000, 10, 50, 10),
    (64, 200, dict(periodic=0, tile=(16, 16, 16)), 2000, 10, 50, 10),
    (48, 100, dict(periodic=0, tile=(48, 24, 24)), 2000, 10, 50, 10),
    (64, 200, dict(periodic=0, tile=(32, 32, 32)), 2000, 1, 20, 1),     # one step per launch
    (32, 100, dict(), 3000, 25, 50, 25),                                 # whole box, many steps per launch
    (24, 60, dict(), 3000, 10, 50, 10),                                  # whole box, 24 colours
]


@pytest.mark.parametrize("L,N,kw,relax,spl,steps,every", GPU_RELAXED)
def test_gpu_relaxed_melts_step_like_the_replay(L, N, kw, relax, spl, steps, every):
    """Melts relaxed on the GPU for thousands of steps, then compared with the
    replay over further steps (launches of several steps included)."""
    seed = 5000 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl, **kw)
    assert m.info().specialised == 1
    m.init_melt()
    m.run(relax)
    w, rec = m.state()
    assert occupied_fraction(w) > 0.6, "not relaxed"
    r = replay_like(m, seed)
    r.set_state(w, rec, m.step)
    compare_run(m, r, steps, every, f"L={L} N={N} {kw}")


def test_gpu_relaxed_linear_melt():
    seed = 5150
    m = elp.Melt(L=64, N=200, seed=seed, linear=1, periodic=0, tile=(32, 32, 32), steps_per_launch=10)
    m.init_melt()
    m.run(3000)
    w, rec = m.state()
    assert occupied_fraction(w) > 0.5
    r = replay_like(m, seed, linear=True)
    r.set_state(w, rec, m.step)
    compare_run(m, r, 50, 10, "linear L=64 N=200")


@pytest.mark.parametrize("L,N,kw,relax,spl", [
    (32, 20, dict(), 2000, 20),                                            # 1966 rings in 2048 slots
    (64, 14, dict(periodic=0, tile=(32, 16, 16)), 2000, 10),               # ~700 monomer-0 runs per 1024-slot tile
    (64, 16, dict(periodic=0, tile=(16, 16, 16)), 2000, 10),               # ~310 per 512
])
def test_label_slots_near_capacity(L, N, kw, relax, spl):
    """Short rings: most tiles hold hundreds of monomer-0 runs, so the label
    slot table works close to capacity on every tile load."""
    seed = 6000 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl, **kw)
    assert m.info().specialised == 1
    m.init_melt()
    m.run(relax)
    w, rec = m.state()
    r = replay_like(m, seed)
    r.set_state(w, rec, m.step)
    compare_run(m, r, 40, 10, f"short rings L={L} N={N}")
    assert np.count_nonzero(w & 16) == m.P


@pytest.mark.parametrize("L,N,kw,spl", [
    (64, 14, dict(periodic=0, tile=(32, 16, 16)), 1),      # up to 2816 monomer-0 runs in a 1024-slot tile
    (64, 14, dict(periodic=0, tile=(32, 16, 16)), 10),
    (64, 30, dict(periodic=0, tile=(32, 32, 16)), 10),     # up to 1536 in 1024
    (64, 40, dict(periodic=0, tile=(32, 32, 32)), 10),     # up to 2112 in 1792
])
def test_crowded_tiles_take_the_general_move(L, N, kw, spl):
    """CreatePolymers stacks short rings in a slab, so some tiles hold more
    monomer-0 runs than their slot table: those tiles run the general move
    (bookkeeping in the chain records) and the step stays exact, from the
    initial melt on, every step."""
    seed = 6100 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl, **kw)
    assert m.info().specialised == 1
    m.init_melt()
    w, rec = m.state()
    r = replay_like(m, seed)
    r.set_state(w, rec, 0)
    compare_run(m, r, 30, spl, f"crowded L={L} N={N} {kw}")
    m.run(200)
    m.sync()
    assert m.check() == 0


@pytest.mark.parametrize("L,N,seed,spl,relax,steps,every", [
    (128, 1000, 7, 100, 2000, 50, 10),    # the bench's headline melt, its geometry and launch shape
    (256, 5000, 11, 10, 2000, 10, 5),     # the roofline melt
])
def test_bench_melts_relaxed_match_replay(L, N, seed, spl, relax, steps, every):
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl)
    m.init_melt()
    m.run(relax)
    w, rec = m.state()
    assert occupied_fraction(w) > 0.2
    r = replay_like(m, seed)
    r.set_state(w, rec, m.step)
    compare_run(m, r, steps, every, f"L={L} N={N}")
