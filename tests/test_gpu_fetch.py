"""Chain fetch by list ranking (csrc/elp_rank.cu) against the chain walk.

elp_fetch_chains rebuilds the chains of boxes up to L = 512 by list
ranking: every run jumps along its chain by doubling strides, so the fetch
takes ceil(log2 N) passes over the lattice instead of one ring's chain of
dependent loads.  elp_fetch_checked keeps the chain walk (elp_walk.cu),
which follows each ring run by run as the reference's host code does
(gpupol2/oclpol.c:183-376).  The two must give the same bytes on every
melt, and both must reject a broken chain.
"""
import numpy as np
import pytest

import elp

pytestmark = pytest.mark.gpu

VALID = [b for b in range(16) if b not in (0, 3, 12, 15)]


def step_site(s, b, L):
    t, u, v = s % L, (s // L) % L, s // (L * L)
    t = (t + (b & 1) - ((b >> 3) & 1)) % L
    u = (u + ((b >> 1) & 1) - ((b >> 3) & 1)) % L
    v = (v + ((b >> 2) & 1) - ((b >> 3) & 1)) % L
    return t + L * (u + L * v)


def assert_fetches_agree(m):
    s1, b1 = m.fetch()
    s2, b2, code = m.fetch_checked()
    assert code == 0
    assert np.array_equal(s1, s2), "start sites differ between list ranking and the walk"
    assert np.array_equal(b1, b2), "bonds differ between list ranking and the walk"


@pytest.mark.parametrize("L,N,kw,steps", [
    (16, 50, dict(), 500),
    (32, 100, dict(), 2000),
    (24, 60, dict(), 1000),
    (64, 200, dict(), 2000),
    (64, 14, dict(), 1000),                   # short rings: many labelled runs
    (16, 2000, dict(), 400),                  # rings longer than the box, wrapping it
    (128, 1000, dict(steps_per_launch=20), 2000),
    (32, 100, dict(linear=1), 2000),
    (64, 200, dict(linear=1, periodic=0, tile=(32, 32, 32)), 2000),
])
def test_list_ranking_equals_the_walk(L, N, kw, steps):
    m = elp.Melt(L=L, N=N, seed=77, **kw)
    m.init_melt()
    assert_fetches_agree(m)              # the collapsed initial melt
    m.run(steps)
    assert_fetches_agree(m)              # relaxed


def test_list_ranking_on_the_longest_rings_and_the_large_box():
    m = elp.Melt(L=64, N=65536, seed=64)
    m.init_melt()
    m.run(20)
    assert_fetches_agree(m)
    m = elp.Melt(L=256, N=5000, seed=11, steps_per_launch=10)
    m.init_melt()
    m.run(500)
    assert_fetches_agree(m)


def test_batch_fetch_equals_its_single_runs():
    specs = [dict(L=16, N=50, seed=5), dict(L=48, N=300, seed=6), dict(L=64, N=100, seed=7, linear=1)]
    b = elp.Batch(specs)
    b.init_melts()
    b.run(300)
    for j, sp in enumerate(specs):
        m = elp.Melt(**sp)
        m.init_melt()
        m.run(300)
        sa, ba = b.fetch(j)
        sb, bb, code = m.fetch_checked()
        assert code == 0 and np.array_equal(sa, sb) and np.array_equal(ba, bb)


def corrupt(w, L, kind, rng):
    """A copy of the site words with one chain broken (host-side fault)."""
    w = w.copy()
    plain = np.flatnonzero((w != 0) & ((w & 16) == 0))
    if kind == "bond":           # not a lattice bond
        k = int(plain[len(plain) // 2])
        w[k] = (w[k] & ~np.uint32(15)) | np.uint32(3)
    elif kind == "empty":        # a run leading to an empty site
        for k in rng.permutation(plain):
            for b in VALID:
                if w[step_site(int(k), b, L)] == 0:
                    w[k] = (w[k] & ~np.uint32(15)) | np.uint32(b)
                    return w
        raise AssertionError("no run next to an empty site")
    elif kind == "merge":        # a run leading into the middle of another run's chain
        for k in rng.permutation(plain):
            k = int(k)
            succ = step_site(k, int(w[k] & 15), L)
            for b in VALID:
                n = step_site(k, b, L)
                if n != succ and w[n] != 0 and not (w[n] & 16):
                    w[k] = (w[k] & ~np.uint32(15)) | np.uint32(b)
                    return w
        raise AssertionError("no run next to another chain")
    elif kind == "label":        # a chain's labelled run loses its label
        k = int(np.flatnonzero(w & 16)[0])
        w[k] = (w[k] & np.uint32(15)) | np.uint32(2 << 16)
    return w


@pytest.mark.parametrize("kind", ["bond", "empty", "merge", "label"])
@pytest.mark.parametrize("linear", [0, 1])
def test_broken_chains_are_rejected(kind, linear):
    rng = np.random.default_rng(5)
    m = elp.Melt(L=32, N=100, seed=19, linear=linear)
    m.init_melt()
    m.run(1500)
    w, r = m.state()
    m.set_state(corrupt(w, 32, kind, rng), r, m.step)
    with pytest.raises(elp.ElpError) as e:
        m.fetch()
    assert e.value.status == elp.ERR_INTEGRITY
    assert m.fetch_checked()[2] != 0
    m.set_state(w, r, m.step)            # the context stays usable
    assert_fetches_agree(m)
