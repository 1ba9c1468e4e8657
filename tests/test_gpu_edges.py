"""Edge cases at the limits of the engine: the smallest ring (N=3), the
smallest workable box (L=14: the colour modulus must divide L and be at
least 13, and a substep's anchors come in groups of four, so odd boxes and
boxes below 14 are refused cleanly), a single ring, the longest rings the
16-bit run lengths allow (N=65536) and the longest linear chains (65535),
and a ragged TUV file.  Each runs against the host replay
or the integrity check, or must fail with a clean status."""
import os

import numpy as np
import pytest

import elp
import observables as obs
from oracle_binding import Efpol, Replay

pytestmark = pytest.mark.gpu


def replay_check(m, seed, steps, linear=False):
    i = m.info()
    r = Replay(i.L, i.N, i.P, seed=seed, periodic=bool(i.periodic), tile=tuple(i.tile), ncol=i.ncol, linear=linear)
    start, bonds = m.fetch()
    assert r.load(start, bonds) == 0
    for _ in range(steps):
        m.run(1)
        r.steps(1)
        w, rec = m.state()
        assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())
    assert m.check() == 0


def test_smallest_ring():
    m = elp.Melt(L=16, N=3, seed=61)
    assert m.P == int(1.2 * 16 ** 3 / 3 + 0.5)
    m.init_melt()
    replay_check(m, 61, 5)


def test_smallest_box_runs_the_generic_kernel():
    m = elp.Melt(L=14, N=20, seed=62)
    i = m.info()
    assert i.ncol == 14 and i.periodic == 1 and i.specialised == 0
    m.init_melt()
    replay_check(m, 62, 5)
    for L in (12, 13, 15):
        with pytest.raises(elp.ElpError) as e:
            elp.Melt(L=L, N=20)
        assert e.value.status == elp.ERR_ARG, L


def test_single_ring():
    m = elp.Melt(L=16, N=50, P=1, seed=63)
    assert m.P == 1
    m.init_melt()
    replay_check(m, 63, 20)
    # a vanishing density still gives one ring, as efpol's MAX(GetNPol, 1)
    assert elp.Melt(L=16, N=50, density=1e-6).P == 1


@pytest.mark.parametrize("N,linear", [(65536, 0), (65535, 1)])
def test_longest_chains(N, linear):
    m = elp.Melt(L=64, N=N, seed=64, linear=linear)
    m.init_melt()
    m.run(3)
    assert m.check() == 0
    s, b = m.fetch()
    m2 = elp.Melt(L=64, N=N, seed=64, linear=linear)
    m2.load_chains(s, b, 3)
    w1, r1 = m.state()
    w2, r2 = m2.state()
    assert np.array_equal(w1, w2) and np.array_equal(r1, r2)
    assert int(r1[:, 1].max()) <= 65535


def test_limits_refused_cleanly(tmp_path):
    for kw in (dict(L=64, N=65537), dict(L=64, N=65536, linear=1), dict(L=16, N=2)):
        with pytest.raises(elp.ElpError) as e:
            elp.Melt(**kw)
        assert e.value.status == elp.ERR_ARG, kw
    # a ragged file: one ring shorter than the header's maxPolLength
    m = elp.Melt(L=16, N=50, seed=65)
    m.init_melt()
    s, b = m.fetch()
    text = obs.format_tuv(16, s, b).replace("len= 50\n", "len= 49\n", 1)
    lines = text.split("\n")
    k = next(i for i, l in enumerate(lines) if l.startswith("len= 49"))
    lines[k + 1] = lines[k + 1][:-1]
    p = tmp_path / "ragged.res"
    p.write_text("\n".join(lines))
    with pytest.raises(elp.ElpError) as e:
        m.load_tuv(str(p))
    assert e.value.status == elp.ERR_FORMAT


def test_kernel_count_of_a_run():
    """elp_info.kernels counts the sweep path's kernels: one per launch, and
    a CUDA-graph replay (tiled melts, 100 steps per graph) its launches plus
    the step-counter update."""
    m = elp.Melt(L=16, N=50, seed=3, steps_per_launch=10)     # whole box: direct launches
    m.init_melt()
    k0 = m.info().kernels
    m.run(35)
    assert m.info().kernels - k0 == 4
    m = elp.Melt(L=64, N=200, seed=3, periodic=0, tile=(32, 32, 32), steps_per_launch=20)
    m.init_melt()
    k0 = m.info().kernels
    m.run(20)                      # fewer steps than a graph: one launch
    assert m.info().kernels - k0 == 1
    m.run(230)                     # two graph replays of 5 launches + counter, then 30 steps: 2 launches
    assert m.info().kernels - k0 == 1 + 2 * 6 + 2
    assert m.check() == 0
