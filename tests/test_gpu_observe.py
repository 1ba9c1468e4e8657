"""In-situ observables (elp_observe) against the observables oracle.

The device sums exact integers per ring; the oracle (oracle/observables.py,
numpy float64, following analysis/mode_compute.c:145-217) computes the same
quantities from the rings fetched to the host.  Tolerances: the centre of
mass and Rg^2 within 1e-12 relative (different summation order in float64),
the stored-length fraction and the run-length histogram exactly."""
import numpy as np
import pytest

import elp
import observables as obs

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def oracle(start, bonds, nbins):
    start = start.astype(np.int64)
    rg2, _, sl = obs.chain_stats(start, bonds)
    return dict(cms_tuv=obs.cms_tuv(start, bonds), rg2=rg2, sl=sl, run_hist=obs.run_length_hist(bonds, nbins))


def compare(got, want):
    np.testing.assert_allclose(got["cms_tuv"], want["cms_tuv"], rtol=RTOL, atol=1e-9)
    np.testing.assert_allclose(got["rg2"], want["rg2"], rtol=RTOL)
    assert np.array_equal(got["sl"], want["sl"])
    assert np.array_equal(got["run_hist"].astype(np.int64), want["run_hist"])


@pytest.mark.parametrize("kw,steps,nbins", [
    (dict(L=16, N=50, seed=21), 0, 16),
    (dict(L=16, N=50, seed=21), 300, 16),
    (dict(L=32, N=100, seed=22), 150, 64),
    (dict(L=24, N=200, seed=23), 200, 8),
    (dict(L=64, N=500, seed=24, periodic=0, tile=(32, 32, 32)), 40, 16),
    (dict(L=128, N=1000, seed=25), 20, 16),
])
def test_observe_matches_oracle(kw, steps, nbins):
    m = elp.Melt(**kw)
    m.init_melt()
    if steps:
        m.run(steps)
    got = m.observe(nbins)
    start, bonds = m.fetch()
    compare(got, oracle(start, bonds, nbins))
    assert got["run_hist"].sum() > 0


def test_observe_long_rings_that_wrap_the_box():
    """Rings longer than the box edge: positions are unwrapped along the ring."""
    m = elp.Melt(L=16, N=2000, seed=26)
    m.init_melt()
    m.run(500)
    got = m.observe(32)
    start, bonds = m.fetch()
    compare(got, oracle(start, bonds, 32))


def test_batch_observe_equals_single():
    specs = [dict(L=16, N=50, seed=31), dict(L=32, N=120, seed=32), dict(L=48, N=300, seed=33)]
    b = elp.Batch(specs)
    b.init_melts()
    b.run(30)
    for j, kw in enumerate(specs):
        m = elp.Melt(**kw)
        m.init_melt()
        m.run(30)
        got, want = b.observe(j, 16), m.observe(16)
        for k in want:
            assert np.array_equal(got[k], want[k]), k
        start, bonds = b.fetch(j)
        compare(got, oracle(start, bonds, 16))


def test_observe_rejects_bad_arguments_and_broken_rings():
    m = elp.Melt(L=16, N=50, seed=34)
    m.init_melt()
    with pytest.raises(elp.ElpError) as e:
        m.observe(elp.OBS_MAX_BINS + 1)
    assert e.value.status == elp.ERR_ARG
    w, r = m.state()
    bad = w.copy()
    k = int(np.flatnonzero((bad != 0) & ((bad & 16) == 0))[0])
    bad[k] = (bad[k] & ~np.uint32(15)) | np.uint32(3)   # invalid bond code
    m.set_state(bad, r, 0)
    with pytest.raises(elp.ElpError) as e:
        m.observe(16)
    assert e.value.status == elp.ERR_INTEGRITY
