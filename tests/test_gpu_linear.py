"""Linear chains (efpol built with POL_TYPE=POL_LIN, efpol_lin) on the GPU.

Same bar as rings: the kernel state equals the host replay (oracle/replay.c,
linear mode) after every step, the initial melt is the reference efpol_lin's
t=0 file byte for byte, reference efpol_lin states load and stay valid
chains (oracle integrity check), resumes are bit-identical, batch members
equal single runs and the in-situ observables match the observables oracle.
Statistics against efpol_lin ensembles are in test_gpu_stats.py."""
import gzip
import os

import numpy as np
import pytest

import elp
import observables as obs
from oracle_binding import Efpol, Replay

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(REPO, "tests", "golden")


def replay_for(m: elp.Melt, seed, salt=0):
    i = m.info()
    return Replay(i.L, i.N, i.P, seed=seed, salt=salt, periodic=bool(i.periodic), tile=tuple(i.tile), ncol=i.ncol,
                  linear=True)


def efpol_lin_start(L, N, P):
    e = Efpol(L, N, P, 0, pol_type=2)
    e.create()
    return e.export()


CASES = [
    (16, 50, dict(), 12),                                   # whole box, 16 colours
    (32, 100, dict(), 6),                                   # whole box
    (24, 60, dict(), 6),                                    # whole box, 24 colours
    (32, 100, dict(periodic=0, tile=(16, 16, 16)), 8),      # tiled with origin shifts
    (64, 200, dict(periodic=0, tile=(32, 32, 32)), 3),
    (48, 100, dict(periodic=0, tile=(48, 24, 24)), 3),
    (64, 150, dict(periodic=0, tile=(32, 16, 16)), 3),      # two CTAs per SM
]


@pytest.mark.parametrize("L,N,kw,steps", CASES)
def test_linear_kernel_matches_replay_every_step(L, N, kw, steps):
    seed = 2000 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, linear=1, **kw)
    assert m.info().linear == 1 and m.info().specialised == 1
    m.init_melt()
    r = replay_for(m, seed)
    start, bonds = efpol_lin_start(L, N, m.P)
    assert r.load(start, bonds) == 0
    w, rec = m.state()
    assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())
    for s in range(steps):
        m.run(1)
        r.steps(1)
        w, rec = m.state()
        assert np.array_equal(w, r.lattice()), f"site words differ after step {s + 1}"
        assert np.array_equal(rec, r.records()), f"records differ after step {s + 1}"
    assert m.check() == 0
    assert m.accepted() == r.accepted


def test_linear_initial_melt_is_reference_t0(tmp_path):
    m = elp.Melt(L=32, N=100, seed=1, linear=1)
    m.init_melt()
    m.write_tuv(str(tmp_path / "t0.res"))
    want = gzip.open(os.path.join(GOLD, "efpol_lin_L32_N100_s1_t0.res.gz"), "rt").read()
    assert (tmp_path / "t0.res").read_text() == want


def test_reference_linear_state_runs_and_stays_valid(tmp_path):
    src = tmp_path / "t200.res"
    src.write_bytes(gzip.open(os.path.join(GOLD, "efpol_lin_L32_N100_s1_t200.res.gz"), "rb").read())
    m = elp.Melt(L=32, N=100, seed=5, linear=1, periodic=0, tile=(16, 16, 16))
    m.load_tuv(str(src), 200)
    s0, b0 = m.fetch()
    L, start, bonds = obs.read_tuv(str(src))
    assert np.array_equal(s0, start) and np.array_equal(b0, bonds)
    m.run(300)
    assert m.check() == 0
    s1, b1 = m.fetch()
    assert np.all(b1[:, -1] == 15) and not np.any(b1[:, :-1] == 15)
    e = Efpol(32, 100, m.P, 0, pol_type=2)
    assert e.read(obs.format_tuv(32, s1, b1)) == 0 and e.check() == 0
    assert np.any(s1 != s0)       # monomer 0 moves


def test_linear_resume_is_bit_identical(tmp_path):
    a = elp.Melt(L=32, N=100, seed=8, linear=1)
    a.init_melt()
    a.run(120)
    b = elp.Melt(L=32, N=100, seed=8, linear=1)
    b.init_melt()
    b.run(60)
    b.write_tuv(str(tmp_path / "t60.res"))
    c = elp.Melt(L=32, N=100, seed=8, linear=1)
    c.load_tuv(str(tmp_path / "t60.res"), 60)
    c.run(60)
    sa, ba = a.fetch()
    sc, bc = c.fetch()
    assert np.array_equal(sa, sc) and np.array_equal(ba, bc)


def test_linear_batch_members_equal_single_runs():
    specs = [dict(L=16, N=50, seed=41, linear=1), dict(L=32, N=100, seed=42), dict(L=32, N=80, seed=43, linear=1),
             dict(L=64, N=200, seed=44, linear=1, periodic=0, tile=(32, 32, 32))]
    b = elp.Batch(specs)
    b.init_melts()
    b.run(20)
    for j, kw in enumerate(specs):
        m = elp.Melt(**kw)
        m.init_melt()
        m.run(20)
        wb, rb = b.state(j)
        wm, rm = m.state()
        assert np.array_equal(wb, wm) and np.array_equal(rb, rm), j
        assert b.check(j) == 0


def test_linear_observe_matches_oracle():
    m = elp.Melt(L=32, N=100, seed=45, linear=1)
    m.init_melt()
    m.run(200)
    got = m.observe(16)
    start, bonds = m.fetch()
    start = start.astype(np.int64)
    rg2, _, sl = obs.chain_stats(start, bonds)
    np.testing.assert_allclose(got["rg2"], rg2, rtol=1e-12)
    np.testing.assert_allclose(got["cms_tuv"], obs.cms_tuv(start, bonds), rtol=1e-12, atol=1e-9)
    assert np.array_equal(got["sl"], sl)                       # zero bonds / (N - 1)
    assert np.array_equal(got["run_hist"].astype(np.int64), obs.run_length_hist(bonds, 16))


def test_linear_rejected_where_unsupported():
    with pytest.raises(elp.ElpError) as e:
        elp.Melt(L=32, N=100, linear=1, kernel=1)               # generic kernel: rings only
    assert e.value.status == elp.ERR_ARG
    with pytest.raises(elp.ElpError) as e:
        elp.Melt(L=32, N=50, linear=1, periodic=0, tile=(32, 16, 8))   # no specialised shape
    assert e.value.status == elp.ERR_ARG
    # the serving loop takes linear jobs (tests/test_gpu_server.py); one whose
    # box has no specialised shape finishes with ELP_ERR_ARG
    s = elp.Server(quantum=10)
    jid = s.submit(100, L=32, N=50, linear=1, periodic=0, tile=(32, 16, 8))
    s.drain(120)
    r = s.poll()
    assert len(r) == 1 and r[0]["id"] == jid and r[0]["status"] == elp.ERR_ARG
    s.close()
