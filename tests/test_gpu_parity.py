"""Bit-exact parity of the sm_100a sweep kernel with the host replay.

The replay (oracle/replay.c) applies the same schedule -- origin shifts,
colours, anchors, Philox counters -- on the CPU; the GPU state (every site
word and every chain record) must equal it after every step.  The replay is in
turn tied to the reference: its initial states are the reference's t=0
configurations and its statistics match reference efpol (test_gpu_stats.py).
"""
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
    return Replay(i.L, i.N, i.P, seed=seed, salt=salt, periodic=bool(i.periodic),
                  tile=tuple(i.tile), ncol=i.ncol)


def efpol_start(L, N, P):
    e = Efpol(L, N, P, 0)
    e.create()
    return e.export()


CASES = [
    # (L, N, kwargs, steps)
    (16, 50, dict(), 12),                                   # whole box, 16 colours
    (32, 100, dict(), 6),                                   # the plain L=32 melt, whole box
    (24, 60, dict(), 6),                                    # whole box, 24 colours
    (32, 100, dict(periodic=0, tile=(16, 16, 16)), 8),      # tiled with origin shifts
    (64, 200, dict(periodic=0, tile=(32, 32, 32)), 3),
    (48, 100, dict(periodic=0, tile=(48, 24, 24)), 3),
    (64, 150, dict(periodic=0, tile=(32, 16, 16)), 3),      # two CTAs per SM
    (32, 50, dict(periodic=0, tile=(32, 16, 8)), 6),
]


@pytest.mark.parametrize("L,N,kw,steps", CASES)
def test_kernel_matches_replay_every_step(L, N, kw, steps):
    seed = 1000 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, **kw)
    m.init_melt()
    r = replay_for(m, seed)
    start, bonds = efpol_start(L, N, m.P)
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


def test_multi_step_launches_equal_single_steps():
    a = elp.Melt(L=16, N=50, seed=9, steps_per_launch=1)
    b = elp.Melt(L=16, N=50, seed=9, steps_per_launch=25)
    a.init_melt()
    b.init_melt()
    a.run(50)
    b.run(50)
    wa, ra = a.state()
    wb, rb = b.state()
    assert np.array_equal(wa, wb) and np.array_equal(ra, rb)


@pytest.mark.parametrize("L,N,kw,spl,steps", [
    (64, 200, dict(periodic=0, tile=(32, 32, 32)), 4, 9),
    (48, 100, dict(periodic=0, tile=(48, 24, 24)), 3, 7),
    (32, 100, dict(periodic=0, tile=(16, 16, 16)), 5, 10),
])
def test_tiled_multi_step_launches_match_replay(L, N, kw, spl, steps):
    """Tiled melts run several steps per launch (each tile waiting for the
    tiles of the previous step it overlaps); every launch boundary still
    matches the replay."""
    seed = 2000 + L + N
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl, **kw)
    m.init_melt()
    r = replay_for(m, seed)
    start, bonds = efpol_start(L, N, m.P)
    assert r.load(start, bonds) == 0
    done = 0
    while done < steps:
        k = min(spl, steps - done)
        m.run(k)
        r.steps(k)
        done += k
        w, rec = m.state()
        assert np.array_equal(w, r.lattice()), f"site words differ after step {done}"
        assert np.array_equal(rec, r.records()), f"records differ after step {done}"
    assert m.check() == 0
    assert m.accepted() == r.accepted


def test_tiled_steps_per_launch_do_not_change_bits():
    states = []
    for spl in (1, 3, 10, 64):
        m = elp.Melt(L=64, N=200, seed=5, steps_per_launch=spl)
        m.init_melt()
        m.run(167)                 # graph replays (100, 99, 100 or 2 x 64 steps) plus single launches
        states.append(m.state())
        assert m.check() == 0
    for w, rec in states[1:]:
        assert np.array_equal(w, states[0][0]) and np.array_equal(rec, states[0][1])


def test_initial_melt_is_reference_t0(tmp_path):
    m = elp.Melt(L=32, N=100, seed=1)
    m.init_melt()
    p = str(tmp_path / "t=0_dev=0.res")
    m.write_tuv(p)
    ref = gzip.open(os.path.join(GOLD, "efpol_L32_N100_s1_t0.res.gz"), "rt").read()
    assert open(p).read() == ref


def test_chains_roundtrip_through_device():
    text = gzip.open(os.path.join(GOLD, "efpol_L16_N50_s3_t100.res.gz"), "rt").read()
    L, start, bonds = obs.parse_tuv(text)
    m = elp.Melt(L=16, N=50, seed=3)
    m.load_chains(start, bonds)
    s2, b2 = m.fetch()
    assert np.array_equal(s2, start) and np.array_equal(b2, bonds)
    assert m.check() == 0


def test_resume_from_tuv_is_bit_identical(tmp_path):
    """A run stopped at a dump and resumed from the TUV file (with its step
    count) continues the same trajectory: the counter RNG is keyed by the
    absolute step."""
    a = elp.Melt(L=32, N=100, seed=5, periodic=0, tile=(16, 16, 16))
    a.init_melt()
    a.run(40)
    b = elp.Melt(L=32, N=100, seed=5, periodic=0, tile=(16, 16, 16))
    b.init_melt()
    b.run(17)
    p = str(tmp_path / "t=17_dev=0.res")
    b.write_tuv(p)
    c = elp.Melt(L=32, N=100, seed=5, periodic=0, tile=(16, 16, 16))
    c.load_tuv(p, step=17)
    c.run(23)
    wa, ra = a.state()
    wc, rc = c.state()
    assert np.array_equal(wa, wc) and np.array_equal(ra, rc)


def test_invariants_hold_over_a_long_run():
    m = elp.Melt(L=32, N=100, seed=77)
    m.init_melt()
    for _ in range(20):
        m.run(50)
        assert m.check() == 0
    start, bonds = m.fetch()
    e = Efpol(32, 100, m.P, 0)
    assert e.read(obs.format_tuv(32, start, bonds)) == 0
    assert e.check() == 0          # the reference's own integrity rules, restated


def test_large_box_invariants_and_conservation():
    """The L=256, N=5000 melt (20.1 M monomers): a few steps keep every
    invariant; the monomer total is conserved."""
    m = elp.Melt(L=256, N=5000, seed=11)
    assert m.P == 4027
    m.init_melt()
    m.run(3)
    assert m.check() == 0
    w, rec = m.state()
    counts = np.where(w & 16, 0, w >> 16).astype(np.int64).sum() + rec[:, 1].astype(np.int64).sum()
    assert counts == 5000 * 4027


def test_default_tile_shapes():
    """The default geometry follows the box: whole box up to L=32, then the
    tile shape with the highest measured physical rate (attempted moves/s
    times the shape's time factor): 16^3 below L=128, 32x16x16 from 128 to
    256, 32^3 above.  Every default shape has a measured time factor."""
    for L, N, tile in [(32, 100, None), (48, 100, (16, 16, 16)), (64, 200, (16, 16, 16)), (128, 1000, (32, 16, 16)),
                       (256, 5000, (32, 16, 16)), (320, 5000, (32, 32, 32))]:
        i = elp.Melt(L=L, N=N, seed=1).info()
        if tile is None:
            assert i.periodic == 1
            continue
        assert i.periodic == 0 and tuple(i.tile) == tile and i.specialised == 1, (L, tuple(i.tile))
        assert elp.time_factor(0, *tile) > 0


def test_l128_matches_replay():
    """The single large melt L=128, N=1000 (2517 rings), default geometry."""
    m = elp.Melt(L=128, N=1000, seed=7)
    assert m.P == 2517
    m.init_melt()
    r = replay_for(m, 7)
    assert r.load(*efpol_start(128, 1000, m.P)) == 0
    for _ in range(2):
        m.run(1)
        r.steps(1)
    w, rec = m.state()
    assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())


@pytest.mark.parametrize("L,N,seed,spl,steps", [(128, 1000, 7, 20, 3), (256, 5000, 11, 2, 2)])
def test_bench_workloads_match_replay_in_multi_step_launches(L, N, seed, spl, steps):
    """The bench's headline and roofline melts at full size, run as the bench
    runs them (several steps per launch), equal the replay."""
    m = elp.Melt(L=L, N=N, seed=seed, steps_per_launch=spl)
    m.init_melt()
    r = replay_for(m, seed)
    assert r.load(*efpol_start(L, N, m.P)) == 0
    m.run(steps)
    r.steps(steps)
    w, rec = m.state()
    assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())
    assert m.check() == 0 and m.accepted() == r.accepted


def test_bad_inputs_fail_cleanly(tmp_path):
    m = elp.Melt(L=16, N=50, seed=1)
    with pytest.raises(elp.ElpError) as e:
        m.run(1)                                   # nothing loaded yet
    assert e.value.status == elp.ERR_STATE
    with pytest.raises(elp.ElpError) as e:
        m.load_tuv(str(tmp_path / "missing.res"))
    assert e.value.status == elp.ERR_IO
    text = gzip.open(os.path.join(GOLD, "efpol_L16_N50_s3_t100.res.gz"), "rt").read()
    p = tmp_path / "garbled.res"
    p.write_text(text[: len(text) // 2] + "zz")
    with pytest.raises(elp.ElpError) as e:
        m.load_tuv(str(p))
    assert e.value.status == elp.ERR_FORMAT
    L, start, bonds = obs.parse_tuv(text)
    bad = bonds.copy()
    bad[3, int(np.flatnonzero(bad[3])[0])] = 0x3   # not a lattice bond
    with pytest.raises(elp.ElpError) as e:
        m.load_chains(start, bad)
    assert e.value.status == elp.ERR_INTEGRITY
    clash = start.copy()
    clash[1] = clash[0]                            # two rings on one site
    b2 = bonds.copy()
    b2[1] = b2[0]
    with pytest.raises(elp.ElpError) as e:
        m.load_chains(clash, b2)
    assert e.value.status == elp.ERR_INTEGRITY


@pytest.mark.parametrize("L,N,kw", [(16, 50, dict()), (24, 60, dict()), (32, 100, dict()),
                                     (64, 200, dict(periodic=0, tile=(32, 32, 32))),
                                     (64, 200, dict(periodic=0, tile=(32, 32, 16))),
                                     (64, 200, dict(periodic=0, tile=(32, 16, 16))),
                                     (32, 100, dict(periodic=0, tile=(16, 16, 16))),
                                     (48, 100, dict(periodic=0, tile=(48, 24, 24)))])
def test_specialised_kernels_equal_generic(L, N, kw):
    a = elp.Melt(L=L, N=N, seed=31, kernel=0, **kw)
    b = elp.Melt(L=L, N=N, seed=31, kernel=1, **kw)
    a.init_melt()
    b.init_melt()
    for _ in range(5):
        a.run(7)
        b.run(7)
        wa, ra = a.state()
        wb, rb = b.state()
        assert np.array_equal(wa, wb) and np.array_equal(ra, rb)
    assert a.accepted() == b.accepted()


@pytest.mark.parametrize("name,L,N,linear", [("efpol_L32_N100_s1_t200", 32, 100, 0),
                                             ("efpol_L16_N50_s3_t100", 16, 50, 0),
                                             ("efpol_lin_L32_N100_s1_t200", 32, 100, 1)])
def test_device_load_builds_the_replay_state(name, L, N, linear):
    """elp_load_chains builds site words and records on the device from the
    chains alone; they equal the host replay's load of the same chains."""
    _, start, bonds = obs.read_tuv(os.path.join(GOLD, name + ".res.gz"))
    m = elp.Melt(L=L, N=N, seed=1, linear=linear)
    m.load_chains(start, bonds, 7)
    r = Replay(L, N, m.P, 1, linear=bool(linear))
    assert r.load(start, bonds) == 0
    w, rec = m.state()
    assert np.array_equal(w, r.lattice()) and np.array_equal(rec, r.records())
    assert np.any(rec[:, 2] > 0) or linear          # rings with monomer 0 inside a run
    assert m.step == 7 and m.check() == 0


def test_device_load_of_rings_wrapping_the_box():
    m = elp.Melt(L=16, N=2000, seed=3)
    m.init_melt()
    m.run(400)
    s, b = m.fetch()
    m2 = elp.Melt(L=16, N=2000, seed=3)
    m2.load_chains(s, b, 400)
    w1, r1 = m.state()
    w2, r2 = m2.state()
    assert np.array_equal(w1, w2) and np.array_equal(r1, r2)


def test_fetch_checked_reports_a_corrupted_word():
    """Every dump of the drop-in programs goes through elp_fetch_checked: a
    word corrupted between intervals (elp_set_state) is caught at the next
    dump with efpol's code, not written out."""
    m = elp.Melt(L=32, N=100, seed=61)
    m.init_melt()
    m.run(300)
    s, b, code = m.fetch_checked()
    assert code == 0
    s2, b2 = m.fetch()
    assert np.array_equal(s, s2) and np.array_equal(b, b2)
    w, rec = m.state()
    bad = w.copy()
    i = int(np.flatnonzero((w != 0) & ((w & 16) == 0))[0])
    bad[i] = (bad[i] & ~np.uint32(15)) | np.uint32(3)        # not a lattice bond
    m.set_state(bad, rec, m.step)
    assert m.fetch_checked()[2] == 4
    dup = w.copy()
    j = int(np.flatnonzero(w == 0)[0])
    dup[j] = w[i]                                            # a run that no ring reaches
    m.set_state(dup, rec, m.step)
    assert m.fetch_checked()[2] != 0
