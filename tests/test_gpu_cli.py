"""Drop-in front-ends: same arguments, directories, file names and exit
codes as the reference programs, so do_run.sh and the analysis run on their
output unchanged."""
import gzip
import os
import subprocess

import pytest

import observables as obs
from oracle_binding import Efpol

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "mc-polymer-simulation_b200", "bin")
GOLD = os.path.join(REPO, "tests", "golden")

# keys and order of cpupol/efpol_io.c:111-140, as the reference's own run wrote them
EFPOL_KEYS = ["Start_seed", "Length", "Polytype", "Density", "Latsize", "Start_polysize", "Double_step", "Interval",
              "Equilibrated", "Npol", "Polymodel", "Executable"]


def test_efpol_ring_cli(tmp_path):
    out = tmp_path / "run"
    r = subprocess.run([os.path.join(BIN, "efpol_ring"), "1", str(out), "1.2", "200", "100", "100", "0", "32",
                        "sl_equal"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    d = out / "N_100"
    assert sorted(os.listdir(d)) == ["simulation_settings.txt", "t=0_dev=0.res", "t=100_dev=0.res", "t=200_dev=0.res"]
    ref0 = gzip.open(os.path.join(GOLD, "efpol_L32_N100_s1_t0.res.gz"), "rt").read()
    assert (d / "t=0_dev=0.res").read_text() == ref0
    for t in (100, 200):
        L, start, bonds = obs.parse_tuv((d / f"t={t}_dev=0.res").read_text())
        e = Efpol(32, 100, start.shape[0], 0)
        assert e.read(obs.format_tuv(L, start, bonds)) == 0 and e.check() == 0
    keys = [ln.split(" = ")[0] for ln in (d / "simulation_settings.txt").read_text().splitlines()]
    assert keys == EFPOL_KEYS
    assert "Npol = 393" in (d / "simulation_settings.txt").read_text()


def test_efpol_ring_cli_rejects_unsupported(tmp_path):
    r = subprocess.run([os.path.join(BIN, "efpol_ring"), "1", str(tmp_path), "1.2", "10", "5", "100", "0", "32",
                        "sl_nonsense"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 193


def test_gpupol_cli_resume_is_bit_identical(tmp_path):
    exe = os.path.join(BIN, "gpupol3_cuda_ring")
    a, b = tmp_path / "a", tmp_path / "b"
    args = ["100", "{T}", "7", "{D}", "1.2", "0", "100", "32", "32", "32"]
    run = lambda T, D: subprocess.run([exe] + [x.format(T=T, D=D) for x in args], capture_output=True, text=True,
                                      timeout=120)
    assert run(400, a).returncode == 0
    assert run(200, b).returncode == 0
    assert run(200, b).returncode == 0            # resumes from t=200 and runs 200 more
    for t in (0, 100, 200, 300, 400):
        assert (a / f"t={t}_dev=0.res").read_text() == (b / f"t={t}_dev=0.res").read_text(), t
    s = (a / "simulation_settings.txt").read_text()
    assert "Executable = efpol" in s and "Npol = 393" in s


@pytest.mark.parametrize("L", [64, 48])
def test_tiled_run_names_its_clock(tmp_path, L):
    """A tiled run writes Executable = elp_<tile shape>; the shape has a
    measured time factor, and bin/elp_ne_list gives the analysis its line
    (Ne of efpol, tFac / f) from efpol's."""
    import elp
    d = tmp_path / "run"
    r = subprocess.run([os.path.join(BIN, "gpupol3_cuda_ring"), "100", "40", "7", str(d), "1.2", "0", "20", str(L),
                        str(L), str(L)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    s = (d / "simulation_settings.txt").read_text()
    exe = [ln.split(" = ")[1] for ln in s.splitlines() if ln.startswith("Executable = ")][0]
    assert exe.startswith("elp_"), exe
    tile = tuple(int(v) for v in exe[len("elp_"):].split("x"))
    f = elp.time_factor(0, *tile)
    assert 0 < f < 1
    ne = tmp_path / "ne_list.dat"
    ne.write_text("efpol 1.2 124 1.08 0.85 30\n")
    lines = subprocess.run([os.path.join(BIN, "elp_ne_list"), str(ne)], capture_output=True, text=True,
                           check=True).stdout.splitlines()
    mine = [ln.split() for ln in lines if ln.startswith(exe + " ")]
    assert len(mine) == 1 and mine[0][1] == "1.2" and mine[0][2] == "124"
    assert abs(float(mine[0][4]) - 0.85 / f) < 1e-3


def _ptl_from_tuv_files(d, times):
    """The per-ring files the reference's create_ptl would build from the TUV
    dumps in d (analysis/create_ptl.c:46-115), made by the writer the tests pin
    to create_ptl's own output (test_ptl.py)."""
    import elp
    dumps = [obs.parse_tuv((d / f"t={t}_dev=0.res").read_text())[1:] for t in times]
    P, N = dumps[0][1].shape
    ref = d.parent / (d.name + "_ref")
    w = elp.PTLWriter(str(ref), P, N, len(dumps))
    for start, bonds in dumps:
        w.append(start, bonds)
    w.close()
    return {n: (ref / "ptl" / n).read_text() for n in os.listdir(ref / "ptl")}


@pytest.mark.parametrize("prog", ["efpol_ring", "gpupol3_cuda_ring"])
def test_cli_writes_ptl_in_situ(tmp_path, prog):
    out = tmp_path / "run"
    env = dict(os.environ, ELP_PTL="1")
    if prog == "efpol_ring":
        cmd = [os.path.join(BIN, prog), "5", str(out), "1.2", "250", "50", "60", "0", "16", "sl_equal"]
        d, times = out / "N_60", [0, 50, 100, 150, 200, 250]
    else:
        cmd = [os.path.join(BIN, prog), "60", "250", "5", str(out), "1.2", "0", "50", "16", "16", "16"]
        d, times = out, [0, 50, 100, 150, 200, 250]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    got = {n: (d / "ptl" / n).read_text() for n in os.listdir(d / "ptl")}
    assert got == _ptl_from_tuv_files(d, times)
    # newer than the settings file: create_ptl's NeedsUpdatePath (util/file.c:3-33) skips the pass
    assert os.stat(d / "ptl" / "pol=0_dev=0.res").st_mtime >= os.stat(d / "simulation_settings.txt").st_mtime


def test_efpol_ring_cli_doubling(tmp_path):
    """DBLSTEP=1: L=16, N=50 for TIME steps, DoubleLattice, then L=32, N=400
    (cpupol/efpol.c:84-101): both levels' dumps and settings, and the second
    level starting from the doubled last state of the first."""
    import elp
    out = tmp_path / "run"
    r = subprocess.run([os.path.join(BIN, "efpol_ring"), "9", str(out), "1.2", "100", "50", "400", "1", "32",
                        "sl_equal"], capture_output=True, text=True, timeout=180)
    assert r.returncode == 0, r.stderr
    for n, L in ((50, 16), (400, 32)):
        d = out / f"N_{n}"
        assert sorted(os.listdir(d)) == ["simulation_settings.txt", "t=0_dev=0.res", "t=100_dev=0.res",
                                         "t=50_dev=0.res"]
        for t in (0, 50, 100):
            Lf, start, bonds = obs.parse_tuv((d / f"t={t}_dev=0.res").read_text())
            assert Lf == L and bonds.shape == (98, n)
            e = Efpol(L, n, 98, 0)
            assert e.read(obs.format_tuv(Lf, start, bonds)) == 0 and e.check() == 0
        s = (d / "simulation_settings.txt").read_text()
        assert f"Length = {n}\n" in s and f"Latsize = {L}\n" in s and "Start_polysize = 50\n" in s
        assert f"Double_step = {0 if n == 50 else 1}\n" in s and "Npol = 98\n" in s
    L, start, bonds = obs.parse_tuv((out / "N_50" / "t=100_dev=0.res").read_text())
    L2, s2, b2 = elp.double_chains(L, start, bonds)
    assert (out / "N_400" / "t=0_dev=0.res").read_text() == elp.format_tuv(L2, s2, b2)


def test_gpupol_doubling_flow_with_scaleup(tmp_path):
    """do_run.sh's GPU doubling (do_run.sh:290-330): run, scaleup the last
    dump into a new directory as t=0, run there with 8N in a box of 2L."""
    exe = os.path.join(BIN, "gpupol3_cuda_ring")
    a, b = tmp_path / "a", tmp_path / "b"
    r = subprocess.run([exe, "50", "100", "3", str(a), "1.2", "0", "50", "16", "16", "16"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    b.mkdir()
    assert subprocess.run([os.path.join(BIN, "scaleup"), str(a / "t=100_dev=0.res"), str(b / "t=0_dev=0.res")],
                          timeout=60).returncode == 0
    r = subprocess.run([exe, "400", "100", "3", str(b), "1.2", "0", "50", "32", "32", "32"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert sorted(x for x in os.listdir(b) if x.startswith("t=")) == ["t=0_dev=0.res", "t=100_dev=0.res",
                                                                      "t=50_dev=0.res"]
    L, start, bonds = obs.parse_tuv((b / "t=100_dev=0.res").read_text())
    assert L == 32 and bonds.shape == (98, 400)
    e = Efpol(32, 400, 98, 0)
    assert e.read(obs.format_tuv(L, start, bonds)) == 0 and e.check() == 0


def test_efpol_lin_cli(tmp_path):
    """efpol_lin: the reference's efpol built for linear chains (do_run.sh
    runs efpol_$POL_TYPE with POL_TYPE=lin): t=0 file byte-identical, valid
    linear chains after, 'Polytype = lin', and doubling refused (193)."""
    out = tmp_path / "run"
    r = subprocess.run([os.path.join(BIN, "efpol_lin"), "1", str(out), "1.2", "200", "100", "100", "0", "32",
                        "sl_equal"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    d = out / "N_100"
    ref0 = gzip.open(os.path.join(GOLD, "efpol_lin_L32_N100_s1_t0.res.gz"), "rt").read()
    assert (d / "t=0_dev=0.res").read_text() == ref0
    for t in (100, 200):
        L, start, bonds = obs.parse_tuv((d / f"t={t}_dev=0.res").read_text())
        assert (bonds[:, -1] == 15).all()
        e = Efpol(32, 100, start.shape[0], 0, pol_type=2)
        assert e.read(obs.format_tuv(L, start, bonds)) == 0 and e.check() == 0
    s = (d / "simulation_settings.txt").read_text()
    assert "Polytype = lin\n" in s and [ln.split(" = ")[0] for ln in s.splitlines()] == EFPOL_KEYS
    r = subprocess.run([os.path.join(BIN, "efpol_lin"), "1", str(tmp_path / "x"), "1.2", "10", "5", "800", "1", "32",
                        "sl_equal"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 193


def test_gpupol_lin_cli_resume(tmp_path):
    exe = os.path.join(BIN, "gpupol3_cuda_lin")
    a, b = tmp_path / "a", tmp_path / "b"
    args = ["60", "{T}", "4", "{D}", "1.2", "0", "50", "16", "16", "16"]
    run = lambda T, D: subprocess.run([exe] + [x.format(T=T, D=D) for x in args], capture_output=True, text=True,
                                      timeout=120)
    assert run(200, a).returncode == 0
    assert run(100, b).returncode == 0
    assert run(100, b).returncode == 0
    for t in (0, 50, 100, 150, 200):
        assert (a / f"t={t}_dev=0.res").read_text() == (b / f"t={t}_dev=0.res").read_text(), t
    assert "Polytype = lin" in (a / "simulation_settings.txt").read_text()
