"""Host tools around the melt files against the reference's own tools.

tests/golden/scaleup_*.res.gz, xyz_*.txt.gz, pov_*.pov.gz and
pov_sha256.json were written by the reference's analysis/scaleup.c,
analysis/tuv2xyz.c and analysis/tuv2pov.c (built from its sources,
tests/golden/make_golden.py) from committed reference TUV files.
elp_scaleup_tuv / elp_tuv_to_xyz / elp_tuv_to_pov, and the drop-in programs
bin/scaleup, bin/tuv2xyz and bin/tuv2pov built on them, must write the same
bytes and exit codes."""
import gzip
import hashlib
import json
import os
import subprocess

import pytest

import elp
import observables as obs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "mc-polymer-simulation_b200", "bin")


def unpack(tmp_path, name):
    p = tmp_path / name.replace(".gz", "")
    with gzip.open(os.path.join(GOLD, name), "rb") as f:
        p.write_bytes(f.read())
    return p


@pytest.mark.parametrize("name", ["efpol_L16_N50_s3_t100", "efpol_L32_N100_s1_t0", "efpol_L32_N100_s1_t200"])
def test_scaleup_matches_reference(tmp_path, name):
    src = unpack(tmp_path, name + ".res.gz")
    want = gzip.open(os.path.join(GOLD, f"scaleup_{name}.res.gz"), "rb").read()
    out = tmp_path / "lib.res"
    elp.check(elp.lib().elp_scaleup_tuv(str(src).encode(), str(out).encode()))
    assert out.read_bytes() == want
    cli = tmp_path / "cli.res"
    assert subprocess.run([os.path.join(BIN, "scaleup"), str(src), str(cli)], timeout=60).returncode == 0
    assert cli.read_bytes() == want
    # a valid melt: every upscaled ring closes, no site is shared (oracle check)
    from oracle_binding import Efpol
    L, start, bonds = obs.parse_tuv(want.decode())
    e = Efpol(L, bonds.shape[1], bonds.shape[0], 0)
    assert e.read(obs.format_tuv(L, start, bonds)) == 0 and e.check() == 0


@pytest.mark.parametrize("pid", [0, 3, 97])
def test_tuv2xyz_matches_reference(tmp_path, pid):
    src = unpack(tmp_path, "efpol_L16_N50_s3_t100.res.gz")
    want = gzip.open(os.path.join(GOLD, f"xyz_efpol_L16_N50_s3_t100_p{pid}.txt.gz"), "rb").read()
    out = tmp_path / "x.txt"
    assert subprocess.run([os.path.join(BIN, "tuv2xyz"), str(src), str(out), str(pid)], timeout=60).returncode == 0
    assert out.read_bytes() == want


def test_tools_exit_codes(tmp_path):
    src = unpack(tmp_path, "efpol_L16_N50_s3_t100.res.gz")
    assert subprocess.run([os.path.join(BIN, "scaleup"), str(src)], capture_output=True).returncode == 192
    assert subprocess.run([os.path.join(BIN, "scaleup"), str(tmp_path / "missing.res"), str(tmp_path / "o")],
                          capture_output=True).returncode == 192
    assert subprocess.run([os.path.join(BIN, "tuv2xyz"), str(src), str(tmp_path / "o")],
                          capture_output=True).returncode == 192
    assert subprocess.run([os.path.join(BIN, "tuv2xyz"), str(src), str(tmp_path / "o"), "98"],
                          capture_output=True).returncode == 193


def test_tuv2pov_one_ring_matches_reference(tmp_path):
    src = unpack(tmp_path, "efpol_L16_N50_s3_t100.res.gz")
    want = gzip.open(os.path.join(GOLD, "pov_efpol_L16_N50_s3_t100_p3.pov.gz"), "rb").read()
    out = tmp_path / "lib.pov"
    elp.check(elp.lib().elp_tuv_to_pov(str(src).encode(), str(out).encode(), 3))
    assert out.read_bytes() == want
    cli = tmp_path / "cli.pov"
    assert subprocess.run([os.path.join(BIN, "tuv2pov"), str(src), str(cli), "3"], timeout=60).returncode == 0
    assert cli.read_bytes() == want


@pytest.mark.parametrize("key", ["efpol_L16_N50_s3_t100/-1", "efpol_L32_N100_s1_t0/-1",
                                 "efpol_lin_L32_N100_s1_t200/-1", "efpol_lin_L32_N100_s1_t200/0"])
def test_tuv2pov_scenes_match_reference(tmp_path, key):
    """Whole-melt scenes (rings, compact t=0 rings, linear chains) and one
    linear chain: the SHA-256 of the reference's scene text."""
    name, pid = key.split("/")
    want = json.load(open(os.path.join(GOLD, "pov_sha256.json")))[key]
    src = unpack(tmp_path, name + ".res.gz")
    out = tmp_path / "s.pov"
    args = [os.path.join(BIN, "tuv2pov"), str(src), str(out)] + ([pid] if int(pid) >= 0 else [])
    assert subprocess.run(args, timeout=60).returncode == 0
    assert hashlib.sha256(out.read_bytes()).hexdigest() == want


def test_tuv2pov_exit_codes(tmp_path):
    src = unpack(tmp_path, "efpol_L16_N50_s3_t100.res.gz")
    run = lambda *a: subprocess.run([os.path.join(BIN, "tuv2pov")] + [str(x) for x in a], capture_output=True)
    assert run(src).returncode == 192                                   # missing POV_FILE
    assert run(tmp_path / "missing.res", tmp_path / "o.pov").returncode == 192
    assert run(src, tmp_path / "o.pov", 98).returncode == 193           # np= 98: chains 0..97
