"""The PTL writer (elp_ptl_*) against the reference's create_ptl.

tests/golden/ptl_L16_N50_s3.json.gz holds the per-ring files that the
reference's analysis/create_ptl.c wrote for the reference efpol trajectory
efpol_L16_N50_s3_t{0..100}.  Feeding the same dumps to the writer must give
the same files byte for byte, whatever the buffer size.  Host only: the
writer needs no device."""
import ctypes as C
import gzip
import json
import os

import numpy as np
import pytest

import elp
import observables as obs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_ptl():
    with gzip.open(os.path.join(GOLD, "ptl_L16_N50_s3.json.gz")) as f:
        return json.loads(f.read())


def trajectory():
    out = []
    for t in range(0, 101, 10):
        L, start, bonds = obs.read_tuv(os.path.join(GOLD, f"efpol_L16_N50_s3_t{t}.res.gz"))
        out.append((start, bonds))
    return out


@pytest.mark.parametrize("buffer_bytes", [0, 1, 5000])
def test_ptl_writer_matches_reference_create_ptl(tmp_path, buffer_bytes):
    traj = trajectory()
    P, N = traj[0][1].shape
    w = elp.PTLWriter(str(tmp_path), P, N, len(traj), buffer_bytes=buffer_bytes)
    for start, bonds in traj:
        w.append(start, bonds)
    w.close()
    want = golden_ptl()
    got = {n: open(os.path.join(tmp_path, "ptl", n)).read() for n in sorted(os.listdir(tmp_path / "ptl"))}
    assert sorted(got) == sorted(want)
    for name in want:
        assert got[name] == want[name], name


def test_ptl_writer_rejects_bad_use(tmp_path):
    traj = trajectory()
    P, N = traj[0][1].shape
    lib = elp.lib()
    h = C.c_void_p()
    assert lib.elp_ptl_open(str(tmp_path).encode(), 0, 0, N, 2, 0, C.byref(h)) == elp.ERR_ARG
    assert lib.elp_ptl_open(str(tmp_path).encode(), 0, P, N, 0, 0, C.byref(h)) == elp.ERR_ARG
    # more dumps than announced
    w = elp.PTLWriter(str(tmp_path / "a"), P, N, 1)
    w.append(*traj[0])
    with pytest.raises(elp.ElpError) as e:
        w.append(*traj[1])
    assert e.value.status == elp.ERR_STATE
    w.close()
    # fewer dumps than announced: files are written, close reports it
    w = elp.PTLWriter(str(tmp_path / "b"), P, N, 3)
    w.append(*traj[0])
    with pytest.raises(elp.ElpError) as e:
        w.close()
    assert e.value.status == elp.ERR_STATE
    assert os.path.exists(tmp_path / "b" / "ptl" / "pol=0_dev=0.res")
    # a byte that is not a 4-bit bond code
    w = elp.PTLWriter(str(tmp_path / "c"), P, N, 1)
    bad = traj[0][1].copy()
    bad[3, 7] = 16
    with pytest.raises(elp.ElpError) as e:
        w.append(traj[0][0], bad)
    assert e.value.status == elp.ERR_ARG
    w.append(*traj[0])
    w.close()


def test_ptl_files_reload_as_the_trajectory(tmp_path):
    """What LoadPTL reads back (analysis/mode_io.c:509-606) is the trajectory."""
    traj = trajectory()
    P, N = traj[0][1].shape
    w = elp.PTLWriter(str(tmp_path), P, N, len(traj))
    for start, bonds in traj:
        w.append(start, bonds)
    w.close()
    for p in (0, 41, P - 1):
        lines = open(tmp_path / "ptl" / f"pol={p}_dev=0.res").read().splitlines()
        assert lines[:3] == [f"polId= {p}", f"nTime= {len(traj)}", f"len= {N}"]
        for (start, bonds), line in zip(traj, lines[3:]):
            t, u, v, s = line.split()
            assert [int(t), int(u), int(v)] == list(start[p])
            assert np.array_equal(np.array([int(c, 16) for c in s], dtype=np.uint8), bonds[p])
