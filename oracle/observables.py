"""TEST INFRASTRUCTURE ONLY -- observables of ring melts, restated in numpy.

These follow the reference analysis code so that statistics computed from this
project's output and from the reference efpol's output are comparable:

* ``xyz`` from lattice (t, u, v): x = t+u-v, y = t-u, z = v, and lengths in
  units of 1/sqrt(2)  (cpupol/efpol_lib.c:71-93, analysis/mode_compute.c:191-217)
* radius of gyration squared per chain (ComputeGyration, mode_compute.c:191-203)
* centre of mass per chain (ComputeCMS, mode_compute.c:205-217)
* stored-length fraction per chain: share of monomers that sit on the same
  site as their successor (ComputeSL, mode_compute.c:145-153)
* centre-of-mass mean-square displacement (AddCMS, mode_compute.c:548-569):
  the reference removes the melt's mean drift using avg_pos.dat, which its
  first pass over a sample only writes (AddAvgPos, :244-252; mode_init.c:389),
  so the cmsdif_raw.dat of that pass holds the MSD without drift removal.
  Both forms are here (``drift``).  Pinned to the reference's lowm_modes
  output by tests/test_observables_ref.py.
* stored-length histogram: number of monomers per occupied site.  The
  reference has no such histogram; it is defined here from the same run
  lengths for both engines.
"""
from __future__ import annotations

import gzip
import re

import numpy as np

_UNIT = np.zeros((16, 3), dtype=np.int64)
for _b in range(16):
    _w = (_b >> 3) & 1
    _UNIT[_b] = ((_b & 1) - _w, ((_b >> 1) & 1) - _w, ((_b >> 2) & 1) - _w)

VALID = np.array([b not in (0, 3, 12, 15) for b in range(16)])


def parse_tuv(text: str):
    """Parse a TUV file (cpupol/efpol_io.c:50-77) -> (L, start[P,3], bonds[P,N])."""
    head = re.match(r"LT=\s*(\d+)\s+LU=\s*(\d+)\s+LV=\s*(\d+)\s+np=\s*(\d+)\s+maxPolLength=\s*(\d+)\s*", text)
    if not head:
        raise ValueError("not a TUV file")
    lt, lu, lv, npol, nmax = map(int, head.groups())
    body = text[head.end():].split()
    start = np.zeros((npol, 3), dtype=np.int64)
    bonds = np.zeros((npol, nmax), dtype=np.uint8)
    k = 0
    for p in range(npol):
        if body[k] != "len=":
            raise ValueError("bad chain header")
        n = int(body[k + 1])
        start[p] = (int(body[k + 2]), int(body[k + 3]), int(body[k + 4]))
        s = body[k + 5]
        if len(s) != n or n != nmax:
            raise ValueError("bad bond string")
        bonds[p] = np.frombuffer(bytes.fromhex("".join("0" + c for c in s)), dtype=np.uint8)
        k += 6
    return lt, start, bonds


def read_tuv(path: str):
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "rt") as f:
        return parse_tuv(f.read())


def format_tuv(L: int, start: np.ndarray, bonds: np.ndarray) -> str:
    """Byte-identical to the reference's WriteLatticeFile."""
    P, N = bonds.shape
    out = [f"LT= {L}\nLU= {L}\nLV= {L}\nnp= {P}\nmaxPolLength= {N}\n"]
    hexd = np.array(list("0123456789abcdef"))
    for p in range(P):
        t, u, v = (int(x) for x in start[p])
        out.append(f"len= {N}\n{t}  {u}  {v}\t" + "".join(hexd[bonds[p]]) + "\n")
    return "".join(out)


def unwrapped_tuv(start: np.ndarray, bonds: np.ndarray) -> np.ndarray:
    """Monomer positions (P, N, 3) obtained by walking the bonds from monomer 0."""
    steps = _UNIT[bonds.astype(np.int64)]                      # (P, N, 3)
    pos = np.concatenate([np.zeros_like(steps[:, :1]), np.cumsum(steps[:, :-1], axis=1)], axis=1)
    return pos + start[:, None, :]


def to_xyz(tuv: np.ndarray) -> np.ndarray:
    t, u, v = tuv[..., 0], tuv[..., 1], tuv[..., 2]
    return np.stack([t + u - v, t - u, v], axis=-1).astype(np.float64) / np.sqrt(2.0)


def is_linear(bonds: np.ndarray) -> bool:
    """Linear chains end in the marker bond 0xf (TUV character 'f')."""
    return bool(np.all(bonds[:, -1] == 0xF))


def chain_stats(start: np.ndarray, bonds: np.ndarray):
    """Per chain: Rg^2, centre of mass (xyz), stored-length fraction.  For
    linear chains the end marker is no bond: ComputeSL divides by N - 1
    (LoadPTL, analysis/mode_io.c:590-597, sets polSize = nMono - 1)."""
    xyz = to_xyz(unwrapped_tuv(start, bonds))
    cms = xyz.mean(axis=1)
    rg2 = ((xyz - cms[:, None, :]) ** 2).sum(axis=2).mean(axis=1)
    sl = (bonds[:, :-1] == 0).mean(axis=1) if is_linear(bonds) else (bonds == 0).mean(axis=1)
    return rg2, cms, sl


def run_length_hist(bonds: np.ndarray, nbins: int = 16) -> np.ndarray:
    """Histogram of monomers per occupied site (ring runs); last bin is overflow."""
    hist = np.zeros(nbins, dtype=np.int64)
    for b in bonds:
        nz = np.flatnonzero(b)
        # runs end at monomers with a non-zero bond; lengths are gaps between ends (cyclic)
        ends = np.concatenate([nz, nz[:1] + len(b)])
        lens = np.diff(ends)
        np.add.at(hist, np.minimum(lens, nbins) - 1, 1)
    return hist


def unwrap_series(cms_series: np.ndarray, L: int) -> np.ndarray:
    """Make centre-of-mass trajectories continuous across periodic images.

    Positions come from walking the bonds from monomer 0, whose stored
    coordinate is wrapped into the box; the chain shape itself is continuous,
    so only whole-box jumps of the start site need undoing.  ``cms_series`` is
    (T, P, 3) in lattice (t, u, v) units.
    """
    out = cms_series.copy()
    for i in range(1, out.shape[0]):
        d = out[i] - out[i - 1]
        out[i] -= L * np.round(d / L)
    return out


def cms_tuv(start: np.ndarray, bonds: np.ndarray) -> np.ndarray:
    return unwrapped_tuv(start, bonds).mean(axis=1)


def cms_msd(cms_t: np.ndarray, lags, drift: bool = True) -> np.ndarray:
    """Mean-square displacement of chain centres of mass (xyz units) at the
    given lags (in dump intervals), averaged over every time origin and
    chain; with ``drift`` the melt's mean displacement over the lag is
    removed first.  cms_t: (T, P, 3) in continuous lattice units."""
    xyz = to_xyz(cms_t)
    res = []
    for lag in lags:
        d = xyz[lag:] - xyz[:-lag] if lag > 0 else np.zeros_like(xyz)
        if drift:
            d = d - d.mean(axis=1, keepdims=True)
        res.append((d ** 2).sum(axis=2).mean())
    return np.array(res)
