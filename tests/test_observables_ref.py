"""The observables oracle (oracle/observables.py) against the reference's own
statistics program.

tests/golden/lowm_L16_N50_s3.json holds what the reference's create_ptl and
lowm_modes (analysis/, built from source by tests/golden/make_golden.py)
write for the reference efpol's own L=16, N=50 trajectory (the
efpol_L16_N50_s3_t*.res.gz fixtures, dumps every 10 steps): the mean radius
of gyration squared and the stored-length ratio per dump
(ComputeGyration / ComputeSL, analysis/mode_compute.c:145-203, written by
analysis/mode_io.c:269,500) and the centre-of-mass mean-square displacement
per lag (AddCMS, mode_compute.c:548-569; on the first pass over a sample,
which writes cmsdif_raw.dat, the reference has no drift record yet and
removes no drift, mode_init.c:389).  The restatement must give the same
numbers from the same files, to the printed precision of the reference's
output (7 significant digits).
"""
import gzip
import json
import os

import numpy as np

import observables as obs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 2e-6


def series():
    out = []
    for t in range(0, 101, 10):
        with gzip.open(os.path.join(GOLD, f"efpol_L16_N50_s3_t{t}.res.gz"), "rt") as f:
            L, start, bonds = obs.parse_tuv(f.read())
        out.append((t, start.astype(np.int64), bonds))
    return L, out


def test_rg2_and_stored_length_per_dump_match_lowm_modes():
    ref = json.load(open(os.path.join(GOLD, "lowm_L16_N50_s3.json")))
    _, ser = series()
    assert [r[0] for r in ref["rgyr_time"]] == [t for t, _, _ in ser]
    for (t, start, bonds), (_, rg_ref), (_, sl_ref) in zip(ser, ref["rgyr_time"], ref["slrat"]):
        rg2, _, sl = obs.chain_stats(start, bonds)
        assert np.isclose(rg2.mean(), rg_ref, rtol=RTOL, atol=1e-9), f"Rg^2 at t={t}"
        assert np.isclose(sl.mean(), sl_ref, rtol=RTOL, atol=1e-9), f"stored-length ratio at t={t}"


def test_cms_msd_matches_lowm_modes():
    ref = json.load(open(os.path.join(GOLD, "lowm_L16_N50_s3.json")))
    L, ser = series()
    cms = obs.unwrap_series(np.array([obs.cms_tuv(s, b) for _, s, b in ser]), L)
    lags = [int(round(r[0] / 10)) for r in ref["cmsdif_raw"]]
    msd = obs.cms_msd(cms, lags, drift=False)
    for lag, m, (_, m_ref) in zip(lags, msd, ref["cmsdif_raw"]):
        assert np.isclose(m, m_ref, rtol=RTOL, atol=1e-9), f"CMS MSD at lag {10 * lag}: {m} vs {m_ref}"
