"""Ensemble statistics of the GPU engine against the reference's CPU efpol.

tests/golden/efpol_stats_*.json and efpol_lin_stats_*.json hold per-seed
statistics of reference efpol_ring and efpol_lin runs (built from the
reference sources, tests/golden/make_golden.py).  The
GPU runs the same melts (same L, N, density, initial state, step count and
dump interval) with other seeds -- its parallel schedule cannot reproduce
efpol's random stream -- and the ensemble means must agree within the
combined standard error of the two seed ensembles:

    |mean_gpu - mean_ref| <= Z * sqrt(se_gpu^2 + se_ref^2),   Z = 4

for the radius of gyration squared, the stored-length fraction, each of the
first four bins of the run-length histogram, and the centre-of-mass MSD at
each lag.  Whole-box domains (L = 16, 32) have no tile walls, so the time
scale of the MSD is compared too.
"""
import json
import os

import numpy as np
import pytest

import elp
import observables as obs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
Z = 4.0


def gpu_ensemble(L, N, steps, interval, therm, lags, seeds, linear=0, **geom):
    b = elp.Batch([dict(L=L, N=N, seed=s, steps_per_launch=interval, linear=linear, **geom) for s in seeds])
    b.init_melts()
    nseed = len(seeds)
    cms = [[] for _ in range(nseed)]
    rg = [[] for _ in range(nseed)]
    sl = [[] for _ in range(nseed)]
    hist = [None] * nseed
    for t in range(0, steps + 1, interval):
        for j in range(nseed):
            start, bonds = b.fetch(j)
            start = start.astype(np.int64)
            r, _, s = obs.chain_stats(start, bonds)
            cms[j].append(obs.cms_tuv(start, bonds))
            if t >= therm:
                rg[j].append(r.mean())
                sl[j].append(s.mean())
                h = obs.run_length_hist(bonds)
                hist[j] = h if hist[j] is None else hist[j] + h
        if t < steps:
            b.run(interval)
    per = []
    for j in range(nseed):
        msd = obs.cms_msd(obs.unwrap_series(np.array(cms[j]), L)[therm // interval:], lags)
        per.append(dict(rg2=float(np.mean(rg[j])), sl_frac=float(np.mean(sl[j])),
                        run_hist=(hist[j] / hist[j].sum()).tolist(), msd=msd.tolist()))
        assert b.check(j) == 0
    return per


def compare(ref, gpu, key, idx=None):
    a = np.array([s[key] if idx is None else s[key][idx] for s in ref], dtype=float)
    g = np.array([s[key] if idx is None else s[key][idx] for s in gpu], dtype=float)
    se = np.sqrt(a.var(ddof=1) / len(a) + g.var(ddof=1) / len(g))
    return abs(a.mean() - g.mean()), se, a.mean(), g.mean()


@pytest.mark.parametrize("name,seeds,linear", [("efpol_stats_L16_N50.json", range(2001, 2009), 0),
                                               ("efpol_stats_L32_N100.json", range(3001, 3005), 0),
                                               ("efpol_lin_stats_L16_N50.json", range(4001, 4009), 1),
                                               ("efpol_lin_stats_L32_N100.json", range(5001, 5005), 1)])
def test_statistics_match_reference_efpol(name, seeds, linear):
    ref = json.load(open(os.path.join(GOLD, name)))
    gpu = gpu_ensemble(ref["L"], ref["N"], ref["steps"], ref["interval"], ref["therm"], ref["msd_lags_intervals"],
                       list(seeds), linear)
    rows = []
    checks = [("rg2", None), ("sl_frac", None)] + [("run_hist", i) for i in range(4)] + \
             [("msd", i) for i in range(len(ref["msd_lags_intervals"]))]
    for key, idx in checks:
        d, se, ma, mg = compare(ref["per_seed"], gpu, key, idx)
        rows.append((key, idx, ma, mg, d, se))
        assert d <= Z * se, f"{key}[{idx}]: efpol {ma:.5g} vs GPU {mg:.5g} differ by {d:.3g} > {Z} x {se:.3g}"


# Tiled geometries: L=64 melts run as 32^3 tiles (the default at L > 256
# and the largest specialised shape), 32x16x16 tiles (the default at
# L = 128 and 256) or 16x16x8 tiles (the smallest shape of the default list,
# on the generic kernel).  A move whose footprint crosses a tile wall is
# rejected, as gpupol's out-of-block moves are (gpupol2/ringpol3.cu:58-76);
# the walls move every step, so the equilibrium (Rg^2, stored length, run
# lengths) is efpol's, compared here over steps 15000-50000, while the clock
# runs slower: the GPU's centre-of-mass MSD after t steps is efpol's after
# f*t steps, f the time factor that elp_time_factor records for the shape
# (and the drop-in programs hand to the analysis through their Executable
# name).
TILED = [((32, 32, 32), range(7001, 7009)), ((32, 16, 16), range(7101, 7109)), ((16, 16, 8), range(7801, 7809))]


def msd_step_ratio(lags, ref_msd, msd):
    """Per lag, the factor f with msd(lag) = ref_msd(f * lag), ref_msd
    interpolated (and at the ends extrapolated) linearly in log-log."""
    x, y = np.log(lags), np.log(ref_msd)
    out = []
    for lx, v in zip(x, np.log(msd)):
        if v <= y[0]:
            X = x[0] + (v - y[0]) * (x[1] - x[0]) / (y[1] - y[0])
        elif v >= y[-1]:
            X = x[-1] + (v - y[-1]) * (x[-1] - x[-2]) / (y[-1] - y[-2])
        else:
            X = np.interp(v, y, x)
        out.append(np.exp(X - lx))
    return np.array(out)


@pytest.mark.parametrize("tile,seeds", TILED)
def test_tiled_statistics_match_reference_efpol(tile, seeds):
    ref = json.load(open(os.path.join(GOLD, "efpol_stats_L64_N100.json")))
    gpu = gpu_ensemble(ref["L"], ref["N"], ref["steps"], ref["interval"], ref["therm"], ref["msd_lags_intervals"],
                       list(seeds), periodic=0, tile=tile)
    for key, idx in [("rg2", None), ("sl_frac", None)] + [("run_hist", i) for i in range(4)]:
        d, se, ma, mg = compare(ref["per_seed"], gpu, key, idx)
        assert d <= Z * se, f"{tile} {key}[{idx}]: efpol {ma:.5g} vs GPU {mg:.5g} differ by {d:.3g} > {Z} x {se:.3g}"
    lags = np.array(ref["msd_lags_intervals"], dtype=float)
    ma = np.mean([s["msd"] for s in ref["per_seed"]], axis=0)
    per_seed = np.array([msd_step_ratio(lags, ma, s["msd"]) for s in gpu])
    f = per_seed.mean(axis=0)
    f_se = per_seed.std(axis=0, ddof=1) / np.sqrt(len(per_seed))
    rec = elp.time_factor(0, *tile)
    assert rec > 0
    # the recorded factor has three decimals: half a unit of the last one is slack
    assert np.all(np.abs(f - rec) <= Z * f_se + 0.0005), f"{tile}: step ratio per lag {np.round(f, 4)} vs {rec}"
