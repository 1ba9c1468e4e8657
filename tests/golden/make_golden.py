"""Regenerate the golden fixtures in this directory from the REFERENCE itself.

Run in a checkout where the reference sources are available:

    python tests/golden/make_golden.py [--ref <reference checkout>]

(--ref defaults to the environment variable ELP_REFERENCE.)

It compiles the reference's efpol from its own sources (oracle/Makefile target
``ref``; outputs only under oracle/_ref/), then records

* ``table_<model>.npz``  -- the reference's LookupTables for sl_equal,
  sl_double and sl_quad (cpupol/efpol_init.c:314-424), via oracle/ref_table_dump.c;
* ``efpol_L32_N100_s1_t{0,100,200}.res.gz`` -- the reference's own TUV dumps
  for the plain ring melt L=32, N=100, density 1.2, seed 1;
* ``efpol_L16_N50_s3_t{0..100}.res.gz`` -- a short reference trajectory, one
  dump every 10 steps (pins the oracle's restatement step for step);
* ``ptl_L16_N50_s3.json.gz`` -- the per-ring time series files that the
  reference's create_ptl (analysis/create_ptl.c, built into oracle/_ref)
  writes for that trajectory: {file name: content};
* ``efpol_dbl_s5_t{1,100}_{in,out}.res.gz`` -- hierarchical doubling: the
  reference efpol run with DBLSTEP=1 (final L=32, N=400; first level L=16,
  N=50) for 1 and for 100 steps; ``in`` is its last dump of the first level,
  ``out`` its first dump of the doubled level (DoubleLattice,
  cpupol/efpol_init.c:114-207).  After one step many rings still sit on two
  sites, which exercises the rebuilt-ring branch;
* ``scaleup_<input>.res.gz`` -- the reference's analysis/scaleup.c output
  for three of the TUV files above (compact t=0 rings and relaxed melts);
  ``xyz_efpol_L16_N50_s3_t100_p{0,3,97}.txt.gz`` -- its analysis/tuv2xyz.c
  export of three rings; ``pov_efpol_L16_N50_s3_t100_p3.pov.gz`` -- its
  analysis/tuv2pov.c scene of one ring, and ``pov_sha256.json`` the SHA-256
  of its whole-melt scenes (rings and linear chains);
* ``efpol_lin_*`` -- the same for linear chains (the reference built with
  POL_TYPE=POL_LIN as efpol_lin): ``efpol_lin_L32_N100_s1_t{0,100,200}``,
  ``efpol_lin_L16_N50_s3_t{0..100}`` and ``efpol_lin_stats_L16_N50.json`` /
  ``efpol_lin_stats_L32_N100.json``;
* ``efpol_stats_L16_N50.json`` / ``efpol_stats_L32_N100.json`` -- ensemble
  statistics of reference efpol runs (16 and 8 distinct seeds) computed with
  oracle/observables.py: Rg^2, stored-length fraction, run-length histogram and
  centre-of-mass MSD, with per-seed values for error bars.

Nothing at test time reads the reference; the tests read these files only.
"""
from __future__ import annotations

import argparse
import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import observables as obs  # noqa: E402

MODELS = {"sl_equal": 1, "sl_double": 2, "sl_quad": 4}
STAT_LAGS = [1, 2, 5, 10, 20, 50]


def run_efpol(ref_bin, seed, L, N, tmax, interval, tmpdir):
    out = os.path.join(tmpdir, f"run_{L}_{N}_{seed}")
    subprocess.run([ref_bin, str(seed), out, "1.2", str(tmax), str(interval), str(N), "0", str(L), "sl_equal"],
                   check=True, stdout=subprocess.DEVNULL)
    return os.path.join(out, f"N_{N}")


def stats_of_run(d, tmax, interval, L, therm):
    rg, sl, hist, cms = [], [], None, []
    for t in range(0, tmax + 1, interval):
        with open(os.path.join(d, f"t={t}_dev=0.res")) as f:
            _, start, bonds = obs.parse_tuv(f.read())
        r, _, s = obs.chain_stats(start, bonds)
        cms.append(obs.cms_tuv(start, bonds))
        if t >= therm:
            rg.append(r.mean())
            sl.append(s.mean())
            h = obs.run_length_hist(bonds)
            hist = h if hist is None else hist + h
    cms_t = obs.unwrap_series(np.array(cms), L)[therm // interval:]
    msd = obs.cms_msd(cms_t, STAT_LAGS)
    return float(np.mean(rg)), float(np.mean(sl)), (hist / hist.sum()).tolist(), msd.tolist()


def make_ptl(refdir, efpol, tmp):
    """The reference's create_ptl on the reference's own L=16 trajectory."""
    d = run_efpol(efpol, 3, 16, 50, 100, 10, os.path.join(tmp, "ptl_run"))
    subprocess.run([os.path.join(refdir, "create_ptl"), d], check=True, stdout=subprocess.DEVNULL)
    files = {}
    for name in sorted(os.listdir(os.path.join(d, "ptl"))):
        with open(os.path.join(d, "ptl", name)) as f:
            files[name] = f.read()
    with gzip.GzipFile(os.path.join(HERE, "ptl_L16_N50_s3.json.gz"), "wb", mtime=0) as g:
        g.write(json.dumps(files, sort_keys=True).encode())


def make_double(efpol, tmp):
    """Reference runs with one doubling step: last dump of level 0, first of level 1."""
    for tmax in (1, 100):
        out = os.path.join(tmp, f"dbl_{tmax}")
        subprocess.run([efpol, "5", out, "1.2", str(tmax), str(tmax), "400", "1", "32", "sl_equal"], check=True,
                       stdout=subprocess.DEVNULL)
        for src, name in ((os.path.join(out, "N_50", f"t={tmax}_dev=0.res"), f"efpol_dbl_s5_t{tmax}_in.res.gz"),
                          (os.path.join(out, "N_400", "t=0_dev=0.res"), f"efpol_dbl_s5_t{tmax}_out.res.gz")):
            with open(src, "rb") as f, gzip.GzipFile(os.path.join(HERE, name), "wb", mtime=0) as g:
                g.write(f.read())


def make_export(refdir, tmp):
    """The reference's scaleup and tuv2xyz on committed reference TUV files."""
    for name in ("efpol_L16_N50_s3_t100", "efpol_L32_N100_s1_t0", "efpol_L32_N100_s1_t200"):
        src = os.path.join(tmp, name + ".res")
        with gzip.open(os.path.join(HERE, name + ".res.gz"), "rb") as f, open(src, "wb") as g:
            g.write(f.read())
        dst = os.path.join(tmp, "scaleup_" + name + ".res")
        subprocess.run([os.path.join(refdir, "scaleup"), src, dst], check=True, stdout=subprocess.DEVNULL)
        with open(dst, "rb") as f, gzip.GzipFile(os.path.join(HERE, "scaleup_" + name + ".res.gz"), "wb",
                                                  mtime=0) as g:
            g.write(f.read())
    src = os.path.join(tmp, "efpol_L16_N50_s3_t100.res")
    for pid in (0, 3, 97):
        dst = os.path.join(tmp, f"xyz_{pid}.txt")
        subprocess.run([os.path.join(refdir, "tuv2xyz"), src, dst, str(pid)], check=True, stdout=subprocess.DEVNULL)
        with open(dst, "rb") as f, gzip.GzipFile(
                os.path.join(HERE, f"xyz_efpol_L16_N50_s3_t100_p{pid}.txt.gz"), "wb", mtime=0) as g:
            g.write(f.read())


def make_pov(refdir, tmp):
    """The reference's tuv2pov on committed reference TUV files: one chain's
    scene in full, and the SHA-256 of whole-melt scenes (megabytes of text)."""
    hashes = {}
    for name, pids in (("efpol_L16_N50_s3_t100", (3, -1)), ("efpol_lin_L32_N100_s1_t200", (0, -1)),
                       ("efpol_L32_N100_s1_t0", (-1,))):
        src = os.path.join(tmp, name + ".res")
        with gzip.open(os.path.join(HERE, name + ".res.gz"), "rb") as f, open(src, "wb") as g:
            g.write(f.read())
        for pid in pids:
            dst = os.path.join(tmp, f"pov_{name}_{pid}.pov")
            args = [os.path.join(refdir, "tuv2pov"), src, dst] + ([str(pid)] if pid >= 0 else [])
            subprocess.run(args, check=True, stdout=subprocess.DEVNULL)
            with open(dst, "rb") as f:
                data = f.read()
            hashes[f"{name}/{pid}"] = hashlib.sha256(data).hexdigest()
            if pid >= 0 and name.startswith("efpol_L16"):
                with gzip.GzipFile(os.path.join(HERE, f"pov_{name}_p{pid}.pov.gz"), "wb", mtime=0) as g:
                    g.write(data)
    with open(os.path.join(HERE, "pov_sha256.json"), "w") as f:
        json.dump(hashes, f, indent=1, sort_keys=True)


def make_linear(refdir, tmp):
    """efpol_lin: initial melt, short trajectories and ensemble statistics."""
    lin = os.path.join(refdir, "efpol_lin")
    d = run_efpol(lin, 1, 32, 100, 200, 100, os.path.join(tmp, "lin"))
    for t in (0, 100, 200):
        with open(os.path.join(d, f"t={t}_dev=0.res"), "rb") as f, \
                gzip.GzipFile(os.path.join(HERE, f"efpol_lin_L32_N100_s1_t{t}.res.gz"), "wb", mtime=0) as g:
            g.write(f.read())
    d = run_efpol(lin, 3, 16, 50, 100, 10, os.path.join(tmp, "lin"))
    for t in range(0, 101, 10):
        with open(os.path.join(d, f"t={t}_dev=0.res"), "rb") as f, \
                gzip.GzipFile(os.path.join(HERE, f"efpol_lin_L16_N50_s3_t{t}.res.gz"), "wb", mtime=0) as g:
            g.write(f.read())
    # L=32, N=100 linear chains unfold from the collapsed initial melt for
    # ~40000 steps (Rg^2 still rises through 10^4 steps), so their ensemble is
    # compared at equilibrium: 10^5 steps, averages after step 40000
    write_stats(lin, "efpol_lin", "reference efpol_lin (cpupol, POL_LIN, sl_equal), built from source",
                [(16, 50, 20000, 100, 2000, range(301, 333, 2)), (32, 100, 100000, 1000, 40000, range(401, 417, 2))],
                os.path.join(tmp, "lin_stats"))


def write_stats(binary, prefix, engine, cases, tmp, workers=1):
    from concurrent.futures import ThreadPoolExecutor

    for (L, N, tmax, interval, therm, seeds) in cases:
        def one(s):
            d = run_efpol(binary, s, L, N, tmax, interval, tmp)
            rg, sl, hist, msd = stats_of_run(d, tmax, interval, L, therm)
            shutil.rmtree(os.path.dirname(d))
            return {"seed": s, "rg2": rg, "sl_frac": sl, "run_hist": hist, "msd": msd}

        with ThreadPoolExecutor(max_workers=workers) as ex:
            per_seed = list(ex.map(one, seeds))
        out = {"engine": engine, "L": L, "N": N, "density": 1.2, "steps": tmax, "interval": interval, "therm": therm,
               "msd_lags_intervals": STAT_LAGS, "per_seed": per_seed}
        with open(os.path.join(HERE, f"{prefix}_stats_L{L}_N{N}.json"), "w") as f:
            json.dump(out, f, indent=1)


def make_lowm(refdir, tmp):
    """The reference's own statistics program on the reference's own
    trajectory: create_ptl then lowm_modes on efpol's L=16, N=50 dumps
    (t = 0..100, every 10; the efpol_L16_N50_s3_t*.res.gz fixtures).  Keeps
    rgyr_time.dat (mean Rg^2 per dump), slrat.dat (stored-length ratio per
    dump) and cmsdif_raw.dat (centre-of-mass MSD per lag) as
    lowm_L16_N50_s3.json; oracle/observables.py is checked against them."""
    d = os.path.join(tmp, "lowm")
    os.makedirs(d)
    for t in range(0, 101, 10):
        with gzip.open(os.path.join(HERE, f"efpol_L16_N50_s3_t{t}.res.gz"), "rb") as f, \
                open(os.path.join(d, f"t={t}_dev=0.res"), "wb") as g:
            g.write(f.read())
    with open(os.path.join(d, "simulation_settings.txt"), "w") as f:
        f.write("Start_seed = 3\nLength = 50\nPolytype = ring\nDensity = 1.200000\nLatsize = 16\n"
                "Start_polysize = 50\nDouble_step = 0\nInterval = 10\nExecutable = efpol\n"
                "Polymodel = sl_equal\nEquilibrated = 1\n")
    subprocess.run([os.path.join(refdir, "create_ptl"), d], check=True, stdout=subprocess.DEVNULL)
    subprocess.run([os.path.join(refdir, "lowm_modes"), d], check=True, stdout=subprocess.DEVNULL)

    def table(name):
        with open(os.path.join(d, name)) as f:
            return [[float(x) for x in ln.split()] for ln in f if ln.strip()]

    out = {"source": "reference create_ptl + lowm_modes (analysis/), built from source, on efpol_L16_N50_s3 dumps",
           "rgyr_time": table("rgyr_time.dat"), "slrat": table("slrat.dat"), "cmsdif_raw": table("cmsdif_raw.dat")}
    with open(os.path.join(HERE, "lowm_L16_N50_s3.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_tiled_stats(efpol, tmp):
    """An L=64 ensemble, the box the GPU runs in tiles (32^3 or 32x16x16):
    efpol rounds L to a power of two, so 64 is the largest box it runs in
    minutes.  Averages from step 15000 on, where the stored length and Rg^2
    have stopped drifting, so that statics are compared at equilibrium and
    the MSD ratio measures the clock alone.  Compared with tiled GPU runs in
    tests/test_gpu_stats.py."""
    write_stats(efpol, "efpol", "reference efpol_ring (cpupol, sl_equal), built from source",
                [(64, 100, 50000, 500, 15000, range(601, 617, 2))], tmp, workers=os.cpu_count() or 1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("ELP_REFERENCE"),
                    help="reference checkout (default: $ELP_REFERENCE)")
    ap.add_argument("--only", choices=["all", "ptl", "double", "export", "pov", "linear", "tiled", "lowm"],
                    default="all")
    args = ap.parse_args()
    if not args.ref:
        ap.error("name the reference checkout with --ref or ELP_REFERENCE")
    subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref", f"REF={args.ref}"], check=True,
                   stdout=subprocess.DEVNULL)
    refdir = os.path.join(REPO, "oracle", "_ref")
    efpol = os.path.join(refdir, "efpol_ring")
    tmp = tempfile.mkdtemp(prefix="elp_golden_")
    try:
        if args.only == "ptl":
            make_ptl(refdir, efpol, tmp)
            return
        if args.only == "double":
            make_double(efpol, tmp)
            return
        if args.only == "export":
            make_export(refdir, tmp)
            return
        if args.only == "pov":
            make_pov(refdir, tmp)
            return
        if args.only == "linear":
            make_linear(refdir, tmp)
            return
        if args.only == "tiled":
            make_tiled_stats(efpol, tmp)
            return
        if args.only == "lowm":
            make_lowm(refdir, tmp)
            return
        for name, code in MODELS.items():
            raw = os.path.join(tmp, f"tab_{name}.bin")
            subprocess.run([os.path.join(refdir, "ref_table_dump_ring"), str(code), "5", raw], check=True)
            a = np.fromfile(raw, dtype=np.uint32)
            np.savez_compressed(os.path.join(HERE, f"table_{name}.npz"), trans=a[:4096],
                                add_occ=a[4096:8192].astype(np.int32), rem_occ=a[8192:].astype(np.int32))

        d = run_efpol(efpol, 1, 32, 100, 200, 100, tmp)
        for t in (0, 100, 200):
            with open(os.path.join(d, f"t={t}_dev=0.res"), "rb") as f, \
                    gzip.GzipFile(os.path.join(HERE, f"efpol_L32_N100_s1_t{t}.res.gz"), "wb", mtime=0) as g:
                g.write(f.read())

        d = run_efpol(efpol, 3, 16, 50, 100, 10, tmp)
        for t in range(0, 101, 10):
            with open(os.path.join(d, f"t={t}_dev=0.res"), "rb") as f, \
                    gzip.GzipFile(os.path.join(HERE, f"efpol_L16_N50_s3_t{t}.res.gz"), "wb", mtime=0) as g:
                g.write(f.read())
        make_ptl(refdir, efpol, tmp)
        make_double(efpol, tmp)
        make_export(refdir, tmp)
        make_pov(refdir, tmp)
        make_linear(refdir, tmp)
        make_tiled_stats(efpol, tmp)
        make_lowm(refdir, tmp)

        # efpol's seeding drops bit 0 of every Tausworthe word (util/rng.h:13-20,
        # 26-31), so seeds 2k and 2k+1 give the same run: use odd seeds only.
        for (L, N, tmax, interval, therm, seeds) in [(16, 50, 20000, 100, 2000, range(101, 133, 2)),
                                                      (32, 100, 10000, 100, 3000, range(201, 217, 2))]:
            per_seed = []
            for s in seeds:
                d = run_efpol(efpol, s, L, N, tmax, interval, tmp)
                rg, sl, hist, msd = stats_of_run(d, tmax, interval, L, therm)
                per_seed.append({"seed": s, "rg2": rg, "sl_frac": sl, "run_hist": hist, "msd": msd})
                shutil.rmtree(os.path.dirname(d))
            out = {"engine": "reference efpol_ring (cpupol, sl_equal), built from source",
                   "L": L, "N": N, "density": 1.2, "steps": tmax, "interval": interval, "therm": therm,
                   "msd_lags_intervals": STAT_LAGS, "per_seed": per_seed}
            with open(os.path.join(HERE, f"efpol_stats_L{L}_N{N}.json"), "w") as f:
                json.dump(out, f, indent=1)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
