"""Benchmark of the ELP ring-melt sweep: attempted monomer moves per second.

One bench step is one Monte Carlo time step (N*P attempted monomer moves, the
reference efpol's unit, cpupol/efpol_lib.c:123) of the workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl elp|reference]

Default workload: the single large ring melt L=128, N=1000, density 1.2
(2517 rings), seed 7, initialised like the reference's CreatePolymers and
then RELAXED for --relax steps on the GPU (untimed) before the warm-up and
the timed steps, so that the timed steps see the dense melt a production run
of 10^5 steps spends its time in, not the collapsed initial melt (synthetic:
no dataset exists for this path).  The melt runs --spl steps per kernel
launch (a cooperative launch whose CTAs meet at a grid barrier between
steps; the same bits as one step per launch).  The lattice
(8 MB) is smaller than L2, so L2 is flushed before every timed launch (a
256 MB write outside the timed events).  After the timed launches the same
melt runs --one-step-launches launches of one step each
(`one_step_per_launch` in the line: one kernel per MC step).

Extra legs (one GPU only): the L=256, N=5000 melt (roofline configuration,
relaxed --l256-relax steps), the reference CPU efpol timed on this host from
the same relaxed melt (read by the reference's own ReadLatticeFile), the
reference's own GPU engine gpupol3 on this GPU, the end-to-end path through
the C ABI with host buffers, the 512-replica ensemble (batched vs plain,
from relaxed members) and the served stream.

--gpus N runs N independent replicas (one process per GPU, seeds offset by
rank); there is no data-path collective -- replicas only.

--impl reference times the reference's own efpol (compiled from its sources
into oracle/_ref) on all host cores, on the same relaxed melt: the relaxed
configuration is produced on the GPU by this engine (untimed, as a run's
earlier dump would be) and read by the reference from its TUV file.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "mc-polymer-simulation_b200", "python"))

METRIC = "attempted monomer moves/s"
UNIT = "moves/s"
WORKLOADS = {
    "L128": dict(L=128, N=1000, seed=7, density=1.2),
    "L256": dict(L=256, N=5000, seed=11, density=1.2),
    "L32": dict(L=32, N=100, seed=1, density=1.2),
}


def npol(w):
    return max(1, int(w["density"] * w["L"] ** 3 / w["N"] + 0.5))


def algo_bytes(w):
    """Algorithmic bytes of one sweep: every uint32 site word read and written
    once, every int8 bond read and written once: 8*S + 2*M."""
    return 8 * w["L"] ** 3 + 2 * w["N"] * npol(w)


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def issue_ceiling(name, spl, ms_per_step, sm_mhz, sms_busy):
    """The ceiling that binds this integer kernel: warp-instruction issue
    (4 per cycle per SM).  Instructions per launch come from the committed ncu
    capture of the same launch shape; frac is the issue rate achieved over the
    step against the SMs that hold work at the sampled clock."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(p) as f:
            inst = json.load(f).get(f"inst/{name}/spl{spl}")
    except Exception:
        inst = None
    if not inst or not sm_mhz:
        return None
    per_step = inst / spl
    achieved = per_step / (ms_per_step / 1e3)
    peak = 4.0 * sms_busy * sm_mhz * 1e6
    return {"bound": "issue", "warp_inst_per_step": per_step, "achieved": achieved, "peak": peak,
            "unit": "warp inst/s", "frac": achieved / peak, "sms_with_work": sms_busy, "sm_mhz": sm_mhz}


def profile_traffic(name, spl):
    """DRAM bytes per sweep launch of `spl` steps from the committed ncu
    summary, if one was captured for that launch shape."""
    p = os.path.join(REPO, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(f"{name}/spl{spl}")
    except Exception:
        return None


class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def _wait_for(self, n, timeout):
        t0 = time.perf_counter()
        while len(self.lines) < n and time.perf_counter() - t0 < timeout:
            time.sleep(0.005)

    def __enter__(self):
        # samples every 50 ms; the timed region starts once the sampler has
        # answered, and ends after one more sample, so short timed regions
        # are bracketed by samples
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self._wait_for(1, 5.0)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self._wait_for(len(self.lines) + 1, 1.0)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def ref_binary():
    """The reference efpol's bench driver (oracle/_ref, compiled from the
    reference sources) or, where the reference was not built, the oracle's
    restatement of it."""
    ref = os.path.join(REPO, "oracle", "_ref", "ref_bench")
    if os.path.exists(ref):
        return ref, "reference"
    port = os.path.join(REPO, "oracle", "efpol_port")
    if not os.path.exists(port):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle")], check=True, stdout=subprocess.DEVNULL)
    return port, "port"


def cpu_baseline(w, steps, threads=1, tuv=None, start_desc="CreatePolymers initial melt"):
    """Reference efpol timed on this host: `threads` independent processes,
    each `steps` MC steps of the melt, from the TUV file `tuv` (read by the
    reference's ReadLatticeFile) or from CreatePolymers."""
    ref, kind = ref_binary()
    if tuv and kind != "reference":
        tuv, start_desc = None, "CreatePolymers initial melt (the restatement reads no TUV)"
    t0 = time.perf_counter()
    procs = [subprocess.Popen([ref, str(w["L"]), str(w["N"]), str(w["density"]), str(w["seed"] + i), str(steps)]
                              + ([tuv] if tuv else []), stdout=subprocess.PIPE, text=True) for i in range(threads)]
    outs = []
    for p in procs:
        o = p.communicate()[0]
        if p.returncode != 0:
            raise RuntimeError(f"{ref} exited {p.returncode}")
        outs.append(json.loads(o.strip().splitlines()[-1]))
    wall = time.perf_counter() - t0
    moves = sum(o["moves"] for o in outs)
    # processes run concurrently; each times its own DoMCStep window
    rate = moves / max(o["seconds"] for o in outs)
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{steps} MC steps of L={w['L']} N={w['N']} per process from the {start_desc}, "
                      f"{threads} process(es), {moves:.3g} attempted moves in {wall:.2f} s"}


def occupied_fraction(m):
    import numpy as np
    w, _ = m.state()
    return float(np.count_nonzero(w)) / w.size


def relaxed_melt(elp, w, seed, dev, spl, relax):
    """The workload's melt: CreatePolymers' initial melt, then `relax` steps
    on the GPU (untimed)."""
    m = elp.Melt(L=w["L"], N=w["N"], seed=seed, device=dev, steps_per_launch=spl)
    m.init_melt()
    if relax > 0:
        m.run(relax)
    m.sync()
    return m


def common_config(w, relax):
    """The `config` both arms print (identical keys and values)."""
    return {"workload": f"ring melt L={w['L']} N={w['N']} density={w['density']} P={npol(w)} seed={w['seed']}, "
                        f"relaxed: {relax} steps from CreatePolymers",
            "L": w["L"], "N": w["N"], "P": npol(w), "density": w["density"], "seed": w["seed"],
            "sites": w["L"] ** 3, "monomers": w["N"] * npol(w), "relax_steps": relax,
            "l2": "GPU arm: flushed before every timed launch (256 MB write on the melt's stream, queued before the "
                  "start event), the lattice staying in L2 inside a launch; CPU arm: host caches, no flush"}


def replica_seed(w, rank):
    """Replica r of a workload runs the same melt with seed + r."""
    return w["seed"] + rank


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """Max of a host-side number over all ranks (the job's time is its
    slowest replica's).  Replicas exchange nothing else; the reduction runs
    on gloo over host memory."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_elp(args, rank, world):
    import tempfile

    import torch
    import elp

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    w = WORKLOADS[args.workload]
    M = w["N"] * npol(w)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")

    spl = max(1, args.spl)
    m = relaxed_melt(elp, w, replica_seed(w, rank), dev, spl, args.relax)
    occ = occupied_fraction(m)
    m.run(args.warmup)
    m.sync()
    info = m.info()
    a0 = m.accepted()

    barrier(world)
    with ClockSampler(dev) as clk:
        times = timed_steps(m, torch, flush, dev, args.steps, spl)
    # this library's kernels in the timed region: the sweep launches, and the
    # step-counter update of each CUDA-graph replay (the library counts them)
    kernels = m.info().kernels - info.kernels
    total_ms = max_over_ranks(sum(times), world)
    barrier(world)
    accepted = m.accepted() - a0
    value = world * args.steps * M / (total_ms / 1e3)
    ms_per_step = total_ms / args.steps
    assert m.check() == 0, "integrity check failed after the timed run"
    extras = rank == 0 and world == 1 and not args.no_extras
    # the same melt with one kernel launch per MC step (every launch flushed
    # from L2 first), beside the multi-step launches of the headline
    one = None
    if args.one_step_launches > 0 and extras:
        ot = timed_steps(m, torch, flush, dev, args.one_step_launches, 1)
        one_ms = sum(ot) / len(ot)
        one = {"ms_per_step": one_ms, "value": M / (one_ms / 1e3), "unit": UNIT, "launches": len(ot),
               "l2": "flushed before every launch"}
        assert m.check() == 0, "integrity check failed after the one-step launches"

    peak, peak_kind = measured_peak()
    achieved = algo_bytes(w) / (ms_per_step / 1e3) / 1e9
    tr = profile_traffic(args.workload, spl)
    cfg = common_config(w, args.relax)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (reference CreatePolymers initial melt, relaxed on "
                                                      "the GPU before timing)",
        "config": dict(cfg, parallelism=f"replicas x{world}"),
        "kernel": {"steps_per_launch": spl,
                   "geometry": {"periodic": info.periodic, "tile": list(info.tile), "ncol": info.ncol,
                                "domains": info.domains, "threads": info.threads}},
        "state": {"occupied_site_fraction": occ,
                  "accepted_moves_per_s": accepted / (total_ms / 1e3) if world == 1 else None,
                  "acceptance": accepted / (args.steps * M)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": spl * algo_bytes(w),
                     "traffic": tr},
        "gpu_launches": kernels,
        "timed_launches": len(times),
    }
    if one:
        line["one_step_per_launch"] = one
    clk_s = clk.summary()
    if clk_s:
        line["clocks"] = clk_s
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    ic = issue_ceiling(args.workload, spl, ms_per_step, (clk_s or {}).get("sm_mhz"), min(sms, info.domains))
    if ic:
        line["issue_roofline"] = ic

    if extras:
        with tempfile.TemporaryDirectory(prefix="elp_bench_") as tmp:
            tuv = os.path.join(tmp, f"relaxed_L{w['L']}.res")
            m.write_tuv(tuv)
            line["cpu_baseline"] = cpu_baseline(w, args.cpu_steps, 1, tuv, f"relaxed melt after {m.step} steps")
        line["e2e"] = e2e_leg(elp, w, dev, args)
        if not args.no_gpu_reference:
            line["gpu_reference"] = gpu_reference_leg(w, ms_per_step, args.gp3_interval)
        if args.workload != "L256" and not args.no_l256:
            line["L256"] = l256_leg(elp, torch, dev, flush, args, (clk_s or {}).get("sm_mhz"))
        if not args.no_batched:
            line["ensemble"] = batched_leg(elp, dev, args)
        if not args.no_served:
            line["served"] = served_leg(elp, dev, args)
    return line


def e2e_leg(elp, w, dev, args):
    """Through the C ABI with host buffers: per bench step, load the rings from
    pinned host memory (H2D), run one dump interval, fetch them back (D2H).
    Starts from the relaxed melt."""
    import torch

    interval = args.e2e_interval
    P, N = npol(w), w["N"]
    m = relaxed_melt(elp, w, w["seed"], dev, max(1, args.spl), args.relax)
    m.run(args.warmup)
    start_t = torch.empty((P, 3), dtype=torch.int32).pin_memory()
    bonds_t = torch.empty((P, N), dtype=torch.uint8).pin_memory()
    start, bonds = start_t.numpy(), bonds_t.numpy()
    s0, b0 = m.fetch()
    start[:], bonds[:] = s0, b0
    reps = max(2, args.e2e_reps)
    step = m.step

    def cycle(step):
        m.load_chains(start, bonds, step)
        m.run(interval)
        m.fetch(start, bonds)          # rings back into the same pinned buffers

    cycle(step)                        # warm-up (first-call set-up), not timed
    step += interval
    t0 = time.perf_counter()
    for _ in range(reps):
        cycle(step)
        step += interval
    dt = time.perf_counter() - t0
    # where a cycle's time goes: a few more cycles (not in the number above),
    # with a synchronisation after elp_run so that each part is closed
    parts = {"load_chains": [], "run": [], "fetch_chains": []}
    for _ in range(5):
        t1 = time.perf_counter()
        m.load_chains(start, bonds, step)
        t2 = time.perf_counter()
        m.run(interval)
        m.sync()
        t3 = time.perf_counter()
        m.fetch(start, bonds)
        t4 = time.perf_counter()
        step += interval
        parts["load_chains"].append(t2 - t1)
        parts["run"].append(t3 - t2)
        parts["fetch_chains"].append(t4 - t3)
    assert m.check() == 0
    return {"value": reps * interval * N * P / dt, "unit": UNIT,
            "h2d_bytes_per_step": 12 * P + N * P, "d2h_bytes_per_step": 12 * P + N * P,
            "steps_per_call": interval, "calls_timed": reps,
            "bytes_per": f"call cycle (load, {interval} MC steps, fetch): the chains go in and come back once per cycle",
            "ms_per_call": 1e3 * dt / reps,
            "parts_ms_median": {k: 1e3 * sorted(v)[len(v) // 2] for k, v in parts.items()},
            "path": "elp_load_chains(host) + elp_run(interval) + elp_fetch_chains(host), wall clock, from the "
                    f"melt relaxed {args.relax} steps"}


def timed_steps(m, torch, flush, dev, nsteps, spl=1):
    """nsteps MC steps in launches of spl steps.  Per launch: flush L2 (a
    256 MB write) on the melt's own stream, then the launch between CUDA
    events on that stream.  The flush is queued ahead of the start event, so
    the events see the sweep launch alone and the host's launch latency hides
    behind the flush.  Returns the time of each launch (ms)."""
    s = torch.cuda.ExternalStream(m.stream_ptr(), device=f"cuda:{dev}")
    torch.cuda.synchronize()
    times = []
    done = 0
    while done < nsteps:
        k = min(spl, nsteps - done)
        with torch.cuda.stream(s):
            flush.fill_(1.0)
        times.append(m.run_timed(k))
        done += k
    torch.cuda.synchronize()
    return times


def l256_leg(elp, torch, dev, flush, args, clock_mhz):
    w = WORKLOADS["L256"]
    M = w["N"] * npol(w)
    spl = max(1, args.l256_spl)
    m = relaxed_melt(elp, w, w["seed"], dev, spl, args.l256_relax)
    occ = occupied_fraction(m)
    m.run(3 * spl)
    m.sync()
    nsteps = max(3 * spl, args.steps // 2 // spl * spl)
    a0 = m.accepted()
    times = timed_steps(m, torch, flush, dev, nsteps, spl)
    acc = m.accepted() - a0
    ms = sum(times) / nsteps
    assert m.check() == 0
    peak, _ = measured_peak()
    achieved = algo_bytes(w) / (ms / 1e3) / 1e9
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    out = {"workload": f"ring melt L=256 N=5000 P=4027 seed=11, relaxed: {args.l256_relax} steps from "
                       f"CreatePolymers, {spl} steps per sweep launch",
           "value": M / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "steps": nsteps, "steps_per_launch": spl,
           "state": {"occupied_site_fraction": occ, "accepted_moves_per_s": acc / (sum(times) / 1e3),
                     "acceptance": acc / (nsteps * M)},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "algorithmic_bytes_per_launch": spl * algo_bytes(w),
                        "traffic": profile_traffic("L256", spl)}}
    ic = issue_ceiling("L256", spl, ms, clock_mhz, min(sms, m.info().domains))
    if ic:
        out["issue_roofline"] = ic
    return out


def gpu_reference_leg(w, ms_per_step, interval, timeout=900):
    """The reference's own GPU engine, gpupol3 (gpupol2/ with 4^3 cells and
    32^3 blocks), built from its unmodified sources for sm_100a
    (oracle/Makefile target _ref/gpupol3_cuda_ring: -gencode for sm_100a,
    the system host compiler), run on this GPU on the same box, ring length,
    density and seed, and timed by its own progress line: "MF/s" = lattice
    sites x steps per second (gpupol2/gpupol2.c:58), over intervals of
    `interval` steps that end with its synchronous dump
    (gpupol2/gpupol_cuda.cu:52-76).  Its move set is not efpol's (three move
    kinds on 1-byte site words, gpupol2/ringpol3.cu:92-219), so the
    comparison is per lattice site and step, the unit it reports; per step it
    makes 51 x 4 move attempts per 64-site cell (3.19 per site) against two
    anchor visits per site here."""
    exe = os.path.join(REPO, "oracle", "_ref", "gpupol3_cuda_ring")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/gpupol3_cuda_ring not built (set ELP_REFERENCE and make -C oracle ref)"}
    import re
    import tempfile
    L = w["L"]
    with tempfile.TemporaryDirectory(prefix="elp_gp3_") as tmp:
        cmd = [exe, str(w["N"]), str(2 * interval), str(w["seed"]), os.path.join(tmp, "run"), str(w["density"]), "0",
               str(interval), str(L), str(L), str(L)]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"gpupol3 did not finish {2 * interval} steps in {timeout} s"}
    rates = [float(x) for x in re.findall(r"at ([0-9.]+) MF/s", r.stdout.replace("\r", "\n"))]
    if r.returncode != 0 or not rates:
        return {"unavailable": f"gpupol3 exited {r.returncode}: {(r.stdout + r.stderr)[-300:]}"}
    ref = rates[-1] * 1e6                       # sites x steps / s, the last interval (the first pays start-up)
    ours = L ** 3 / (ms_per_step / 1e3)
    return {"engine": "reference gpupol3_cuda_ring (gpupol2/, LCELL=4), unmodified sources built for sm_100a",
            "workload": f"L={L} N={w['N']} density={w['density']} seed={w['seed']}, {2 * interval} steps, "
                        f"its own MF/s over the last interval of {interval} steps (synchronous dump included)",
            "mf_per_s": rates, "sites_steps_per_s": ref, "ours_sites_steps_per_s": ours, "ours_over_reference": ours / ref,
            "move_attempts_per_site_step": {"gpupol3": 51 * 4 / 64, "ours": 2.0}}


# ---- batched ensemble (512 replicas) ------------------------------------------
def _philox(ctr, key):
    """Philox4x32-10 (Salmon et al., SC'11); used only to draw the synthetic mix."""
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    M = 0xFFFFFFFF
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M, p1 & M, ((p0 >> 32) ^ c3 ^ k1) & M, p0 & M
        k0, k1 = (k0 + 0x9E3779B9) & M, (k1 + 0xBB67AE85) & M
    return c0, c1, c2, c3


def ensemble_mix(n=512, first_seed=1000, density=1.2):
    """Replica i: seed 1000+i; L uniform on {16,24,32,48,64}; N log-uniform on
    [50, 1000]; both drawn from Philox keyed by the replica's seed."""
    import math
    Ls = (16, 24, 32, 48, 64)
    out = []
    for i in range(n):
        seed = first_seed + i
        w = _philox((0, 0, 0, 0), (seed, 0xC0F4))
        L = Ls[(w[0] * len(Ls)) >> 32]
        u = w[1] / 2.0 ** 32
        N = int(round(math.exp(math.log(50) + u * (math.log(1000) - math.log(50)))))
        N = max(3, min(N, int(density * L ** 3 / 2)))
        out.append(dict(L=L, N=N, seed=seed, density=density))
    return out


def cpu_ensemble(mix, target_moves=1e8, max_procs=None, tuvs=None):
    """The reference efpol on the ensemble's members it can run (L a power of
    two: 16, 32, 64), one process per host core at once, each a bounded sample
    of about target_moves attempted moves; the aggregate is the sum of the
    processes' own rates (they run concurrently).  tuvs maps a member's seed
    to a TUV file of its relaxed state (read by the reference's
    ReadLatticeFile); members without one start from CreatePolymers."""
    ref, kind = ref_binary()
    members = [m for m in mix if m["L"] in (16, 32, 64)]
    nproc = min(len(members), max_procs or os.cpu_count() or 1)
    members = members[:nproc]
    procs = []
    relaxed = 0
    for m in members:
        M = m["N"] * max(1, int(m["density"] * m["L"] ** 3 / m["N"] + 0.5))
        steps = max(10, int(target_moves / M))
        tuv = (tuvs or {}).get(m["seed"]) if kind == "reference" else None
        relaxed += 1 if tuv else 0
        procs.append(subprocess.Popen([ref, str(m["L"]), str(m["N"]), str(m["density"]), str(m["seed"]), str(steps)]
                                      + ([tuv] if tuv else []), stdout=subprocess.PIPE, text=True))
    outs = [json.loads(p.communicate()[0].strip().splitlines()[-1]) for p in procs]
    rate = sum(o["moves"] / o["seconds"] for o in outs)
    return {"value": rate, "unit": UNIT, "cores": nproc, "kind": kind,
            "sample": f"the first {nproc} members with L in {{16,32,64}} (efpol rounds L up to a power of two, so "
                      f"L=24/48 do not run), about {target_moves:.0e} attempted moves each, one process per core, "
                      f"{relaxed} of them from the members' relaxed states"}


def batched_leg(elp, dev, args):
    import tempfile

    mix = ensemble_mix(args.replicas)
    tuned = {}
    for L in sorted({m["L"] for m in mix}):
        ms = [m for m in mix if m["L"] == L]
        sp, t = elp.autotune(copies=min(len(ms), 128), steps=10, device=dev, **dict(ms[0], steps_per_launch=100))
        tuned[L] = sp
    specs = []
    for m in mix:
        t = tuned[m["L"]]
        specs.append(dict(m, periodic=t["periodic"], tile=t["tile"], ncol=t["ncol"],
                          steps_per_launch=t["steps_per_launch"], device=dev))
    moves = sum(sp["N"] * max(1, int(sp["density"] * sp["L"] ** 3 / sp["N"] + 0.5)) for sp in specs)
    b = elp.Batch(specs, device=dev)
    b.init_melts()
    b.run(args.batch_relax)            # relax every member (untimed)
    b.sync()
    relaxed = [b.state(j) for j in range(len(specs))]
    step0 = args.batch_relax
    b.run(args.batch_warmup)
    b.sync()
    bms = b.run_timed(args.batch_steps)
    batched = moves * args.batch_steps / (bms / 1e3)
    # plain kernel, same mix, one replica at a time, from the same relaxed states
    pms, check_idx, same = 0.0, list(range(0, len(specs), max(1, len(specs) // 16))), True
    for j, sp in enumerate(specs):
        m = elp.Melt(**sp)
        m.set_state(relaxed[j][0], relaxed[j][1], step0)
        m.run(args.batch_warmup)
        pms += m.run_timed(args.batch_steps)
        if j in check_idx:
            wa, ra = b.state(j)
            wb, rb = m.state()
            same = same and bool((wa == wb).all() and (ra == rb).all())
        m.close()
    plain = moves * args.batch_steps / (pms / 1e3)
    occ = sum(int((r[0] != 0).sum()) for r in relaxed) / sum(r[0].size for r in relaxed)
    # the reference on its members, from their relaxed states
    with tempfile.TemporaryDirectory(prefix="elp_ens_") as tmp:
        tuvs = {}
        for j, sp in enumerate(specs):
            if sp["L"] in (16, 32, 64) and len(tuvs) < (os.cpu_count() or 1):
                mm = elp.Melt(**sp)
                mm.set_state(relaxed[j][0], relaxed[j][1], step0)
                path = os.path.join(tmp, f"m{sp['seed']}.res")
                mm.write_tuv(path)
                mm.close()
                tuvs[sp["seed"]] = path
        cpu = cpu_ensemble(mix, tuvs=tuvs)
    b.close()
    # tiled groups take one step per launch inside a batch of several groups
    geoms = {str(L): {"periodic": t["periodic"], "tile": list(t["tile"]), "ncol": t["ncol"],
                      "steps_per_launch": t["steps_per_launch"] if t["periodic"] == 1 else 1}
             for L, t in tuned.items()}
    return {"workload": f"{len(specs)} ring melts, L uniform on {{16,24,32,48,64}}, N log-uniform on [50,1000], "
                        f"density 1.2, seeds 1000..{999 + len(specs)}, relaxed: {args.batch_relax} steps from "
                        f"CreatePolymers",
            "monomers": moves, "steps": args.batch_steps, "warmup": args.batch_warmup,
            "occupied_site_fraction": occ,
            "batched": {"value": batched, "unit": UNIT, "ms": bms},
            "plain": {"value": plain, "unit": UNIT, "ms": pms,
                      "how": "each replica alone, same specs, sequential, from the same relaxed state"},
            "speedup": batched / plain, "batched_equals_plain_bits": same,
            "replicas_compared": len(check_idx), "autotuned_geometry": geoms,
            "cpu_reference": cpu}


# ---- served stream ------------------------------------------------------------
def served_leg(elp, dev, args):
    """Poisson arrivals into the continuous-batching server; job sizes drawn as
    the ensemble mix plus 5 % L=128/N=1000 jobs; latency = done - submitted."""
    import random
    import threading
    rate, dur = 200.0, args.served_seconds
    steps, dump = args.served_steps, args.served_dump
    full = (dur, steps, dump) == (60.0, 10000, 1000)
    rng = random.Random(20261203)
    mix = ensemble_mix(4096, first_seed=50000)
    arrivals, t = [], 0.0
    while True:
        t += rng.expovariate(rate)
        if t >= dur:
            break
        arrivals.append(t)
    jobs = []
    for i, ta in enumerate(arrivals):
        if rng.random() < 0.05:
            jobs.append((ta, dict(L=128, N=1000, seed=90000 + i)))
        else:
            m = mix[i % len(mix)]
            jobs.append((ta, dict(L=m["L"], N=m["N"], seed=m["seed"])))
    srv = elp.Server(device=dev, hbm_budget=150 << 30, quantum=args.served_quantum)
    # warm-up, not measured: one job per box size, so that the server's
    # groups (streams, job tables, layouts) exist before the stream starts,
    # as they do in a server that has been running
    for L in sorted({kw["L"] for _, kw in jobs}):
        kw = next(k for _, k in jobs if k["L"] == L)
        srv.submit(2 * args.served_quantum, dump_interval=args.served_quantum, device=dev,
                   **dict(kw, seed=kw["seed"] + 7))
    srv.drain(600)
    srv.poll(64)
    t0 = time.perf_counter()

    def submitter():
        for ta, kw in jobs:
            d = ta - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            srv.submit(steps, dump_interval=dump, device=dev, **kw)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    srv.drain(3600)
    wall = time.perf_counter() - t0
    res = srv.poll(len(jobs) + 16)
    srv.close()
    lat = sorted(r["t_done"] - r["t_submit"] for r in res)
    moves = sum(r["moves"] for r in res)
    ok = all(r["status"] == 0 and r["integrity"] == 0 for r in res)
    q = lambda f: lat[min(len(lat) - 1, int(f * len(lat)))]
    makespan = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    return {"workload": f"Poisson arrivals {rate:.0f} jobs/s for {dur:.0f} s ({len(jobs)} jobs), sizes as the ensemble "
                        f"mix plus 5% L=128/N=1000, {steps} steps each, dump every {dump} (rebuilt and copied to host, "
                        f"no files), HBM budget 150 GB; one warm-up job per box size before the stream"
                        + ("" if full else " [scaled-down stream]"),
            "jobs": len(res), "all_ok": ok, "latency_s": {"p50": q(0.50), "p99": q(0.99), "max": lat[-1]},
            "value": moves / makespan, "unit": UNIT, "makespan_s": makespan, "wall_s": wall,
            "quantum": args.served_quantum}


def reference_start(w, relax, tmpdir):
    """The relaxed melt the reference arm starts from: produced on the GPU by
    this engine (untimed), written as a TUV file.  Without a GPU the
    reference starts from its own CreatePolymers melt."""
    try:
        import torch
        if not torch.cuda.is_available() or relax <= 0:
            return None, "CreatePolymers initial melt (no GPU to relax it)" if relax > 0 else "CreatePolymers"
        sys.path.insert(0, os.path.join(REPO, "mc-polymer-simulation_b200", "python"))
        import elp
        m = relaxed_melt(elp, w, w["seed"], 0, 20, relax)
        path = os.path.join(tmpdir, f"relaxed_L{w['L']}.res")
        m.write_tuv(path)
        m.close()
        return path, f"melt relaxed {relax} steps on the GPU (untimed), read by the reference's ReadLatticeFile"
    except Exception as e:   # the arm still runs, from the reference's own initial melt
        return None, f"CreatePolymers initial melt (relaxing failed: {e})"


def run_reference(args, rank, world):
    import tempfile

    if rank != 0:
        return None
    w = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    steps_per = max(1, args.ref_steps)
    tot_moves, tot_wall = 0.0, 0.0
    cb = None
    with tempfile.TemporaryDirectory(prefix="elp_ref_") as tmp:
        tuv, desc = reference_start(w, args.relax, tmp)
        for i in range(args.warmup + args.steps):
            cb = cpu_baseline(w, steps_per, threads, tuv, desc)
            if i >= args.warmup:
                moves = threads * steps_per * w["N"] * npol(w)
                tot_moves += moves
                tot_wall += moves / cb["value"]
    value = tot_moves / tot_wall
    cb["value"] = value
    cfg = common_config(w, args.relax)
    return {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (reference CreatePolymers initial melt, relaxed on the GPU before timing)",
            "config": dict(cfg, parallelism=f"replicas x{world}"),
            "reference_step": f"{steps_per} MC steps of the reference's DoMCStep per process, {threads} processes "
                              f"at once on {threads} host cores, from the {desc}",
            "cpu_baseline": cb, "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="elp", choices=["elp", "reference"])
    ap.add_argument("--workload", default="L128", choices=sorted(WORKLOADS))
    ap.add_argument("--spl", type=int, default=100, help="MC steps per sweep launch (headline workload and e2e)")
    ap.add_argument("--relax", type=int, default=2000,
                    help="untimed GPU steps from CreatePolymers before the headline melt is timed (both arms)")
    ap.add_argument("--l256-relax", type=int, default=5000)
    ap.add_argument("--batch-relax", type=int, default=2000)
    ap.add_argument("--l256-spl", type=int, default=10, help="MC steps per sweep launch of the L=256 leg")
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--ref-steps", type=int, default=8)
    ap.add_argument("--one-step-launches", type=int, default=100,
                    help="launches of one MC step each, timed after the headline launches (0: none)")
    ap.add_argument("--e2e-interval", type=int, default=100)
    ap.add_argument("--e2e-reps", type=int, default=20)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-l256", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-gpu-reference", action="store_true")
    ap.add_argument("--gp3-interval", type=int, default=5000,
                    help="steps per timed interval of the reference gpupol3 leg (it runs two)")
    ap.add_argument("--replicas", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--batch-warmup", type=int, default=20)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--served-seconds", type=float, default=60.0)
    ap.add_argument("--served-steps", type=int, default=10000)
    ap.add_argument("--served-dump", type=int, default=1000)
    ap.add_argument("--served-quantum", type=int, default=50)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    try:
        line = run_reference(args, rank, world) if args.impl == "reference" else run_elp(args, rank, world)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
