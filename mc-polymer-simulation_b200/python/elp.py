"""ctypes binding of lib/libelp.so (the C ABI declared in include/elp.h).

This is what the tests and bench.py use to drive the engine; it adds no logic
of its own.  The library must exist (``make -C mc-polymer-simulation_b200``);
there is no fallback: every call goes to the sm_100a kernels through the
C ABI, and a missing library or device raises ``ElpError``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "lib", "libelp.so")

OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_IO, ERR_FORMAT, ERR_INTEGRITY, ERR_STATE, ERR_BUSY = range(9)


class ElpError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"elp status {status}: {msg}")
        self.status = status


class JobSpec(C.Structure):
    _fields_ = [("L", C.c_int32), ("N", C.c_int32), ("P", C.c_int32), ("density", C.c_double),
                ("seed", C.c_uint32), ("salt", C.c_uint32), ("periodic", C.c_int32), ("tile", C.c_int32 * 3),
                ("ncol", C.c_int32), ("device", C.c_int32), ("steps_per_launch", C.c_int32),
                ("kernel", C.c_int32), ("linear", C.c_int32)]


class Info(C.Structure):
    _fields_ = [("L", C.c_int32), ("N", C.c_int32), ("P", C.c_int32), ("periodic", C.c_int32),
                ("tile", C.c_int32 * 3), ("ncol", C.c_int32), ("domains", C.c_int32), ("threads", C.c_int32),
                ("specialised", C.c_int32), ("smem_bytes", C.c_uint64), ("step", C.c_uint64), ("device_bytes", C.c_uint64),
                ("linear", C.c_int32), ("kernels", C.c_uint64)]


EXPORTED = [
    "elp_default_spec", "elp_create", "elp_init_melt", "elp_load_chains", "elp_load_tuv", "elp_run",
    "elp_run_timed", "elp_stream", "elp_sync", "elp_fetch_chains", "elp_fetch_checked", "elp_write_tuv", "elp_check", "elp_get_info",
    "elp_get_state", "elp_set_state", "elp_accepted", "elp_debug_waits", "elp_time_factor", "elp_destroy", "elp_transition_table",
    "elp_format_tuv", "elp_status_string", "elp_last_error",
    "elp_batch_create", "elp_batch_size", "elp_batch_init_melts", "elp_batch_load_chains", "elp_batch_run",
    "elp_batch_run_timed", "elp_batch_sync", "elp_batch_fetch_chains", "elp_batch_get_state", "elp_batch_check",
    "elp_batch_accepted", "elp_batch_job_info", "elp_batch_destroy", "elp_autotune",
    "elp_server_default_opts", "elp_server_create", "elp_server_submit", "elp_server_poll", "elp_server_get_stats",
    "elp_server_drain", "elp_server_destroy", "elp_check_noalloc", "elp_observe", "elp_batch_observe",
    "elp_ptl_open", "elp_ptl_append", "elp_ptl_close", "elp_double_chains",
    "elp_scaleup_tuv", "elp_tuv_to_xyz", "elp_tuv_to_pov",
]

OBS_MAX_BINS = 64

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ElpError(ERR_STATE, f"{LIB_PATH} not built (run make -C {PKG})")
    L = C.CDLL(LIB_PATH)
    vp, i32, u32, i64, u64 = C.c_void_p, C.c_int32, C.c_uint32, C.c_int64, C.c_uint64
    sig = {
        "elp_default_spec": (None, [vp]),
        "elp_create": (i32, [vp, vp]),
        "elp_init_melt": (i32, [vp]),
        "elp_load_chains": (i32, [vp, vp, vp, u64]),
        "elp_load_tuv": (i32, [vp, C.c_char_p, u64]),
        "elp_run": (i32, [vp, i64]),
        "elp_run_timed": (i32, [vp, i64, vp]),
        "elp_stream": (vp, [vp]),
        "elp_sync": (i32, [vp]),
        "elp_fetch_chains": (i32, [vp, vp, vp]),
        "elp_fetch_checked": (i32, [vp, vp, vp, vp]),
        "elp_write_tuv": (i32, [vp, C.c_char_p]),
        "elp_check": (i32, [vp, vp]),
        "elp_get_info": (i32, [vp, vp]),
        "elp_get_state": (i32, [vp, vp, vp]),
        "elp_set_state": (i32, [vp, vp, vp, u64]),
        "elp_accepted": (i32, [vp, vp]),
        "elp_debug_waits": (i32, [vp, u32, i32]),
        "elp_time_factor": (C.c_double, [i32, i32, i32, i32]),
        "elp_destroy": (None, [vp]),
        "elp_transition_table": (i32, [vp]),
        "elp_format_tuv": (i32, [i32, i32, i32, vp, vp, vp, C.c_size_t, vp]),
        "elp_status_string": (C.c_char_p, [i32]),
        "elp_last_error": (C.c_char_p, []),
        "elp_batch_create": (i32, [vp, i32, i32, vp]),
        "elp_batch_size": (i32, [vp]),
        "elp_batch_init_melts": (i32, [vp]),
        "elp_batch_load_chains": (i32, [vp, i32, vp, vp, u64]),
        "elp_batch_run": (i32, [vp, i64]),
        "elp_batch_run_timed": (i32, [vp, i64, vp]),
        "elp_batch_sync": (i32, [vp]),
        "elp_batch_fetch_chains": (i32, [vp, i32, vp, vp]),
        "elp_batch_get_state": (i32, [vp, i32, vp, vp]),
        "elp_batch_check": (i32, [vp, i32, vp]),
        "elp_batch_accepted": (i32, [vp, i32, vp]),
        "elp_batch_job_info": (i32, [vp, i32, vp]),
        "elp_batch_destroy": (None, [vp]),
        "elp_autotune": (i32, [vp, i32, i32, vp, vp]),
        "elp_server_default_opts": (None, [vp]),
        "elp_server_create": (i32, [vp, vp]),
        "elp_server_submit": (i32, [vp, vp, i64, i64, C.c_char_p, vp]),
        "elp_server_poll": (i32, [vp, vp, i32, vp]),
        "elp_server_get_stats": (i32, [vp, vp]),
        "elp_server_drain": (i32, [vp, C.c_double]),
        "elp_server_destroy": (None, [vp]),
        "elp_check_noalloc": (i32, [vp, vp, i32, i32, i32, vp, vp]),
        "elp_observe": (i32, [vp, vp, vp, vp, vp, i32]),
        "elp_batch_observe": (i32, [vp, i32, vp, vp, vp, vp, i32]),
        "elp_ptl_open": (i32, [C.c_char_p, i32, i32, i32, i32, C.c_size_t, vp]),
        "elp_ptl_append": (i32, [vp, vp, vp]),
        "elp_ptl_close": (i32, [vp]),
        "elp_double_chains": (i32, [i32, i32, i32, vp, vp, vp, vp]),
        "elp_scaleup_tuv": (i32, [C.c_char_p, C.c_char_p]),
        "elp_tuv_to_xyz": (i32, [C.c_char_p, i32, C.c_char_p]),
        "elp_tuv_to_pov": (i32, [C.c_char_p, C.c_char_p, i32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != OK:
        raise ElpError(status, lib().elp_last_error().decode(errors="replace"))


def transition_table() -> np.ndarray:
    out = np.zeros(4096, dtype=np.uint8)
    check(lib().elp_transition_table(out.ctypes.data))
    return out


def time_factor(periodic, tx, ty, tz) -> float:
    """Clock of a domain geometry against reference efpol's (elp_time_factor);
    0 for a tile shape not measured."""
    return lib().elp_time_factor(int(periodic), tx, ty, tz)


def format_tuv(L, start, bonds) -> str:
    start = np.ascontiguousarray(start, dtype=np.int32)
    bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
    P, N = bonds.shape
    n = C.c_size_t()
    check(lib().elp_format_tuv(L, N, P, start.ctypes.data, bonds.ctypes.data, None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(lib().elp_format_tuv(L, N, P, start.ctypes.data, bonds.ctypes.data, buf, n.value + 1, C.byref(n)))
    return buf.raw[:n.value].decode()


def spec(L=32, N=100, P=0, density=1.2, seed=1, salt=0, periodic=-1, tile=(0, 0, 0), ncol=0, device=0,
         steps_per_launch=1, kernel=0, linear=0) -> JobSpec:
    s = JobSpec()
    lib().elp_default_spec(C.byref(s))
    s.L, s.N, s.P, s.density, s.seed, s.salt = L, N, P, density, seed, salt
    s.periodic = periodic
    s.tile[0], s.tile[1], s.tile[2] = tile
    s.ncol, s.device, s.steps_per_launch, s.kernel = ncol, device, steps_per_launch, kernel
    s.linear = 1 if linear else 0
    return s


def _observe(call, P, nbins):
    out = dict(cms_tuv=np.zeros((P, 3)), rg2=np.zeros(P), sl=np.zeros(P), run_hist=np.zeros(nbins, dtype=np.uint64))
    check(call(out["cms_tuv"].ctypes.data, out["rg2"].ctypes.data, out["sl"].ctypes.data,
               out["run_hist"].ctypes.data, nbins))
    return out


def double_chains(L, start, bonds):
    """efpol's DoubleLattice on host chains: (2L, start', bonds' with 8N bonds per ring)."""
    start = np.ascontiguousarray(start, dtype=np.int32)
    bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
    P, N = bonds.shape
    s2 = np.zeros((P, 3), dtype=np.int32)
    b2 = np.zeros((P, 8 * N), dtype=np.uint8)
    check(lib().elp_double_chains(L, N, P, start.ctypes.data, bonds.ctypes.data, s2.ctypes.data, b2.ctypes.data))
    return 2 * L, s2, b2


class PTLWriter:
    """Per-ring time series files written during a run (elp_ptl_*): host only."""

    def __init__(self, sample_dir, P, N, ntime, dev=0, buffer_bytes=0):
        self.h = C.c_void_p()
        self.P, self.N = P, N
        check(lib().elp_ptl_open(sample_dir.encode(), dev, P, N, ntime, buffer_bytes, C.byref(self.h)))

    def append(self, start, bonds):
        start = np.ascontiguousarray(start, dtype=np.int32)
        bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
        assert start.shape == (self.P, 3) and bonds.shape == (self.P, self.N)
        check(lib().elp_ptl_append(self.h, start.ctypes.data, bonds.ctypes.data))

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            h, self.h = self.h, C.c_void_p()
            check(lib().elp_ptl_close(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(copies=1, steps=20, **kw):
    """Fastest domain geometry for a melt (see elp_autotune).  Returns
    (spec dict, ms per step)."""
    src = spec(**kw)
    out = JobSpec()
    ms = C.c_float()
    check(lib().elp_autotune(C.byref(src), copies, steps, C.byref(out), C.byref(ms)))
    d = dict(kw)
    d.update(periodic=out.periodic, tile=tuple(out.tile), ncol=out.ncol, steps_per_launch=out.steps_per_launch)
    return d, ms.value


class Melt:
    """One ring melt on one GPU (an elp_ctx)."""

    def __init__(self, **kw):
        self.h = C.c_void_p()
        check(lib().elp_create(C.byref(spec(**kw)), C.byref(self.h)))
        i = self.info()
        self.L, self.N, self.P = i.L, i.N, i.P

    def info(self) -> Info:
        i = Info()
        check(lib().elp_get_info(self.h, C.byref(i)))
        return i

    @property
    def step(self) -> int:
        return self.info().step

    def init_melt(self):
        check(lib().elp_init_melt(self.h))

    def load_chains(self, start, bonds, step=0):
        start = np.ascontiguousarray(start, dtype=np.int32)
        bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
        assert start.shape == (self.P, 3) and bonds.shape == (self.P, self.N)
        check(lib().elp_load_chains(self.h, start.ctypes.data, bonds.ctypes.data, step))

    def load_tuv(self, path, step=0):
        check(lib().elp_load_tuv(self.h, path.encode(), step))

    def run(self, nsteps):
        check(lib().elp_run(self.h, nsteps))

    def run_timed(self, nsteps) -> float:
        ms = C.c_float()
        check(lib().elp_run_timed(self.h, nsteps, C.byref(ms)))
        return ms.value

    def sync(self):
        check(lib().elp_sync(self.h))

    def stream_ptr(self) -> int:
        """cudaStream_t of this melt (e.g. for torch.cuda.ExternalStream)."""
        return lib().elp_stream(self.h) or 0

    def fetch(self, start=None, bonds=None):
        """Rings as (start (P,3) int32, bonds (P,N) uint8), written into the given
        C-contiguous arrays (e.g. pinned host memory) or into new ones."""
        start = np.zeros((self.P, 3), dtype=np.int32) if start is None else start
        bonds = np.zeros((self.P, self.N), dtype=np.uint8) if bonds is None else bonds
        assert start.shape == (self.P, 3) and start.dtype == np.int32 and start.flags.c_contiguous
        assert bonds.shape == (self.P, self.N) and bonds.dtype == np.uint8 and bonds.flags.c_contiguous
        check(lib().elp_fetch_chains(self.h, start.ctypes.data, bonds.ctypes.data))
        return start, bonds

    def fetch_checked(self):
        """(start, bonds, integrity code) from one walk and one scan (elp_fetch_checked)."""
        start = np.zeros((self.P, 3), dtype=np.int32)
        bonds = np.zeros((self.P, self.N), dtype=np.uint8)
        code = C.c_int32()
        check(lib().elp_fetch_checked(self.h, start.ctypes.data, bonds.ctypes.data, C.byref(code)))
        return start, bonds, code.value

    def write_tuv(self, path):
        check(lib().elp_write_tuv(self.h, path.encode()))

    def observe(self, nbins=16):
        """In-situ observables (elp_observe): cms_tuv (P,3), rg2 (P), sl (P), run_hist (nbins)."""
        return _observe(lambda *a: lib().elp_observe(self.h, *a), self.P, nbins)

    def check(self) -> int:
        code = C.c_int32()
        check(lib().elp_check(self.h, C.byref(code)))
        return code.value

    def state(self):
        w = np.zeros(self.L ** 3, dtype=np.uint32)
        r = np.zeros((self.P, 4), dtype=np.uint32)
        check(lib().elp_get_state(self.h, w.ctypes.data, r.ctypes.data))
        return w, r

    def set_state(self, words, records, step):
        words = np.ascontiguousarray(words, dtype=np.uint32)
        records = np.ascontiguousarray(records, dtype=np.uint32)
        check(lib().elp_set_state(self.h, words.ctypes.data, records.ctypes.data, step))

    def accepted(self) -> int:
        v = C.c_uint64()
        check(lib().elp_accepted(self.h, C.byref(v)))
        return v.value

    def debug_waits(self, polls=0, hold_block=-1):
        """Bound of the grid-barrier waits in tiled multi-step launches (elp_debug_waits)."""
        check(lib().elp_debug_waits(self.h, polls, hold_block))

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().elp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Many melts advanced together on one GPU (an elp_batch)."""

    def __init__(self, specs, device=0):
        arr = (JobSpec * len(specs))()
        for i, kw in enumerate(specs):
            arr[i] = spec(**kw)
        self.h = C.c_void_p()
        check(lib().elp_batch_create(arr, len(specs), device, C.byref(self.h)))
        self.n = lib().elp_batch_size(self.h)
        self.infos = [self.info(j) for j in range(self.n)]

    def info(self, j) -> Info:
        i = Info()
        check(lib().elp_batch_job_info(self.h, j, C.byref(i)))
        return i

    def init_melts(self):
        check(lib().elp_batch_init_melts(self.h))

    def load_chains(self, j, start, bonds, step=0):
        start = np.ascontiguousarray(start, dtype=np.int32)
        bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
        check(lib().elp_batch_load_chains(self.h, j, start.ctypes.data, bonds.ctypes.data, step))

    def run(self, nsteps):
        check(lib().elp_batch_run(self.h, nsteps))

    def run_timed(self, nsteps) -> float:
        ms = C.c_float()
        check(lib().elp_batch_run_timed(self.h, nsteps, C.byref(ms)))
        return ms.value

    def sync(self):
        check(lib().elp_batch_sync(self.h))

    def fetch(self, j):
        i = self.infos[j]
        start = np.zeros((i.P, 3), dtype=np.int32)
        bonds = np.zeros((i.P, i.N), dtype=np.uint8)
        check(lib().elp_batch_fetch_chains(self.h, j, start.ctypes.data, bonds.ctypes.data))
        return start, bonds

    def observe(self, j, nbins=16):
        return _observe(lambda *a: lib().elp_batch_observe(self.h, j, *a), self.infos[j].P, nbins)

    def state(self, j):
        i = self.infos[j]
        w = np.zeros(i.L ** 3, dtype=np.uint32)
        r = np.zeros((i.P, 4), dtype=np.uint32)
        check(lib().elp_batch_get_state(self.h, j, w.ctypes.data, r.ctypes.data))
        return w, r

    def check(self, j) -> int:
        code = C.c_int32()
        check(lib().elp_batch_check(self.h, j, C.byref(code)))
        return code.value

    def accepted(self, j) -> int:
        v = C.c_uint64()
        check(lib().elp_batch_accepted(self.h, j, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().elp_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget", C.c_uint64), ("quantum", C.c_int32),
                ("io_threads", C.c_int32), ("max_jobs", C.c_int32)]


class JobResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("integrity", C.c_int32), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double), ("steps", C.c_uint64), ("moves", C.c_uint64),
                ("dumps", C.c_uint32), ("checksum", C.c_uint64), ("L", C.c_int32), ("N", C.c_int32),
                ("P", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("queued", C.c_uint64),
                ("resident", C.c_uint64), ("bytes_in_use", C.c_uint64), ("moves", C.c_double),
                ("clock", C.c_double), ("fatal", C.c_int32)]


def ring_checksum(start, bonds) -> int:
    """FNV-1a of start[3P] (int32) then bonds[P*N], as the server reports."""
    h = 0xCBF29CE484222325
    for b in np.ascontiguousarray(start, dtype=np.int32).tobytes() + np.ascontiguousarray(bonds, np.uint8).tobytes():
        h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


class Server:
    """Continuous-batching job server on one GPU (an elp_server)."""

    def __init__(self, device=0, hbm_budget=150 << 30, quantum=100, io_threads=4, max_jobs=4096):
        o = ServerOpts()
        lib().elp_server_default_opts(C.byref(o))
        o.device, o.hbm_budget, o.quantum, o.io_threads, o.max_jobs = device, hbm_budget, quantum, io_threads, max_jobs
        self.h = C.c_void_p()
        check(lib().elp_server_create(C.byref(o), C.byref(self.h)))

    def submit(self, nsteps, dump_interval=0, dump_dir=None, **kw) -> int:
        jid = C.c_uint64()
        d = dump_dir.encode() if dump_dir else None
        check(lib().elp_server_submit(self.h, C.byref(spec(**kw)), nsteps, dump_interval, d, C.byref(jid)))
        return jid.value

    def poll(self, cap=1024):
        out = (JobResult * cap)()
        n = C.c_int32()
        check(lib().elp_server_poll(self.h, out, cap, C.byref(n)))
        return [{f: getattr(out[i], f) for f, _ in JobResult._fields_} for i in range(n.value)]

    def stats(self):
        st = ServerStats()
        check(lib().elp_server_get_stats(self.h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}

    def drain(self, timeout=600.0):
        check(lib().elp_server_drain(self.h, timeout))

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            lib().elp_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
