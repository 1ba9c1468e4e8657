"""ctypes binding of oracle/liboracle.so (test infrastructure: efpol restatement
and the host replay of the GPU schedule)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(REPO, "oracle", "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(path)
        L.orc_efpol_new.restype = C.c_void_p
        L.orc_efpol_new.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32]
        L.orc_efpol_free.argtypes = [C.c_void_p]
        L.orc_efpol_create.argtypes = [C.c_void_p]
        L.orc_efpol_mcstep.restype = C.c_long
        L.orc_efpol_mcstep.argtypes = [C.c_void_p, C.c_long]
        L.orc_efpol_check.argtypes = [C.c_void_p]
        L.orc_efpol_write_tuv.restype = C.c_long
        L.orc_efpol_write_tuv.argtypes = [C.c_void_p, C.c_char_p, C.c_long]
        L.orc_efpol_read_tuv.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_efpol_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_build_table.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_get_npol.argtypes = [C.c_double, C.c_int, C.c_long]
        L.orc_philox.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_replay_new.restype = C.c_void_p
        L.orc_replay_new.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_uint32, C.c_uint32]
        L.orc_replay_free.argtypes = [C.c_void_p]
        L.orc_replay_load.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_replay_export.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_replay_steps.argtypes = [C.c_void_p, C.c_long]
        L.orc_replay_set_linear.argtypes = [C.c_void_p, C.c_int]
        L.orc_replay_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64]
        _LIB = L
    return _LIB


def table(model: int = 1):
    """(trans, add_occ, rem_occ) as numpy arrays."""
    buf = (C.c_uint8 * (4096 * 4 * 3 + 256 * 4))()
    lib().orc_build_table(buf, model, 1)
    a = np.frombuffer(bytes(buf), dtype=np.uint32)
    return a[:4096].copy(), a[4096:8192].astype(np.int32), a[8192:12288].astype(np.int32)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


class Efpol:
    """The efpol restatement (one ring melt, sequential Tausworthe dynamics)."""

    def __init__(self, L, N, P, seed, model=1, pol_type=1):
        self.L, self.N, self.P = L, N, P
        self.h = lib().orc_efpol_new(L, N, P, pol_type, model, seed)

    def create(self):
        lib().orc_efpol_create(self.h)

    def step(self, n):
        return lib().orc_efpol_mcstep(self.h, n)

    def check(self):
        return lib().orc_efpol_check(self.h)

    def tuv(self) -> str:
        cap = 64 + self.P * (self.N + 64)
        buf = C.create_string_buffer(cap)
        n = lib().orc_efpol_write_tuv(self.h, buf, cap)
        assert n > 0
        return buf.raw[:n].decode()

    def read(self, text: str):
        return lib().orc_efpol_read_tuv(self.h, text.encode())

    def export(self):
        start = np.zeros((self.P, 3), dtype=np.int32)
        bonds = np.zeros((self.P, self.N), dtype=np.uint8)
        lib().orc_efpol_export(self.h, start.ctypes.data, bonds.ctypes.data)
        return start, bonds

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_efpol_free(self.h)
            self.h = None


class Geom(C.Structure):
    _fields_ = [("L", C.c_int), ("periodic", C.c_int), ("tt", C.c_int), ("tu", C.c_int), ("tv", C.c_int),
                ("ncol", C.c_int)]


class Replay:
    """Host replay of the GPU sweep schedule (bit-exact twin of the kernels)."""

    def __init__(self, L, N, P, seed, salt=0, periodic=True, tile=(32, 32, 32), ncol=16, linear=False):
        self.L, self.N, self.P = L, N, P
        g = Geom(L, 1 if periodic else 0, tile[0], tile[1], tile[2], ncol)
        self.h = lib().orc_replay_new(C.byref(g), N, P, seed, salt)
        lib().orc_replay_set_linear(self.h, 1 if linear else 0)

    def load(self, start, bonds):
        start = np.ascontiguousarray(start, dtype=np.int32)
        bonds = np.ascontiguousarray(bonds, dtype=np.uint8)
        return lib().orc_replay_load(self.h, start.ctypes.data, bonds.ctypes.data)

    def export(self):
        start = np.zeros((self.P, 3), dtype=np.int32)
        bonds = np.zeros((self.P, self.N), dtype=np.uint8)
        rc = lib().orc_replay_export(self.h, start.ctypes.data, bonds.ctypes.data)
        return rc, start, bonds

    def steps(self, n):
        lib().orc_replay_steps(self.h, n)

    def set_state(self, words, records, step):
        """Continue from a given state (site words, records) at absolute `step`."""
        words = np.ascontiguousarray(words, dtype=np.uint32)
        records = np.ascontiguousarray(records, dtype=np.uint32)
        assert words.shape == (self.L ** 3,) and records.shape == (self.P, 4)
        lib().orc_replay_set_state(self.h, words.ctypes.data, records.ctypes.data, step)

    def _struct(self):
        # orc_replay: geom(6 ints), N, P, seed, salt, uint64 step, lat*, rec*, accepted, attempted
        class R(C.Structure):
            _fields_ = [("g", Geom), ("N", C.c_int), ("P", C.c_int), ("seed", C.c_uint32), ("salt", C.c_uint32),
                        ("step", C.c_uint64), ("lat", C.POINTER(C.c_uint32)), ("rec", C.POINTER(C.c_uint32)),
                        ("accepted", C.c_uint64), ("attempted", C.c_uint64), ("linear", C.c_int)]
        return R.from_address(self.h)

    def lattice(self):
        r = self._struct()
        return np.ctypeslib.as_array(r.lat, shape=(self.L ** 3,)).copy()

    def records(self):
        r = self._struct()
        return np.ctypeslib.as_array(r.rec, shape=(self.P, 4)).copy()

    @property
    def accepted(self):
        return self._struct().accepted

    @property
    def step_count(self):
        return self._struct().step

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_replay_free(self.h)
            self.h = None
