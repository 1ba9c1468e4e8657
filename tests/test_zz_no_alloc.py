"""elp_check_noalloc: the integrity check for callers that cannot allocate
device memory (their HBM is owned by another pool, they run under a memory
quota, or they cannot afford an allocation's device synchronisation).  It
must report exactly what elp_check reports for the same melt, call after
call, while its scratch lives in a static device array.

Collected last on purpose, so a stopping run has executed every other test."""
import ctypes as C

import numpy as np
import pytest

import elp

pytestmark = pytest.mark.gpu


def noalloc():
    lib = C.CDLL(elp.LIB_PATH)
    f = lib.elp_check_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    return f


def device_copy(words, records):
    import torch
    dw = torch.from_numpy(np.ascontiguousarray(words).view(np.int32)).cuda()
    dr = torch.from_numpy(np.ascontiguousarray(records).view(np.int32).ravel()).cuda()
    torch.cuda.synchronize()
    return dw, dr


def check_both_ways(m: elp.Melt, words, records):
    """Existing entry point (elp_check) on the melt vs the no-alloc entry point
    on a device copy of the same words, twice in a row."""
    f = noalloc()
    want = m.check()
    dw, dr = device_copy(words, records)
    i = m.info()
    got = []
    for _ in range(2):
        code = C.c_int32(-1)
        st = f(dw.data_ptr(), dr.data_ptr(), i.L, i.N, i.P, None, C.byref(code))
        assert st == 0, elp.lib().elp_last_error().decode()
        got.append(code.value)
    return want, got


@pytest.mark.parametrize("kw,steps", [(dict(L=16, N=50, seed=3), 40),
                                      (dict(L=64, N=200, seed=4, periodic=0, tile=(32, 32, 32)), 5),
                                      (dict(L=32, N=100, seed=5), 20)])
def test_noalloc_check_equals_elp_check(kw, steps):
    m = elp.Melt(**kw)
    m.init_melt()
    m.run(steps)
    w, r = m.state()
    want, got = check_both_ways(m, w, r)
    assert want == 0 and got == [want, want]


def test_noalloc_check_finds_the_same_faults():
    m = elp.Melt(L=16, N=50, seed=6)
    m.init_melt()
    m.run(25)
    w, r = m.state()
    # a run length that no longer adds up: one monomer too many
    bad = w.copy()
    k = int(np.flatnonzero((bad != 0) & ((bad & 16) == 0))[0])
    bad[k] += np.uint32(1 << 16)
    m.set_state(bad, r, 25)
    want, got = check_both_ways(m, bad, r)
    assert want != 0 and got == [want, want]
    # an invalid bond code on an occupied site
    bad = w.copy()
    bad[k] = (bad[k] & ~np.uint32(15)) | np.uint32(3)
    m.set_state(bad, r, 25)
    want, got = check_both_ways(m, bad, r)
    assert want != 0 and got == [want, want]


def test_noalloc_rejects_melts_beyond_its_array():
    f = noalloc()
    code = C.c_int32(-1)
    # the size check comes before any device access
    st = f(C.c_void_p(16), C.c_void_p(16), 128, 1000, 2517, None, C.byref(code))
    assert st == elp.ERR_ARG
    assert b"at most" in elp.lib().elp_last_error()
