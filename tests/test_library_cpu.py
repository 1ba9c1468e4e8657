"""The C ABI without a GPU: the library loads, exports every symbol declared in
include/elp.h, reproduces the reference's transition table and TUV format,
and fails cleanly (status code, no abort) when no CUDA device is present."""
import gzip
import os
import re

import numpy as np
import pytest

import elp
import observables as obs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(REPO, "tests", "golden")


def declared_functions():
    text = open(os.path.join(REPO, "include", "elp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(elp_[a-z_0-9]+)\s*\(", text)))


def test_header_symbols_exported():
    import ctypes
    lib = ctypes.CDLL(elp.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/elp.h but not exported"
    assert set(names) <= set(elp.EXPORTED) | set(names)


def test_transition_table_matches_reference():
    ref = np.load(os.path.join(GOLD, "table_sl_equal.npz"))["trans"]
    assert np.array_equal(elp.transition_table(), (ref & 0xFF).astype(np.uint8))


@pytest.mark.parametrize("name", ["efpol_L32_N100_s1_t0.res.gz", "efpol_L16_N50_s3_t100.res.gz",
                                  "efpol_L32_N100_s1_t200.res.gz"])
def test_tuv_format_byte_identical(name):
    text = gzip.open(os.path.join(GOLD, name), "rt").read()
    L, start, bonds = obs.parse_tuv(text)
    assert elp.format_tuv(L, start, bonds) == text


def test_no_device_is_a_clean_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(elp.ElpError) as e:
        elp.Melt(L=16, N=50)
    assert e.value.status == elp.ERR_CUDA


def test_bad_arguments_rejected_before_device():
    with pytest.raises(elp.ElpError) as e:
        elp.Melt(L=3, N=50)
    assert e.value.status == elp.ERR_ARG
    with pytest.raises(elp.ElpError) as e:
        elp.Melt(L=16, N=2)
    assert e.value.status == elp.ERR_ARG
    with pytest.raises(elp.ElpError) as e:      # 12 has no valid colour modulus, tiles cannot divide it
        elp.Melt(L=17, N=50, periodic=1)
    assert e.value.status == elp.ERR_ARG
