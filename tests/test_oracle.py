"""The oracle pinned against the reference (CPU only).

Fixtures in tests/golden/ were produced by the reference's own efpol, compiled
from its sources (tests/golden/make_golden.py).  The restatement must match
them bit for bit: the transition table, the t=0 configuration and whole
trajectories (it consumes the same Tausworthe stream in the same order).
"""
import gzip
import os

import numpy as np
import pytest

import observables as obs
from oracle_binding import Efpol, philox, table

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold_text(name):
    with gzip.open(os.path.join(GOLD, name), "rt") as f:
        return f.read()


@pytest.mark.parametrize("model,name", [(1, "sl_equal"), (2, "sl_double"), (4, "sl_quad")])
def test_table_matches_reference(model, name):
    ref = np.load(os.path.join(GOLD, f"table_{name}.npz"))
    trans, add, rem = table(model)
    assert np.array_equal(trans, ref["trans"])
    assert np.array_equal(add, ref["add_occ"])
    assert np.array_equal(rem, ref["rem_occ"])


def test_table_is_symmetric_for_rings():
    """Every ring move is listed as often as its reverse, so the single-monomer
    kernel is symmetric and the uniform measure is stationary under any
    state-independent choice of which monomer to update."""
    trans, _, _ = table(1)
    mult = {}
    for s1 in range(15):
        for s2 in range(15):
            for k in range(16):
                e = int(trans[s1 * 256 + s2 * 16 + k])
                d = (e & 15, (e >> 4) & 15)
                if d != (0, 0):
                    mult[(s1, s2, d)] = mult.get((s1, s2, d), 0) + 1
    for (s1, s2, d), m in mult.items():
        assert mult.get((d[0], d[1], (s1, s2)), 0) == m


@pytest.mark.parametrize("name,pol_type", [("efpol_L32_N100_s1_t0.res.gz", 1), ("efpol_lin_L32_N100_s1_t0.res.gz", 2)])
def test_initial_state_byte_identical(name, pol_type):
    ref = gold_text(name)
    e = Efpol(32, 100, 393, 1, pol_type=pol_type)
    e.create()
    assert e.check() == 0
    assert e.tuv() == ref


@pytest.mark.parametrize("L,N,seed,times,fmt,pol_type", [
    (16, 50, 3, list(range(0, 101, 10)), "efpol_L16_N50_s3_t{}.res.gz", 1),
    (32, 100, 1, [0, 100, 200], "efpol_L32_N100_s1_t{}.res.gz", 1),
    (16, 50, 3, list(range(0, 101, 10)), "efpol_lin_L16_N50_s3_t{}.res.gz", 2),
    (32, 100, 1, [0, 100, 200], "efpol_lin_L32_N100_s1_t{}.res.gz", 2),
])
def test_trajectory_bit_exact(L, N, seed, times, fmt, pol_type):
    P = max(1, int(1.2 * L ** 3 / N + 0.5))
    e = Efpol(L, N, P, seed, pol_type=pol_type)
    e.create()
    prev = 0
    for t in times:
        e.step(t - prev)
        prev = t
        assert e.check() == 0
        assert e.tuv() == gold_text(fmt.format(t)), f"diverged by t={t}"


def test_tuv_roundtrip_and_python_formatter():
    text = gold_text("efpol_L16_N50_s3_t100.res.gz")
    L, start, bonds = obs.parse_tuv(text)
    assert obs.format_tuv(L, start, bonds) == text
    e = Efpol(16, 50, start.shape[0], 0)
    assert e.read(text) == 0
    assert e.check() == 0
    assert e.tuv() == text


def test_integrity_check_catches_planted_faults():
    """Faults are planted in the oracle's own state, on the CPU."""
    text = gold_text("efpol_L16_N50_s3_t50.res.gz")
    L, start, bonds = obs.parse_tuv(text)
    broken = bonds.copy()
    k = int(np.flatnonzero(broken[0])[0])
    broken[0, k] = 0x3          # not a bond
    e = Efpol(16, 50, start.shape[0], 0)
    assert e.read(obs.format_tuv(L, start, broken)) == 0
    assert e.check() != 0


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    assert philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]
