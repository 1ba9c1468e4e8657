"""The replay of the GPU schedule for linear chains (host only).

The replay is the bit-exact twin of the kernels; for linear chains it adds
the end moves of efpol_lin (efpol's table rows with the end marker 0xf) at
anchors next to the chain ends.  Here it is checked on its own: states of
the reference efpol_lin load and export unchanged, and after replayed steps
every chain is still a valid efpol_lin chain (oracle integrity check) of the
same length, with both ends moving."""
import os

import numpy as np
import pytest

import observables as obs
from oracle_binding import Efpol, Replay

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["efpol_lin_L32_N100_s1_t0", "efpol_lin_L32_N100_s1_t200"])
def test_linear_state_roundtrip(name):
    L, start, bonds = obs.read_tuv(os.path.join(GOLD, name + ".res.gz"))
    P, N = bonds.shape
    r = Replay(L, N, P, 1, linear=True)
    assert r.load(start, bonds) == 0
    rc, s2, b2 = r.export()
    assert rc == 0 and np.array_equal(s2, start) and np.array_equal(b2, bonds)


@pytest.mark.parametrize("periodic,tile", [(True, (32, 32, 32)), (False, (16, 16, 16))])
def test_linear_replay_keeps_valid_chains(periodic, tile):
    L, start, bonds = obs.read_tuv(os.path.join(GOLD, "efpol_lin_L32_N100_s1_t0.res.gz"))
    P, N = bonds.shape
    r = Replay(L, N, P, 7, periodic=periodic, tile=tile, linear=True)
    assert r.load(start, bonds) == 0
    first = (start.copy(), bonds.copy())
    for _ in range(4):
        r.steps(25)
        rc, s2, b2 = r.export()
        assert rc == 0
        assert np.all(b2[:, -1] == 15) and not np.any(b2[:, :-1] == 15)
        e = Efpol(L, N, P, 0, pol_type=2)
        assert e.read(obs.format_tuv(L, s2, b2)) == 0 and e.check() == 0
    # monomer 0 moved (start sites changed) and the chains changed shape
    assert np.any(s2 != first[0]) and np.any(b2 != first[1])
    assert r.accepted > 0
