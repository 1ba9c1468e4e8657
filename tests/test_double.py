"""Hierarchical doubling (elp_double_chains) against the reference efpol.

tests/golden/efpol_dbl_s5_t{1,100}_{in,out}.res.gz are the reference's own
dumps of a DBLSTEP=1 run: its last state at L=16, N=50 and its first state
at L=32, N=400 after DoubleLattice (cpupol/efpol_init.c:114-207).  Doubling
the first must give the second byte for byte.  After one step 18 rings
still sit on two sites, so the rebuilt-ring branch is covered; after 100
steps none do.  Host only."""
import gzip
import os

import numpy as np
import pytest

import elp
import observables as obs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("t,two_site", [(1, 18), (100, 0)])
def test_double_matches_reference_double_lattice(t, two_site):
    L, start, bonds = obs.read_tuv(os.path.join(GOLD, f"efpol_dbl_s5_t{t}_in.res.gz"))
    assert int(((bonds != 0).sum(axis=1) == 2).sum()) == two_site
    L2, s2, b2 = elp.double_chains(L, start, bonds)
    with gzip.open(os.path.join(GOLD, f"efpol_dbl_s5_t{t}_out.res.gz"), "rt") as f:
        want = f.read()
    assert elp.format_tuv(L2, s2, b2) == want


def test_double_is_a_valid_melt_in_the_oracle():
    """Every doubled ring closes and no two rings share a site (oracle check)."""
    from oracle_binding import Efpol
    L, start, bonds = obs.read_tuv(os.path.join(GOLD, "efpol_dbl_s5_t1_in.res.gz"))
    L2, s2, b2 = elp.double_chains(L, start, bonds)
    e = Efpol(L2, b2.shape[1], b2.shape[0], 0)
    assert e.read(obs.format_tuv(L2, s2, b2)) == 0 and e.check() == 0


def test_double_rejects_bad_input():
    L, start, bonds = obs.read_tuv(os.path.join(GOLD, "efpol_dbl_s5_t1_in.res.gz"))
    bad = np.array(start)
    bad[0, 0] = L
    with pytest.raises(elp.ElpError) as e:
        elp.double_chains(L, bad, bonds)
    assert e.value.status == elp.ERR_ARG
    with pytest.raises(elp.ElpError) as e:
        elp.double_chains(L, start, np.zeros((bonds.shape[0], 9000), dtype=np.uint8))   # 8N > 65536
    assert e.value.status == elp.ERR_ARG
