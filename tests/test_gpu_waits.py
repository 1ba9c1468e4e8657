"""The bounded waits of tiled launches of several steps.

Inside one launch a tile of step s waits for the tiles of step s - 1 that
overlap it (per-tile completion flags, no grid-wide barrier).  Every wait is
bounded: when it runs out, the tile is left as it is, the launch reports
through the device error flags, and the next synchronising call returns
ELP_ERR_STATE.  These tests make a wait run out on purpose, without any GPU
fault: one tile is told never to announce its first step (elp_debug_waits),
so the tiles that overlap it in the second step poll a flag that nothing
sets until their short limit is reached.
"""
import numpy as np
import pytest

import elp

pytestmark = pytest.mark.gpu
GEOM = dict(L=64, N=200, periodic=0, tile=(32, 32, 32), steps_per_launch=4)


def test_a_wait_that_runs_out_reports_and_leaves_the_context_usable():
    m = elp.Melt(seed=3, **GEOM)
    m.init_melt()
    m.run(8)
    m.sync()                                     # normal launches: no report
    m.debug_waits(polls=2000, hold_tile=0)
    m.run(4)
    with pytest.raises(elp.ElpError) as e:
        m.sync()
    assert e.value.status == elp.ERR_STATE
    assert "previous step" in str(e.value)
    with pytest.raises(elp.ElpError):
        m.accepted()                             # the count of incomplete steps is flagged too
    # a new configuration clears the report; the trajectory is the normal one
    m.debug_waits(0, -1)
    m.init_melt()
    m.run(12)
    ref = elp.Melt(seed=3, **GEOM)
    ref.init_melt()
    ref.run(12)
    wa, ra = m.state()
    wb, rb = ref.state()
    assert np.array_equal(wa, wb) and np.array_equal(ra, rb)
    assert m.check() == 0


def test_bad_tile_index_is_an_argument_error():
    m = elp.Melt(seed=5, **GEOM)
    with pytest.raises(elp.ElpError) as e:
        m.debug_waits(10, 8)                     # 8 tiles: 0..7
    assert e.value.status == elp.ERR_ARG
