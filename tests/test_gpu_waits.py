"""The bounded grid-barrier waits of tiled launches of several steps.

Between two steps the CTAs of a cooperative launch meet at a grid barrier.
Every wait there is bounded: when it runs out, the launch stops, reports
through the device error flags, and the next synchronising call returns
ELP_ERR_STATE.  This test makes the wait run out on purpose, without any GPU
fault: one CTA is told never to arrive (elp_debug_waits), so every CTA polls
a count that never reaches its target until a short limit is reached.
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
    m.debug_waits(polls=2000, hold_block=0)
    m.run(4)
    with pytest.raises(elp.ElpError) as e:
        m.sync()
    assert e.value.status == elp.ERR_STATE
    assert "grid barrier" in str(e.value)
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


def test_bad_block_index_is_an_argument_error():
    m = elp.Melt(seed=5, **GEOM)
    with pytest.raises(elp.ElpError) as e:
        m.debug_waits(10, 8)                     # 8 tiles, 8 CTAs: 0..7
    assert e.value.status == elp.ERR_ARG
