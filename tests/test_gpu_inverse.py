"""The inversion between the passes of the proof path's grid-wide rounds: four
lanes per value with table-driven divstep groups (k_flat_invert), against the
one-lane divstep inversion on the device.  Exact integer work: every word must
agree, including for 0, 1, 2 and p - 1."""
import pytest

import vkzg_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,seed", [(1, 3), (5, 4), (2368, 1), (20000, 2)])
def test_four_lane_inversion_matches_one_lane(n, seed):
    assert vkzg_b200.inverse_selftest(n, seed) == 0


def test_inversion_launch_timings():
    """The round inversion's launch time (microbench 17: 16 values per SM, four
    lanes each) against one lane per value (11: fixed divstep batches; 10:
    variable-time batches).  Loose bound: timings on a shared GPU vary."""
    var, one, quad = (vkzg_b200.microbench(w) for w in (10, 11, 17))
    assert var > 0 and one > 0 and quad > 0
    assert quad < 1.1 * one, (var, one, quad)
