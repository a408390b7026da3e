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
