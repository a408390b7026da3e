"""Plans 3-4 with each phase's grid-wide rounds in one cooperative launch
(grid barriers between the passes; $VKZG_COOP=1) against the same plans in
three launches per round (the default), and the grid barrier's bounded wait: a barrier that can never complete
gives up after its poll limit, sets the failure flag and marks the error words,
and the launch ends."""
import time

import numpy as np
import pytest

import vkzg_b200
from conftest import random_blobs

pytestmark = pytest.mark.gpu


def test_grid_barrier_completes():
    passed, flag, marked = vkzg_b200.grid_sync_selftest(0, 1 << 20, 5)
    blocks = passed // 5
    assert passed == 5 * blocks and blocks >= 2
    assert flag == 0 and marked == 0


def test_grid_barrier_wait_runs_out():
    t0 = time.perf_counter()
    passed, flag, marked = vkzg_b200.grid_sync_selftest(1, 20000, 3)
    assert time.perf_counter() - t0 < 30
    assert passed == 0  # no barrier can complete: it waits for a block that does not exist
    assert flag == 1 and marked == 8
    # the device is still usable afterwards
    passed, flag, marked = vkzg_b200.grid_sync_selftest(0, 1 << 20, 2)
    assert flag == 0 and passed > 0


@pytest.mark.parametrize("plan", [3, 4])
def test_cooperative_rounds_match_round_launches(monkeypatch, plan):
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.setenv("VKZG_PLAN", str(plan))
    monkeypatch.setenv("VKZG_COMB_BITS", "10")
    blobs = random_blobs(40, 808)
    outs, launches = {}, {}
    for coop in ("1", "0"):
        monkeypatch.setenv("VKZG_COOP", coop)
        with vkzg_b200.Prover(max_batch_size=40) as p:
            out = np.zeros(40 * 6144, np.uint8)
            assert p.compute_proofs_raw(out, blobs, 40) == 0  # captures the pipeline's graph
            k0 = vkzg_b200.kernel_launches()
            assert p.compute_proofs_raw(out, blobs, 40) == 0
            launches[coop] = vkzg_b200.kernel_launches() - k0
            outs[coop] = out
    assert np.array_equal(outs["1"], outs["0"])
    assert launches["1"] <= 10 < launches["0"]
