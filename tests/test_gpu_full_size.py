"""Full-size workloads (256 + 4 adversarial proof blobs, 512-blob uneven
recovery in one launch) checked by properties that do not depend on size:
batched = one blob at a time, a seeded sample against the oracle, and
cells -> erase -> recover round trips."""
import numpy as np
import pytest

import vkzg_b200
from conftest import adversarial_blobs, random_blobs

pytestmark = pytest.mark.gpu


def test_proofs_256_plus_adversarial(oracle, mainnet_tables, monkeypatch):
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.delenv("VKZG_PLAN", raising=False)
    blobs = np.concatenate([random_blobs(256, 606), adversarial_blobs()])
    n = len(blobs)
    with vkzg_b200.Prover(max_batch_size=256) as p:
        out = np.zeros(n * 6144, np.uint8)
        assert p.compute_proofs_raw(out, blobs, n) == 0  # tunes the 256 class on its first chunk
        again = np.zeros_like(out)
        assert p.compute_proofs_raw(again, blobs, n) == 0
        assert np.array_equal(out, again)
        sample = [0, 77, 255, 256, 257, 258, 259]  # the adversarial blobs are the last four
        for b in sample:
            one = np.zeros(6144, np.uint8)
            assert p.compute_proofs_raw(one, blobs[b], 1) == 0
            assert np.array_equal(one, out[b * 6144:(b + 1) * 6144]), b
    rc, want = oracle.compute_proofs(mainnet_tables, blobs[sample])
    assert rc == 0
    for k, b in enumerate(sample):
        assert np.array_equal(out[b * 6144:(b + 1) * 6144], want[k * 6144:(k + 1) * 6144]), b


def test_uneven_recovery_512_blobs_one_launch(oracle):
    n = 512
    rng = np.random.default_rng(512)
    blobs = random_blobs(n, 707)
    with vkzg_b200.Prover(max_batch_size=n) as p:
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8).reshape(n, 128, 2048)
        present = np.zeros((n, 128), np.uint8)
        for b in range(n):
            if b % 16 == 0:
                present[b, :64] = 1
            elif b % 16 == 1:
                present[b, ::2] = 1
            else:
                present[b, rng.choice(128, int(rng.integers(64, 128)), replace=False)] = 1
        erased = cells.copy()
        erased[present == 0] = rng.integers(0, 256, size=(int((present == 0).sum()), 2048), dtype=np.uint8)
        out = np.zeros(n * 262144, np.uint8)
        assert p.recover_cells_raw(out, erased, present, n) == 0
    assert np.array_equal(out, cells.reshape(-1))
    sample = [0, 1, 2, 511]
    rc, want = oracle.recover_cells(erased[sample], present[sample])
    assert rc == 0
    assert np.array_equal(want, out.reshape(n, -1)[sample].reshape(-1))
