import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


class Golden(dict):
    """Every array of an .npz fixture, read once (an NpzFile decompresses on each
    access and must not be shared between threads)."""

    def __init__(self, path):
        with np.load(path) as z:
            super().__init__({k: z[k] for k in z.files})

    @property
    def files(self):
        return list(self.keys())


@pytest.fixture(scope="session")
def golden_proofs():
    return Golden(os.path.join(GOLDEN, "compute_cells_and_kzg_proofs.npz"))


@pytest.fixture(scope="session")
def golden_recover():
    return Golden(os.path.join(GOLDEN, "recover_cells_and_kzg_proofs.npz"))


@pytest.fixture(scope="session")
def mainnet_setup():
    with open(os.path.join(ROOT, "vkzg_b200", "data", "trusted_setup_g1_monomial.bin"), "rb") as f:
        return f.read()


@pytest.fixture(scope="session")
def mainnet_tables(oracle, mainnet_setup):
    return oracle.tables_from_setup(mainnet_setup)


@pytest.fixture(scope="session")
def synthetic(oracle):
    """Seeded synthetic setup: (tau, monomial setup, oracle tables)."""
    tau, mono, _ = oracle.synthetic_setup(0x7594)
    return tau, mono, oracle.tables_from_setup(mono)


def recover_inputs(golden_recover, name):
    """Full 128-cell array and presence mask for one recovery vector
    (tests/test.cpp:209-218 builds the same)."""
    idx = golden_recover[name + "__indices"]
    cells = golden_recover[name + "__cells"]
    full = np.zeros(128 * 2048, np.uint8)
    present = np.zeros(128, np.uint8)
    for k, i in enumerate(idx):
        full[i * 2048:(i + 1) * 2048] = cells[k * 2048:(k + 1) * 2048]
        present[i] = 1
    return full, present


R_MOD = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


def random_blobs(n, seed):
    """n blobs of field elements uniform in [0, r), 32-byte big-endian (rejection-sampled)."""
    rng = np.random.default_rng(seed)
    r_be = np.frombuffer(R_MOD.to_bytes(32, "big"), np.uint8).astype(np.int16)
    out = np.empty((n * 4096, 32), np.uint8)
    filled = 0
    while filled < out.shape[0]:
        cand = rng.integers(0, 256, size=(max(1024, 2 * (out.shape[0] - filled)), 32), dtype=np.uint8)
        cand[:, 0] &= 0x7F
        diff = cand.astype(np.int16) - r_be
        first = np.argmax(diff != 0, axis=1)
        good = cand[diff[np.arange(len(cand)), first] < 0]
        take = min(len(good), out.shape[0] - filled)
        out[filled:filled + take] = good[:take]
        filled += take
    return out.reshape(n, 131072)


def adversarial_blobs():
    """all-zero, all r-1, a single nonzero element, alternating 0 / r-1."""
    rm1 = (R_MOD - 1).to_bytes(32, "big")
    zero = bytes(32)
    one = (1).to_bytes(32, "big")
    blobs = [zero * 4096, rm1 * 4096, zero * 1234 + one + zero * (4096 - 1235),
             b"".join(zero if i % 2 == 0 else rm1 for i in range(4096))]
    return np.frombuffer(b"".join(blobs), np.uint8).reshape(4, 131072).copy()
