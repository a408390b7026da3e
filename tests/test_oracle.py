"""The CPU oracle against the consensus-spec vectors the reference ships, and
against independent forms of the same math (CPU only)."""
import hashlib
import os

import numpy as np
import pytest

from conftest import recover_inputs, random_blobs, adversarial_blobs

P_MOD = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R_MOD = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001


def test_proof_vectors(oracle, mainnet_tables, golden_proofs):
    """tests/test.cpp:55-91: every valid proof vector, byte for byte."""
    for k, name in enumerate(golden_proofs["valid_names"]):
        rc, proofs = oracle.compute_proofs(mainnet_tables, golden_proofs["valid_blobs"][k])
        assert rc == 0, name
        assert np.array_equal(proofs, golden_proofs["valid_proofs"][k]), name


def test_proof_vectors_batched(oracle, mainnet_tables, golden_proofs):
    """tests/test.cpp:94-119: all valid blobs in one call."""
    rc, proofs = oracle.compute_proofs(mainnet_tables, golden_proofs["valid_blobs"])
    assert rc == 0
    assert np.array_equal(proofs.reshape(-1, 6144), golden_proofs["valid_proofs"])


def test_cells_vectors(oracle, golden_proofs):
    """The vectors' 128 cells (skipped by the reference's test, tests/vectors.h:88-95)."""
    rc, cells = oracle.compute_cells(golden_proofs["valid_blobs"])
    assert rc == 0
    for k in range(len(golden_proofs["valid_names"])):
        digest = hashlib.sha256(cells[k * 262144:(k + 1) * 262144].tobytes()).digest()
        assert digest == golden_proofs["valid_cells_sha256"][k].tobytes()
        # the first 64 cells are the blob's own bytes (wire position p < 4096 is
        # the value at w_8192^(2 brev12(p))): the device kernel copies them
        assert np.array_equal(cells[k * 262144:k * 262144 + 131072], golden_proofs["valid_blobs"][k])


def test_coset_inverse_of_vanishing_polynomial_without_inversion():
    """The identity the device recovery uses for 1/Z on the 7-coset: the roots
    w_128^brev7(m) of the 128 cells are all the 128th roots of unity, so for
    y = 7^64 w_128^j, prod over all m of (y - root_m) = y^128 - 1 = 7^8192 - 1 and
    1/Zs(y) = prod over present m of (y - root_m) / (7^8192 - 1)."""
    w128 = pow(7, (R_MOD - 1) // 128, R_MOD)
    roots = [pow(w128, int(f"{m:07b}"[::-1], 2), R_MOD) for m in range(128)]
    assert sorted(roots) == sorted(pow(w128, k, R_MOD) for k in range(128))
    scale = pow((pow(7, 8192, R_MOD) - 1) % R_MOD, R_MOD - 2, R_MOD)
    seven64 = pow(7, 64, R_MOD)
    rng = np.random.default_rng(7)
    for trial in range(12):
        missing = set(rng.choice(128, int(rng.integers(0, 65)), replace=False).tolist())
        for c in rng.choice(128, 4, replace=False):
            y = seven64 * roots[int(c)] % R_MOD
            zs = 1
            for m in missing:
                zs = zs * (y - roots[m]) % R_MOD
            prod_present = 1
            for m in range(128):
                if m not in missing:
                    prod_present = prod_present * (y - roots[m]) % R_MOD
            assert pow(zs, R_MOD - 2, R_MOD) == prod_present * scale % R_MOD


def test_invalid_blobs(oracle, mainnet_tables, golden_proofs):
    for k, name in enumerate(golden_proofs["invalid_names"]):
        blob = golden_proofs[f"invalid_blob_{k}"]
        if blob.size != 131072:
            continue  # wrong-length cases are rejected by the caller (tests/test.cpp:57-59)
        rc, _ = oracle.compute_proofs(mainnet_tables, blob)
        assert rc == 6, name


def test_recovery_vectors(oracle, golden_recover):
    for name in golden_recover["names"]:
        full, present = recover_inputs(golden_recover, name)
        rc, out = oracle.recover_cells(full, present)
        if name + "__expected" in golden_recover.files:
            assert rc == 0, name
            assert np.array_equal(out, golden_recover[name + "__expected"]), name
        else:
            assert rc == 1, name


def test_g1fft_form_matches(oracle, mainnet_tables, golden_proofs):
    """Phase B via the split-circulant taps equals plain G1 IFFT/truncate/FFT."""
    rc, proofs = oracle.compute_proofs_g1fft(mainnet_tables, golden_proofs["valid_blobs"][4])
    assert rc == 0
    assert np.array_equal(proofs, golden_proofs["valid_proofs"][4])


def test_tau_oracle_synthetic(oracle, synthetic):
    """FK20 over tables regenerated from a synthetic setup equals [q_k(tau)]G1."""
    tau, mono, tables = synthetic
    blobs = np.concatenate([random_blobs(1, 11), adversarial_blobs()[2:3]])
    for blob in blobs:
        rc, p1 = oracle.compute_proofs(tables, blob)
        rc2, p2 = oracle.compute_proofs_tau(tau, blob)
        assert rc == 0 and rc2 == 0
        assert np.array_equal(p1, p2)


def test_recovery_roundtrip_uneven(oracle):
    """cells -> erase any >= 64 -> recover gives the cells back."""
    blobs = random_blobs(2, 3)
    rc, cells = oracle.compute_cells(blobs)
    assert rc == 0
    rng = np.random.default_rng(9)
    present = np.zeros((2, 128), np.uint8)
    for b, keep in enumerate((64, 101)):
        present[b, rng.choice(128, keep, replace=False)] = 1
    erased = cells.reshape(2, 128, 2048).copy()
    erased[present == 0] = 0xAB  # missing bytes are ignored
    rc, out = oracle.recover_cells(erased, present)
    assert rc == 0
    assert np.array_equal(out, cells)


def test_field_kats(oracle):
    rng = np.random.default_rng(1)
    for _ in range(200):
        a = int.from_bytes(rng.bytes(48), "big") % P_MOD
        b = int.from_bytes(rng.bytes(48), "big") % P_MOD
        rc, out = oracle.fp_mul(a.to_bytes(48, "big"), b.to_bytes(48, "big"))
        assert rc == 0 and int.from_bytes(out, "big") == a * b % P_MOD
        x = int.from_bytes(rng.bytes(32), "big") % R_MOD
        y = int.from_bytes(rng.bytes(32), "big") % R_MOD
        rc, out = oracle.fr_mul(x.to_bytes(32, "big"), y.to_bytes(32, "big"))
        assert rc == 0 and int.from_bytes(out, "big") == x * y % R_MOD
        if x:
            rc, out = oracle.fr_inv(x.to_bytes(32, "big"))
            assert int.from_bytes(out, "big") == pow(x, -1, R_MOD)


def test_g1_kats(oracle, mainnet_setup):
    """[tau^i]G1 points: 2*P == P + P, (a+b)P == aP + bP, r*P == infinity."""
    g = mainnet_setup[:48]
    rc, two_g = oracle.g1_mul(g, (2).to_bytes(32, "big"))
    rc2, gg = oracle.g1_add(g, g)
    assert rc == 0 and rc2 == 0 and two_g == gg
    a, b = 123456789, 987654321
    _, ag = oracle.g1_mul(mainnet_setup[48:96], a.to_bytes(32, "big"))
    _, bg = oracle.g1_mul(mainnet_setup[48:96], b.to_bytes(32, "big"))
    _, s = oracle.g1_add(ag, bg)
    _, abg = oracle.g1_mul(mainnet_setup[48:96], (a + b).to_bytes(32, "big"))
    assert s == abg
    _, inf = oracle.g1_mul(g, R_MOD.to_bytes(32, "big"))
    assert inf == bytes([0xC0]) + bytes(47)
    # G1 generator x-coordinate (compressed form of the first setup point)
    assert g[:4].hex() == "97f1d3a7"


def test_spec_vectors_dir_round_trips(tmp_path, golden_proofs, golden_recover, oracle):
    """The vectors directory written for the reference's test program holds the
    fixtures' bytes, laid out as tests/vectors.h:68-136 parses them."""
    import yaml
    from spec_vectors import write_vectors_dir
    root = write_vectors_dir(str(tmp_path), golden_proofs, golden_recover, oracle)
    names = sorted(os.listdir(root))
    assert len(names) == 17
    for k, name in enumerate(golden_proofs["valid_names"]):
        y = yaml.safe_load(open(os.path.join(root, str(name), "data.yaml")))
        assert bytes.fromhex(y["input"]["blob"][2:]) == golden_proofs["valid_blobs"][k].tobytes()
        assert len(y["output"][0]) == 128
        assert b"".join(bytes.fromhex(x[2:]) for x in y["output"][1]) == golden_proofs["valid_proofs"][k].tobytes()
    for name in golden_recover["names"]:
        y = yaml.safe_load(open(os.path.join(root, str(name), "data.yaml")))
        assert y["input"]["cell_indices"] == [int(i) for i in golden_recover[str(name) + "__indices"]]
        assert (y["output"] is None) == (str(name) + "__expected" not in golden_recover)
