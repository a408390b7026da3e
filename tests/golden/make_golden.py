"""Converts the consensus-spec vectors that jtraglia/vkzg ships (tests/vectors/*/data.yaml)
into compact binary fixtures for this repository's tests.

Run from the repository root, where a reference checkout exists:
    python tests/golden/make_golden.py <reference checkout>/tests/vectors
(or with $VKZG_REFERENCE_DIR set and no argument).

compute_cells_and_kzg_proofs.npz
    valid_names, valid_blobs [7,131072] u8, valid_proofs [7,6144] u8 (wire order, as in
    tests/vectors.h:88-95), valid_cells_sha256 [7,32] u8 (sha256 of the 128 expected cells,
    which the reference's own test skips), invalid_names, invalid_blob_<k> (raw bytes, any length).
recover_cells_and_kzg_proofs.npz
    names; per case <name>__indices (u32), <name>__cells (present cells, u8),
    and for valid cases <name>__expected (128 x 2048 B) and <name>__proofs (128 x 48 B).
"""
import hashlib
import os
import sys

import numpy as np
import yaml


def hexbytes(s):
    return bytes.fromhex(s[2:] if s.startswith("0x") else s)


def main(vec_dir, out_dir):
    cases = sorted(os.listdir(vec_dir))
    valid_names, valid_blobs, valid_proofs, valid_cells_sha = [], [], [], []
    invalid = {}
    rec = {}
    rec_names = []
    for c in cases:
        y = yaml.safe_load(open(os.path.join(vec_dir, c, "data.yaml")))
        inp, out = y["input"], y["output"]
        if c.startswith("compute_cells_and_kzg_proofs"):
            blob = hexbytes(inp["blob"])
            if out is None:
                invalid[c] = np.frombuffer(blob, dtype=np.uint8)
                continue
            cells = b"".join(hexbytes(x) for x in out[0])
            proofs = b"".join(hexbytes(x) for x in out[1])
            assert len(blob) == 131072 and len(cells) == 128 * 2048 and len(proofs) == 128 * 48
            valid_names.append(c)
            valid_blobs.append(np.frombuffer(blob, dtype=np.uint8))
            valid_proofs.append(np.frombuffer(proofs, dtype=np.uint8))
            valid_cells_sha.append(np.frombuffer(hashlib.sha256(cells).digest(), dtype=np.uint8))
        elif c.startswith("recover_cells_and_kzg_proofs"):
            idx = np.array(inp["cell_indices"], dtype=np.uint32)
            cells = b"".join(hexbytes(x) for x in inp["cells"])
            rec_names.append(c)
            rec[c + "__indices"] = idx
            rec[c + "__cells"] = np.frombuffer(cells, dtype=np.uint8)
            if out is not None:
                expected = b"".join(hexbytes(x) for x in out[0])
                proofs = b"".join(hexbytes(x) for x in out[1])
                assert len(expected) == 128 * 2048 and len(proofs) == 128 * 48
                for k, i in enumerate(idx):
                    assert expected[i * 2048:(i + 1) * 2048] == cells[k * 2048:(k + 1) * 2048]
                rec[c + "__expected"] = np.frombuffer(expected, dtype=np.uint8)
                rec[c + "__proofs"] = np.frombuffer(proofs, dtype=np.uint8)
    np.savez_compressed(
        os.path.join(out_dir, "compute_cells_and_kzg_proofs.npz"),
        valid_names=np.array(valid_names),
        valid_blobs=np.stack(valid_blobs),
        valid_proofs=np.stack(valid_proofs),
        valid_cells_sha256=np.stack(valid_cells_sha),
        invalid_names=np.array(sorted(invalid)),
        **{f"invalid_blob_{k}": invalid[n] for k, n in enumerate(sorted(invalid))},
    )
    np.savez_compressed(os.path.join(out_dir, "recover_cells_and_kzg_proofs.npz"),
                        names=np.array(rec_names), **rec)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        vec_dir = sys.argv[1]
    elif os.environ.get("VKZG_REFERENCE_DIR"):
        vec_dir = os.path.join(os.environ["VKZG_REFERENCE_DIR"], "tests", "vectors")
    else:
        sys.exit("usage: make_golden.py <reference checkout>/tests/vectors (or set VKZG_REFERENCE_DIR)")
    main(vec_dir, os.path.dirname(os.path.abspath(__file__)))
