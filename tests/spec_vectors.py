"""Writes the consensus-spec vectors back out as a directory of <case>/data.yaml
files, the layout the reference's own test program reads (tests/vectors.cpp:12-46,
tests/vectors.h:68-136), from this repository's fixtures in tests/golden/.

The fixtures keep each valid proof case's 128 cells as one sha256; the cells
are recomputed from the blob by the CPU oracle and must hash to that value
before they are written, so every file written holds the vector's own bytes.
"""
import hashlib
import os

import numpy as np


def _hex(b):
    return "'0x" + bytes(b).hex() + "'"


def _list(items, indent):
    pad = " " * indent
    return "".join(f"{pad}- {_hex(x)}\n" for x in items)


def write_vectors_dir(path, golden_proofs, golden_recover, oracle):
    os.makedirs(path, exist_ok=True)
    g = golden_proofs
    for k, name in enumerate(g["valid_names"]):
        blob = g["valid_blobs"][k]
        rc, cells = oracle.compute_cells(blob)
        assert rc == 0
        cells = np.asarray(cells, np.uint8).reshape(128, 2048)
        assert hashlib.sha256(cells.tobytes()).digest() == g["valid_cells_sha256"][k].tobytes(), name
        proofs = g["valid_proofs"][k].reshape(128, 48)
        text = ("input:\n  blob: " + _hex(blob) + "\noutput:\n- \n" + _list(cells, 2) + "- \n"
                + _list(proofs, 2))
        _write(path, str(name), text)
    for k, name in enumerate(g["invalid_names"]):
        _write(path, str(name), "input:\n  blob: " + _hex(g[f"invalid_blob_{k}"]) + "\noutput: null\n")
    r = golden_recover
    for name in r["names"]:
        name = str(name)
        idx = r[name + "__indices"]
        cells = r[name + "__cells"].reshape(len(idx), 2048) if len(idx) else []
        text = ("input:\n  cell_indices: [" + ", ".join(str(int(i)) for i in idx) + "]\n  cells:"
                + ("\n" + _list(cells, 2) if len(idx) else " []\n"))
        if name + "__expected" in r:
            text += ("output:\n- \n" + _list(r[name + "__expected"].reshape(128, 2048), 2) + "- \n"
                     + _list(r[name + "__proofs"].reshape(128, 48), 2))
        else:
            text += "output: null\n"
        _write(path, name, text)
    return path


def _write(root, name, text):
    d = os.path.join(root, name)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "data.yaml"), "w") as f:
        f.write(text)
