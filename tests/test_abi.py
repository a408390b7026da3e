"""libvkzg.so loads and exports every symbol include/*.h declares; the calls that
need no GPU behave like the reference's (CPU only)."""
import ctypes
import os
import re

import pytest

import vkzg_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("vkzg.h", "vkzg_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(vkzg_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = vkzg_b200.library()
    decl = declared_symbols()
    assert decl == set(vkzg_b200.EXPORTED_SYMBOLS)
    for name in decl:
        assert hasattr(lib, name), name


def test_error_strings():
    # src/vkzg.cpp:170-181
    want = {0: "ok", 1: "invalid argument", 2: "allocation failed", 3: "i/o error",
            4: "malformed trusted setup", 5: "gpu error", 6: "blob contains a non-canonical field element"}
    for code, s in want.items():
        assert vkzg_b200.error_string(code) == s
    assert vkzg_b200.error_string(99) == "unknown error"


def test_options_layout_and_default():
    assert ctypes.sizeof(vkzg_b200._Options) == 4  # Vkzg.java:137-138
    o = vkzg_b200._Options(123)
    vkzg_b200.library().vkzg_options_default(ctypes.byref(o))
    assert o.max_batch_size == 0
    vkzg_b200.library().vkzg_options_default(None)  # NULL-safe


def test_null_prover_contract():
    L = vkzg_b200.library()
    assert L.vkzg_prover_device_name(None) == b""
    assert L.vkzg_prover_gpu_core_count(None) == 0
    L.vkzg_prover_free(None)
    buf = ctypes.create_string_buffer(131072)
    out = ctypes.create_string_buffer(6144)
    # null prover / blobs / proofs -> BADARGS (tests/test.cpp:127-131), before any device work
    assert L.vkzg_compute_proofs_batch(None, out, buf, 1) == 1
    assert L.vkzg_recover_cells_batch(None, out, buf, buf, 1) == 1
    assert L.vkzg_prover_new(None, None) == 1
    assert L.vkzg_b200_write_tables(None, b"/dev/null") == 1
