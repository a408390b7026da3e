"""ctypes wrapper around oracle/_build/liboracle_vkzg.so (TEST INFRASTRUCTURE ONLY)."""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "liboracle_vkzg.so")

BLOB_BYTES = 131072
PROOFS_BYTES = 128 * 48
CELLS_BYTES = 128 * 2048


def build(force=False):
    """Compiles the oracle with its Makefile (gcc)."""
    src = os.path.join(_HERE, "vkzg_oracle.c")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


def _buf(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(ctypes.c_void_p)


class OracleTables:
    def __init__(self, lib, handle):
        self._lib = lib
        self.handle = handle

    def __del__(self):
        if getattr(self, "handle", None):
            self._lib.orc_tables_free(self.handle)
            self.handle = None

    def serialize(self):
        n = self._lib.orc_tables_file_size(self.handle)
        out = np.zeros(n, dtype=np.uint8)
        rc = self._lib.orc_tables_serialize(self.handle, out.ctypes.data_as(ctypes.c_void_p), n)
        assert rc == 0
        return out

    def write(self, path):
        rc = self._lib.orc_tables_write(self.handle, path.encode())
        if rc:
            raise OSError(f"orc_tables_write -> {rc}")

    def position_words(self):
        p = self._lib.orc_tables_position(self.handle)
        return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_uint32)), shape=(262144 * 24,)).copy()


class Oracle:
    def __init__(self):
        self.lib = ctypes.CDLL(build())
        L = self.lib
        vp, sz, i32, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint64
        L.orc_tables_from_setup.argtypes = [ctypes.POINTER(vp), vp, i32]
        L.orc_tables_load.argtypes = [ctypes.POINTER(vp), ctypes.c_char_p]
        L.orc_tables_write.argtypes = [vp, ctypes.c_char_p]
        L.orc_tables_free.argtypes = [vp]
        L.orc_tables_position.argtypes = [vp]
        L.orc_tables_position.restype = vp
        L.orc_tables_file_size.argtypes = [vp]
        L.orc_tables_file_size.restype = sz
        L.orc_tables_serialize.argtypes = [vp, vp, sz]
        L.orc_compute_proofs.argtypes = [vp, vp, vp, sz, i32]
        L.orc_compute_proofs_g1fft.argtypes = [vp, vp, vp]
        L.orc_compute_proofs_tau.argtypes = [vp, vp, vp]
        L.orc_proof_stages.argtypes = [vp, vp, vp, vp, vp, vp]
        L.orc_recover_cells.argtypes = [vp, vp, vp, sz, i32]
        L.orc_compute_cells.argtypes = [vp, vp, sz, i32]
        L.orc_synthetic_setup.argtypes = [u64, vp, vp, vp]
        for name in ("orc_fp_mul_be", "orc_fr_mul_be"):
            getattr(L, name).argtypes = [vp, vp, vp]
        L.orc_fr_inv_be.argtypes = [vp, vp]
        L.orc_fp_to_mont.argtypes = [vp, vp]
        L.orc_fp_from_mont.argtypes = [vp, vp]
        L.orc_fr_to_mont.argtypes = [vp, vp]
        L.orc_fr_from_mont.argtypes = [vp, vp]
        L.orc_g1_decompress.argtypes = [vp, vp]
        L.orc_g1_compress.argtypes = [vp, vp]
        L.orc_g1_mul.argtypes = [vp, vp, vp]
        L.orc_g1_add.argtypes = [vp, vp, vp]

    # ---------------------------------------------------------------- tables
    def tables_from_setup(self, g1_monomial_compressed, nthreads=None):
        h = ctypes.c_void_p()
        a, p = _buf(np.frombuffer(bytes(g1_monomial_compressed), dtype=np.uint8))
        assert a.size == 4096 * 48
        rc = self.lib.orc_tables_from_setup(ctypes.byref(h), p, nthreads or os.cpu_count() or 1)
        if rc:
            raise ValueError(f"orc_tables_from_setup -> {rc}")
        return OracleTables(self.lib, h)

    def tables_load(self, path):
        h = ctypes.c_void_p()
        rc = self.lib.orc_tables_load(ctypes.byref(h), path.encode())
        if rc:
            raise OSError(f"orc_tables_load -> {rc}")
        return OracleTables(self.lib, h)

    # ---------------------------------------------------------------- proofs
    def compute_proofs(self, tables, blobs, nthreads=None):
        """Returns (rc, proofs bytes)."""
        b, bp = _buf(np.frombuffer(bytes(blobs), dtype=np.uint8) if not isinstance(blobs, np.ndarray) else blobs.reshape(-1))
        n = b.size // BLOB_BYTES
        out = np.zeros(n * PROOFS_BYTES, dtype=np.uint8)
        rc = self.lib.orc_compute_proofs(tables.handle, out.ctypes.data_as(ctypes.c_void_p), bp, n,
                                         nthreads or os.cpu_count() or 1)
        return rc, out

    def compute_proofs_g1fft(self, tables, blob):
        b, bp = _buf(np.frombuffer(bytes(blob), dtype=np.uint8))
        out = np.zeros(PROOFS_BYTES, dtype=np.uint8)
        rc = self.lib.orc_compute_proofs_g1fft(tables.handle, out.ctypes.data_as(ctypes.c_void_p), bp)
        return rc, out

    def compute_proofs_tau(self, tau_be, blob):
        t, tp = _buf(np.frombuffer(bytes(tau_be), dtype=np.uint8))
        b, bp = _buf(np.frombuffer(bytes(blob), dtype=np.uint8))
        out = np.zeros(PROOFS_BYTES, dtype=np.uint8)
        rc = self.lib.orc_compute_proofs_tau(tp, out.ctypes.data_as(ctypes.c_void_p), bp)
        return rc, out

    def proof_stages(self, tables, blob):
        b, bp = _buf(np.frombuffer(bytes(blob), dtype=np.uint8))
        f = np.zeros(4096 * 32, np.uint8)
        circ = np.zeros(128 * 64 * 32, np.uint8)
        u = np.zeros(128 * 96, np.uint8)
        nat = np.zeros(128 * 96, np.uint8)
        rc = self.lib.orc_proof_stages(tables.handle, bp, *(x.ctypes.data_as(ctypes.c_void_p) for x in (f, circ, u, nat)))
        return rc, dict(coeffs=f, circ=circ, u=u, proofs_nat=nat)

    # -------------------------------------------------------------- recovery
    def recover_cells(self, cells, present, nthreads=None):
        c, cp = _buf(cells.reshape(-1) if isinstance(cells, np.ndarray) else np.frombuffer(bytes(cells), np.uint8))
        pr, pp = _buf(present.reshape(-1) if isinstance(present, np.ndarray) else np.frombuffer(bytes(present), np.uint8))
        n = pr.size // 128
        out = np.zeros(n * CELLS_BYTES, dtype=np.uint8)
        rc = self.lib.orc_recover_cells(out.ctypes.data_as(ctypes.c_void_p), cp, pp, n, nthreads or os.cpu_count() or 1)
        return rc, out

    def compute_cells(self, blobs, nthreads=None):
        b, bp = _buf(blobs.reshape(-1) if isinstance(blobs, np.ndarray) else np.frombuffer(bytes(blobs), np.uint8))
        n = b.size // BLOB_BYTES
        out = np.zeros(n * CELLS_BYTES, dtype=np.uint8)
        rc = self.lib.orc_compute_cells(out.ctypes.data_as(ctypes.c_void_p), bp, n, nthreads or os.cpu_count() or 1)
        return rc, out

    # ----------------------------------------------------------------- setup
    def synthetic_setup(self, seed, lagrange=False):
        tau = np.zeros(32, np.uint8)
        mono = np.zeros(4096 * 48, np.uint8)
        lag = np.zeros(4096 * 48, np.uint8) if lagrange else None
        rc = self.lib.orc_synthetic_setup(seed, tau.ctypes.data_as(ctypes.c_void_p),
                                          mono.ctypes.data_as(ctypes.c_void_p),
                                          lag.ctypes.data_as(ctypes.c_void_p) if lag is not None else None)
        assert rc == 0
        return tau.tobytes(), mono.tobytes(), (lag.tobytes() if lag is not None else None)

    # ------------------------------------------------------------- primitives
    def _bin(self, fn, a, b, n):
        out = np.zeros(n, np.uint8)
        aa, ap = _buf(np.frombuffer(a, np.uint8))
        bb, bp = _buf(np.frombuffer(b, np.uint8))
        rc = fn(ap, bp, out.ctypes.data_as(ctypes.c_void_p))
        return rc, out.tobytes()

    def fp_mul(self, a, b):
        return self._bin(self.lib.orc_fp_mul_be, a, b, 48)

    def fr_mul(self, a, b):
        return self._bin(self.lib.orc_fr_mul_be, a, b, 32)

    def g1_mul(self, p48, k32):
        return self._bin(self.lib.orc_g1_mul, p48, k32, 48)

    def g1_add(self, p48, q48):
        return self._bin(self.lib.orc_g1_add, p48, q48, 48)

    def g1_decompress(self, p48):
        out = np.zeros(96, np.uint8)
        a, ap = _buf(np.frombuffer(p48, np.uint8))
        rc = self.lib.orc_g1_decompress(ap, out.ctypes.data_as(ctypes.c_void_p))
        return rc, out.tobytes()

    def fr_inv(self, a):
        out = np.zeros(32, np.uint8)
        aa, ap = _buf(np.frombuffer(a, np.uint8))
        rc = self.lib.orc_fr_inv_be(ap, out.ctypes.data_as(ctypes.c_void_p))
        return rc, out.tobytes()
