"""vkzg on one NVIDIA B200: EIP-7594 cell KZG proofs and cell recovery.

The product is libvkzg.so (C ABI of include/vkzg.h, hand-written CUDA for
sm_100a).  This module loads it with ctypes and mirrors the reference's Java
binding (bindings/java/src/main/java/vkzg/Vkzg.java): a global prover opened
with init(), computeCellKzgProofsBatch / recoverCellsBatch taking packed byte
buffers, VkzgException(code, message) on any nonzero status.  Prover is the
same interface as an object, for callers that want more than one.

There is no CPU fallback: if libvkzg.so is missing or the GPU is unusable,
every entry point raises.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvkzg.so")

FIELD_ELEMENTS_PER_BLOB = 4096
BYTES_PER_FIELD_ELEMENT = 32
BYTES_PER_BLOB = FIELD_ELEMENTS_PER_BLOB * BYTES_PER_FIELD_ELEMENT
CELL_PROOFS_PER_BLOB = 128
BYTES_PER_PROOF = 48
FIELD_ELEMENTS_PER_CELL = 64
BYTES_PER_CELL = FIELD_ELEMENTS_PER_CELL * BYTES_PER_FIELD_ELEMENT
BYTES_PER_EXT_BLOB = CELL_PROOFS_PER_BLOB * BYTES_PER_CELL

OK, ERR_BADARGS, ERR_MALLOC, ERR_IO, ERR_SETUP, ERR_GPU, ERR_INVALID_BLOB = range(7)
PENDING = 7  # VKZG_B200_PENDING: a server wait timed out, the request is still in flight

# every symbol declared in include/vkzg.h and include/vkzg_b200.h
PLANS = 5  # VKZG_B200_PLANS

EXPORTED_SYMBOLS = (
    "vkzg_error_string", "vkzg_options_default", "vkzg_prover_new", "vkzg_prover_free",
    "vkzg_prover_device_name", "vkzg_prover_gpu_core_count", "vkzg_compute_proofs_batch",
    "vkzg_recover_cells_batch",
    "vkzg_b200_write_tables", "vkzg_b200_prover_tables_source", "vkzg_b200_set_stage_timing",
    "vkzg_b200_last_stage_times", "vkzg_b200_stage_name", "vkzg_b200_compute_proofs_device",
    "vkzg_b200_recover_cells_device", "vkzg_b200_microbench", "vkzg_b200_recover_cells_device_noalloc",
    "vkzg_b200_bucket_sums_selftest", "vkzg_b200_compute_cells_batch", "vkzg_b200_compute_cells_and_proofs_batch",
    "vkzg_b200_autotune", "vkzg_b200_tuning_table", "vkzg_b200_recover_cells_and_proofs_batch",
    "vkzg_b200_server_options_default", "vkzg_b200_server_new", "vkzg_b200_server_free",
    "vkzg_b200_server_submit_proofs", "vkzg_b200_server_submit_recovery", "vkzg_b200_server_wait",
    "vkzg_b200_server_stats", "vkzg_b200_kernel_launches", "vkzg_b200_digit_table",
    "vkzg_b200_tree_sums_selftest", "vkzg_b200_window_trials", "vkzg_b200_prover_device_bytes",
    "vkzg_b200_grid_sync_selftest",
    "vkzg_b200_inverse_selftest",
)
NOALLOC_MAX_BLOBS = 16  # VKZG_B200_NOALLOC_MAX_BLOBS


class VkzgException(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class _Options(ctypes.Structure):
    _fields_ = [("max_batch_size", ctypes.c_uint32)]


class _ServerOptions(ctypes.Structure):
    _fields_ = [("max_blobs_per_batch", ctypes.c_uint32), ("lanes", ctypes.c_uint32),
                ("hbm_budget_bytes", ctypes.c_uint64), ("table_budget_bytes", ctypes.c_uint64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("blobs", ctypes.c_uint64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("p999_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("seconds", ctypes.c_double), ("deferrals", ctypes.c_uint64),
                ("peak_in_flight_bytes", ctypes.c_uint64), ("resident_bytes", ctypes.c_uint64),
                ("proof_bytes_per_blob", ctypes.c_uint64), ("recover_bytes_per_blob", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_lib_lock = threading.Lock()


def library():
    """Loads libvkzg.so (raises OSError when it has not been built)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(f"{LIB_PATH} not built; run python -m vkzg_b200.build")
            L = ctypes.CDLL(LIB_PATH)
            vp, u8p = ctypes.c_void_p, ctypes.c_void_p
            L.vkzg_error_string.argtypes = [ctypes.c_int]
            L.vkzg_error_string.restype = ctypes.c_char_p
            L.vkzg_options_default.argtypes = [ctypes.POINTER(_Options)]
            L.vkzg_options_default.restype = None
            L.vkzg_prover_new.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_Options)]
            L.vkzg_prover_new.restype = ctypes.c_int
            L.vkzg_prover_free.argtypes = [vp]
            L.vkzg_prover_free.restype = None
            L.vkzg_prover_device_name.argtypes = [vp]
            L.vkzg_prover_device_name.restype = ctypes.c_char_p
            L.vkzg_prover_gpu_core_count.argtypes = [vp]
            L.vkzg_prover_gpu_core_count.restype = ctypes.c_uint32
            L.vkzg_compute_proofs_batch.argtypes = [vp, u8p, u8p, ctypes.c_size_t]
            L.vkzg_compute_proofs_batch.restype = ctypes.c_int
            L.vkzg_recover_cells_batch.argtypes = [vp, u8p, u8p, u8p, ctypes.c_size_t]
            L.vkzg_recover_cells_batch.restype = ctypes.c_int
            L.vkzg_b200_write_tables.argtypes = [u8p, ctypes.c_char_p]
            L.vkzg_b200_write_tables.restype = ctypes.c_int
            L.vkzg_b200_prover_tables_source.argtypes = [vp]
            L.vkzg_b200_prover_tables_source.restype = ctypes.c_char_p
            L.vkzg_b200_set_stage_timing.argtypes = [vp, ctypes.c_int]
            L.vkzg_b200_set_stage_timing.restype = None
            L.vkzg_b200_last_stage_times.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
            L.vkzg_b200_last_stage_times.restype = ctypes.c_int
            L.vkzg_b200_stage_name.argtypes = [ctypes.c_int, ctypes.c_int]
            L.vkzg_b200_stage_name.restype = ctypes.c_char_p
            L.vkzg_b200_compute_proofs_device.argtypes = [vp, vp, vp, vp, ctypes.c_size_t, vp]
            L.vkzg_b200_compute_proofs_device.restype = ctypes.c_int
            L.vkzg_b200_recover_cells_device.argtypes = [vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
            L.vkzg_b200_recover_cells_device.restype = ctypes.c_int
            L.vkzg_b200_microbench.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            L.vkzg_b200_microbench.restype = ctypes.c_int
            L.vkzg_b200_recover_cells_device_noalloc.argtypes = [vp, vp, vp, vp, vp, ctypes.c_size_t, vp]
            L.vkzg_b200_recover_cells_device_noalloc.restype = ctypes.c_int
            L.vkzg_b200_bucket_sums_selftest.argtypes = [vp, vp, ctypes.c_size_t, vp]
            L.vkzg_b200_bucket_sums_selftest.restype = ctypes.c_int
            L.vkzg_b200_compute_cells_batch.argtypes = [vp, vp, vp, ctypes.c_size_t]
            L.vkzg_b200_compute_cells_batch.restype = ctypes.c_int
            L.vkzg_b200_compute_cells_and_proofs_batch.argtypes = [vp, vp, vp, vp, ctypes.c_size_t]
            L.vkzg_b200_compute_cells_and_proofs_batch.restype = ctypes.c_int
            L.vkzg_b200_autotune.argtypes = [vp, ctypes.c_uint32]
            L.vkzg_b200_autotune.restype = ctypes.c_int
            L.vkzg_b200_tuning_table.argtypes = [vp, vp, vp, vp, ctypes.c_int]
            L.vkzg_b200_tuning_table.restype = ctypes.c_int
            L.vkzg_b200_recover_cells_and_proofs_batch.argtypes = [vp, vp, vp, vp, vp, ctypes.c_size_t]
            L.vkzg_b200_recover_cells_and_proofs_batch.restype = ctypes.c_int
            L.vkzg_b200_server_options_default.argtypes = [ctypes.POINTER(_ServerOptions)]
            L.vkzg_b200_server_options_default.restype = None
            L.vkzg_b200_server_new.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_ServerOptions)]
            L.vkzg_b200_server_new.restype = ctypes.c_int
            L.vkzg_b200_server_free.argtypes = [vp]
            L.vkzg_b200_server_free.restype = None
            L.vkzg_b200_server_submit_proofs.argtypes = [vp, vp, vp, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint64)]
            L.vkzg_b200_server_submit_proofs.restype = ctypes.c_int
            L.vkzg_b200_server_submit_recovery.argtypes = [vp, vp, vp, vp, ctypes.c_size_t,
                                                           ctypes.POINTER(ctypes.c_uint64)]
            L.vkzg_b200_server_submit_recovery.restype = ctypes.c_int
            L.vkzg_b200_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_int64]
            L.vkzg_b200_server_wait.restype = ctypes.c_int
            L.vkzg_b200_server_stats.argtypes = [vp, ctypes.POINTER(ServerStats), ctypes.c_int]
            L.vkzg_b200_server_stats.restype = ctypes.c_int
            L.vkzg_b200_tree_sums_selftest.argtypes = [vp, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, vp,
                                                       ctypes.POINTER(ctypes.c_double)]
            L.vkzg_b200_tree_sums_selftest.restype = ctypes.c_int
            L.vkzg_b200_digit_table.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)]
            L.vkzg_b200_digit_table.restype = ctypes.c_int
            L.vkzg_b200_window_trials.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, ctypes.c_int]
            L.vkzg_b200_window_trials.restype = ctypes.c_int
            L.vkzg_b200_prover_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64),
                                                        ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
            L.vkzg_b200_prover_device_bytes.restype = None
            u32p = ctypes.POINTER(ctypes.c_uint32)
            L.vkzg_b200_grid_sync_selftest.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, u32p, u32p, u32p]
            L.vkzg_b200_grid_sync_selftest.restype = ctypes.c_int
            L.vkzg_b200_inverse_selftest.argtypes = [ctypes.c_int, ctypes.c_uint32, u32p]
            L.vkzg_b200_inverse_selftest.restype = ctypes.c_int
            L.vkzg_b200_kernel_launches.argtypes = []
            L.vkzg_b200_kernel_launches.restype = ctypes.c_uint64
            _lib = L
    return _lib


def error_string(code):
    return library().vkzg_error_string(code).decode()


def _check(rc):
    if rc != OK:
        raise VkzgException(rc, error_string(rc))


def _ptr(buf):
    """Address of a bytes-like / numpy / ctypes buffer without copying when possible."""
    if buf is None:
        return None
    if hasattr(buf, "ctypes"):  # numpy
        return buf.ctypes.data_as(ctypes.c_void_p)
    if isinstance(buf, (bytearray, memoryview)):
        mv = memoryview(buf)
        if mv.readonly:
            return ctypes.cast(ctypes.c_char_p(bytes(mv)), ctypes.c_void_p)
        return ctypes.addressof((ctypes.c_char * mv.nbytes).from_buffer(mv))
    if isinstance(buf, bytes):
        return ctypes.cast(ctypes.c_char_p(buf), ctypes.c_void_p)
    if isinstance(buf, int):
        return ctypes.c_void_p(buf)
    return ctypes.cast(buf, ctypes.c_void_p)


class Prover:
    """One vkzg_prover (a CUDA stream, device-resident setup tables, a working set)."""

    def __init__(self, max_batch_size=0):
        L = library()
        opts = _Options()
        L.vkzg_options_default(ctypes.byref(opts))
        if max_batch_size:
            opts.max_batch_size = int(max_batch_size)
        h = ctypes.c_void_p()
        _check(L.vkzg_prover_new(ctypes.byref(h), ctypes.byref(opts)))
        self._h = h
        self._lib = L

    def close(self):
        if getattr(self, "_h", None):
            self._lib.vkzg_prover_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def device_name(self):
        return self._lib.vkzg_prover_device_name(self._h).decode()

    def gpu_core_count(self):
        return int(self._lib.vkzg_prover_gpu_core_count(self._h))

    def tables_source(self):
        return self._lib.vkzg_b200_prover_tables_source(self._h).decode()

    def compute_proofs_raw(self, proofs_out, blobs, n):
        """C-ABI call on caller-owned buffers (numpy arrays or addresses); returns the status."""
        return self._lib.vkzg_compute_proofs_batch(self._h, _ptr(proofs_out), _ptr(blobs), n)

    def recover_cells_raw(self, cells_out, cells, present, n):
        return self._lib.vkzg_recover_cells_batch(self._h, _ptr(cells_out), _ptr(cells), _ptr(present), n)

    def compute_cells_raw(self, cells_out, blobs, n):
        """vkzg_b200_compute_cells_batch on caller-owned buffers; returns the status."""
        return self._lib.vkzg_b200_compute_cells_batch(self._h, _ptr(cells_out), _ptr(blobs), n)

    def compute_cells_and_proofs_raw(self, cells_out, proofs_out, blobs, n):
        return self._lib.vkzg_b200_compute_cells_and_proofs_batch(self._h, _ptr(cells_out), _ptr(proofs_out),
                                                                  _ptr(blobs), n)

    def recover_cells_and_proofs_raw(self, cells_out, proofs_out, cells, present, n):
        return self._lib.vkzg_b200_recover_cells_and_proofs_batch(self._h, _ptr(cells_out), _ptr(proofs_out),
                                                                  _ptr(cells), _ptr(present), n)

    def compute_cell_kzg_proofs_batch(self, blobs, blob_count):
        """Vkzg.computeCellKzgProofsBatch (Vkzg.java:204-229)."""
        if len(blobs) != blob_count * BYTES_PER_BLOB:
            raise ValueError(f"blobs length must be blob_count * {BYTES_PER_BLOB}")
        out = bytearray(blob_count * CELL_PROOFS_PER_BLOB * BYTES_PER_PROOF)
        src = bytes(blobs)
        _check(self._lib.vkzg_compute_proofs_batch(self._h, _ptr(out) if out else None, _ptr(src), blob_count))
        return bytes(out)

    def recover_cells_batch(self, cells, cell_present, blob_count):
        """Vkzg.recoverCellsBatch (Vkzg.java:248-281)."""
        if len(cells) != blob_count * BYTES_PER_EXT_BLOB:
            raise ValueError(f"cells length must be blob_count * {BYTES_PER_EXT_BLOB}")
        if len(cell_present) != blob_count * CELL_PROOFS_PER_BLOB:
            raise ValueError(f"cell_present length must be blob_count * {CELL_PROOFS_PER_BLOB}")
        out = bytearray(len(cells))
        c, pr = bytes(cells), bytes(cell_present)
        _check(self._lib.vkzg_recover_cells_batch(self._h, _ptr(out) if out else None, _ptr(c), _ptr(pr),
                                                  blob_count))
        return bytes(out)

    def compute_proofs_device(self, d_proofs, d_blobs, d_err, n, stream=None):
        """Device pointers (ints); enqueued on `stream` (cudaStream_t as int, None = default stream)."""
        return self._lib.vkzg_b200_compute_proofs_device(self._h, d_proofs, d_blobs, d_err, n, stream)

    def recover_cells_device(self, d_out, d_cells, d_present, d_err, n, stream=None):
        return self._lib.vkzg_b200_recover_cells_device(self._h, d_out, d_cells, d_present, d_err, n, stream)

    def recover_cells_device_noalloc(self, d_out, d_cells, d_present, d_err, n, stream=None):
        """Allocation-free recovery on caller-owned device buffers (at most NOALLOC_MAX_BLOBS blobs);
        the kernel keeps its working state in shared memory and uses no scratch."""
        return self._lib.vkzg_b200_recover_cells_device_noalloc(self._h, d_out, d_cells, d_present, d_err, n,
                                                                stream)

    def compute_cells_batch(self, blobs, blob_count):
        """The 128 cells of each blob (2x Reed-Solomon extension), wire order."""
        if len(blobs) != blob_count * BYTES_PER_BLOB:
            raise ValueError(f"blobs length must be blob_count * {BYTES_PER_BLOB}")
        out = bytearray(max(1, blob_count * BYTES_PER_EXT_BLOB))
        src = bytes(blobs) or b"\0"
        _check(self._lib.vkzg_b200_compute_cells_batch(self._h, _ptr(out), _ptr(src), blob_count))
        return bytes(out[:blob_count * BYTES_PER_EXT_BLOB])

    def compute_cells_and_kzg_proofs_batch(self, blobs, blob_count):
        """(cells, proofs) of each blob: the consensus specs' compute_cells_and_kzg_proofs."""
        if len(blobs) != blob_count * BYTES_PER_BLOB:
            raise ValueError(f"blobs length must be blob_count * {BYTES_PER_BLOB}")
        cells = bytearray(max(1, blob_count * BYTES_PER_EXT_BLOB))
        proofs = bytearray(max(1, blob_count * CELL_PROOFS_PER_BLOB * BYTES_PER_PROOF))
        src = bytes(blobs) or b"\0"
        _check(self._lib.vkzg_b200_compute_cells_and_proofs_batch(self._h, _ptr(cells), _ptr(proofs), _ptr(src),
                                                                  blob_count))
        return (bytes(cells[:blob_count * BYTES_PER_EXT_BLOB]),
                bytes(proofs[:blob_count * CELL_PROOFS_PER_BLOB * BYTES_PER_PROOF]))

    def recover_cells_and_kzg_proofs_batch(self, cells, cell_present, blob_count):
        """(cells, proofs): recovery, then the proofs of the recovered blob (recover_cells_and_kzg_proofs)."""
        if len(cells) != blob_count * BYTES_PER_EXT_BLOB or len(cell_present) != blob_count * CELL_PROOFS_PER_BLOB:
            raise ValueError("cells / cell_present length")
        out = bytearray(max(1, len(cells)))
        proofs = bytearray(max(1, blob_count * CELL_PROOFS_PER_BLOB * BYTES_PER_PROOF))
        c, pr = bytes(cells) or b"\0", bytes(cell_present) or b"\0"
        _check(self._lib.vkzg_b200_recover_cells_and_proofs_batch(self._h, _ptr(out), _ptr(proofs), _ptr(c), _ptr(pr),
                                                                  blob_count))
        return bytes(out[:len(cells)]), bytes(proofs[:blob_count * CELL_PROOFS_PER_BLOB * BYTES_PER_PROOF])

    def autotune(self, max_blobs=0):
        """Times the proof plans for every power-of-two size class up to max_blobs."""
        _check(self._lib.vkzg_b200_autotune(self._h, int(max_blobs)))
        return self.tuning_table()

    def tuning_table(self):
        """{size_class: (plan, (ms of plan 0, ..., ms of plan PLANS-1))}, -1 for plans not timed."""
        cap = 32
        sc = (ctypes.c_uint32 * cap)()
        pl = (ctypes.c_int * cap)()
        ms = (ctypes.c_double * (PLANS * cap))()
        n = self._lib.vkzg_b200_tuning_table(self._h, sc, pl, ms, cap)
        return {int(sc[i]): (int(pl[i]), tuple(ms[PLANS * i:PLANS * i + PLANS])) for i in range(min(n, cap))}

    def digit_table(self):
        """(windows per scalar D, build ms, bytes) of plan 3's digit table, or None
        before it is built (comb_windows(D) gives the window widths)."""
        ms = ctypes.c_double()
        nb = ctypes.c_uint64()
        c = self._lib.vkzg_b200_digit_table(self._h, ctypes.byref(ms), ctypes.byref(nb))
        return (c, ms.value, nb.value) if c else None

    def window_trials(self, size_class):
        """The digit tables the tuner timed for a size class:
        [(windows per scalar D, table bytes, build ms, proof-chunk ms), ...]."""
        cap = 8
        c = (ctypes.c_int * cap)()
        nb = (ctypes.c_uint64 * cap)()
        bms = (ctypes.c_double * cap)()
        ms = (ctypes.c_double * cap)()
        n = self._lib.vkzg_b200_window_trials(self._h, int(size_class), c, nb, bms, ms, cap)
        return [(int(c[i]), int(nb[i]), bms[i], ms[i]) for i in range(min(n, cap))]

    def device_bytes(self):
        """{'working', 'tables', 'digit_table'}: device memory this prover holds."""
        w, t, d = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._lib.vkzg_b200_prover_device_bytes(self._h, ctypes.byref(w), ctypes.byref(t), ctypes.byref(d))
        return {"working": w.value, "tables": t.value, "digit_table": d.value}

    def set_stage_timing(self, enabled):
        self._lib.vkzg_b200_set_stage_timing(self._h, 1 if enabled else 0)

    def last_stage_times(self, recovery=False):
        buf = (ctypes.c_double * 32)()
        n = self._lib.vkzg_b200_last_stage_times(self._h, 1 if recovery else 0, buf, 32)
        return {self._lib.vkzg_b200_stage_name(1 if recovery else 0, i).decode(): buf[i] for i in range(n)}


class Server:
    """Continuous-batching request loop (include/vkzg_b200.h).  Buffers passed to
    submit_* must stay alive until wait() returns for their ticket; numpy arrays
    or raw addresses are accepted."""

    def __init__(self, max_blobs_per_batch=0, lanes=0, hbm_budget_bytes=0, table_budget_bytes=0):
        L = library()
        o = _ServerOptions()
        L.vkzg_b200_server_options_default(ctypes.byref(o))
        o.max_blobs_per_batch, o.lanes, o.hbm_budget_bytes = max_blobs_per_batch, lanes, hbm_budget_bytes
        o.table_budget_bytes = table_budget_bytes
        h = ctypes.c_void_p()
        _check(L.vkzg_b200_server_new(ctypes.byref(h), ctypes.byref(o)))
        self._h, self._lib = h, L
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.vkzg_b200_server_free(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit_proofs(self, proofs_out, blobs, n):
        t = ctypes.c_uint64()
        _check(self._lib.vkzg_b200_server_submit_proofs(self._h, _ptr(proofs_out), _ptr(blobs), n, ctypes.byref(t)))
        self._keep[t.value] = (proofs_out, blobs)
        return t.value

    def submit_recovery(self, cells_out, cells, present, n):
        t = ctypes.c_uint64()
        _check(self._lib.vkzg_b200_server_submit_recovery(self._h, _ptr(cells_out), _ptr(cells), _ptr(present), n,
                                                          ctypes.byref(t)))
        self._keep[t.value] = (cells_out, cells, present)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """Returns the request's final status code (0 = ok), after which the ticket
        is spent and its buffers are released here; or PENDING when timeout_ms ran
        out first, in which case the request is still in flight, its ticket stays
        valid and its buffers stay referenced here."""
        rc = self._lib.vkzg_b200_server_wait(self._h, ticket, int(timeout_ms))
        if rc != PENDING:
            self._keep.pop(ticket, None)
        return rc

    def stats(self, reset=False):
        st = ServerStats()
        _check(self._lib.vkzg_b200_server_stats(self._h, ctypes.byref(st), 1 if reset else 0))
        return st.as_dict()


def comb_windows(d):
    """The widths of the digit table's d windows (as the library cuts a scalar's
    256 bits: the first 256 mod d windows one bit wider than the rest)."""
    w, r = divmod(256, d)
    return [w + 1] * r + [w] * (d - r)


def comb_table_bytes(d):
    """Bytes of the digit table of d windows: 128 x 64 base columns, each with
    2^(width - 1) points of 96 bytes per window."""
    return 128 * 64 * sum(1 << (w - 1) for w in comb_windows(d)) * 96


def grid_sync_selftest(extra_arrivals, spin_limit, rounds):
    """(barriers passed summed over blocks, failure flag, error words marked) of one
    cooperative launch crossing `rounds` grid barriers (vkzg_b200_grid_sync_selftest)."""
    a, b, c = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(library().vkzg_b200_grid_sync_selftest(int(extra_arrivals), int(spin_limit), int(rounds),
                                                  ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return a.value, b.value, c.value


def inverse_selftest(n, seed=1):
    """Words that differ between the four-lane and the one-lane Fp inversion on n
    seeded values (vkzg_b200_inverse_selftest); 0 when they agree."""
    out = ctypes.c_uint32()
    _check(library().vkzg_b200_inverse_selftest(int(n), int(seed), ctypes.byref(out)))
    return out.value


def kernel_launches():
    """Kernels the library has launched in this process (vkzg_b200_kernel_launches)."""
    return int(library().vkzg_b200_kernel_launches())


def microbench(which):
    """0: IMAD issue rate (T/s); 1: Fp multiplies (G/s); 2: Fr multiplies (G/s);
    3: Fp squares; 4: Fp Karatsuba multiplies; 5: Fr Karatsuba multiplies;
    6: Fp Karatsuba squares; 7: Fp two-level Karatsuba multiplies (G/s);
    8: mad.wide.u32 and 9: fma.rn.f64 issue rates (T/s); 10 / 11: one launch of
    16 Fp inversions per SM, variable-time / fixed divstep batches (microseconds);
    12 / 13: Fp multiplies / squares on the FP64 pipe; 14: half the warps on each
    pipe; 15 / 16: FP64-pipe / Karatsuba multiplies with four chains per thread (G/s);
    17: as 11 with four lanes per inversion (microseconds)."""
    out = ctypes.c_double()
    _check(library().vkzg_b200_microbench(int(which), ctypes.byref(out)))
    return out.value


def bucket_sums_selftest(points_xy, bucket_of):
    """Sums affine points (n x 96 bytes, x || y canonical big-endian) into 128 buckets
    with the device's batched-affine routine; returns 128 x 96 bytes."""
    import numpy as np
    pts = np.ascontiguousarray(np.frombuffer(bytes(points_xy), np.uint8))
    idx = np.ascontiguousarray(np.asarray(bucket_of, dtype=np.uint32))
    out = np.zeros(128 * 96, np.uint8)
    _check(library().vkzg_b200_bucket_sums_selftest(_ptr(pts), _ptr(idx), len(idx), _ptr(out)))
    return out.tobytes()


def tree_sums_selftest(points_xy, n_lists, m, seed=0):
    """Sums n_lists lists of m points (96-byte x || y each) with the grid-wide tree
    rounds; points_xy None = seeded device-generated coordinates (timing only).
    Returns (sums bytes or None, device ms)."""
    import numpy as np
    ms = ctypes.c_double()
    pts = None if points_xy is None else np.ascontiguousarray(np.frombuffer(bytes(points_xy), np.uint8))
    out = np.zeros(n_lists * 96, np.uint8) if pts is not None else None
    _check(library().vkzg_b200_tree_sums_selftest(_ptr(pts), n_lists, m, seed, _ptr(out), ctypes.byref(ms)))
    return (out.tobytes() if out is not None else None), ms.value


def write_tables(g1_monomial_compressed, out_path):
    """Generates the FK20 tables on the GPU from a G1 monomial setup and writes them
    in the reference's precomputed_tables.bin format."""
    setup = bytes(g1_monomial_compressed)
    if len(setup) != 4096 * 48:
        raise ValueError("expected 4096 compressed G1 points")
    _check(library().vkzg_b200_write_tables(_ptr(setup), out_path.encode()))


# ---------------------------------------------------------------- Vkzg.java mirror
_global = None
_global_lock = threading.Lock()


def init(max_batch_size=0):
    """Vkzg.init (Vkzg.java:164-184)."""
    global _global
    with _global_lock:
        if _global is not None:
            raise RuntimeError("already initialized")
        _global = Prover(max_batch_size)


def deinit():
    global _global
    with _global_lock:
        _loaded().close()
        _global = None


def _loaded():
    if _global is None:
        raise RuntimeError("not initialized; call init() first")
    return _global


def computeCellKzgProofsBatch(blobs, blob_count):  # noqa: N802 (reference name)
    with _global_lock:
        return _loaded().compute_cell_kzg_proofs_batch(blobs, blob_count)


def recoverCellsBatch(cells, cell_present, blob_count):  # noqa: N802
    with _global_lock:
        return _loaded().recover_cells_batch(cells, cell_present, blob_count)


def deviceName():  # noqa: N802
    with _global_lock:
        return _loaded().device_name()


def gpuCoreCount():  # noqa: N802
    with _global_lock:
        return _loaded().gpu_core_count()
