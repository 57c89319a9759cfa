"""TEST INFRASTRUCTURE ONLY: Python handles on the two checkers in this folder.

* :class:`Oracle` wraps ``_build/libouro_oracle.so``, the sequential C
  restatement of the reference allocator (``ouro_oracle.c``).
* :class:`RefDriver` wraps ``_ref/libouro_ref.so``, the reference's own CUDA
  code compiled for sm_100a (``ref_driver.cu``); it needs a GPU.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
legs of ``bench.py`` import this package.  The allocator itself never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libouro_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libouro_ref.so")

VARIANTS = ("P", "C", "VAP", "VAC", "VLP", "VLC")
STATE_WORDS = 151
NUM_CLASSES = 12
RES_FAIL = 1 << 63
RES_DEVHEAP = 1 << 62

ERRORS = {0: "ok", 1: "bad argument", 2: "reference undefined behaviour", 3: "reference trap",
          4: "reference hang"}


class OracleError(RuntimeError):
    pass


class _Layout(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "object_bytes", "queue_bytes", "total_required", "max_chunks", "locator_bytes", "allocation_bytes")]


_oracle_lib = None


def _olib():
    global _oracle_lib
    if _oracle_lib is None:
        if not os.path.exists(ORACLE_SO):
            raise OracleError(f"{ORACLE_SO} missing: run `make -C oracle oracle`")
        lib = ctypes.CDLL(ORACLE_SO)
        u64, u32, p = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p
        lib.orc_layout_of.argtypes = [ctypes.c_int, u64, ctypes.POINTER(_Layout)]
        lib.orc_create.argtypes = [ctypes.c_int, u64, u32, u32]
        lib.orc_create.restype = p
        lib.orc_destroy.argtypes = [p]
        lib.orc_malloc.argtypes = [p, u64, ctypes.POINTER(u64), ctypes.POINTER(ctypes.c_int64)]
        lib.orc_free.argtypes = [p, u64]
        lib.orc_run_trace.argtypes = [p, p, u64, p, p, ctypes.POINTER(u64)]
        lib.orc_state.argtypes = [p, p]
        lib.orc_next_free_chunk.argtypes = [p]
        lib.orc_next_free_chunk.restype = u64
        _oracle_lib = lib
    return _oracle_lib


def layout(variant: str | int, heap_bytes: int) -> dict:
    v = VARIANTS.index(variant) if isinstance(variant, str) else int(variant)
    out = _Layout()
    rc = _olib().orc_layout_of(v, heap_bytes, ctypes.byref(out))
    if rc:
        raise OracleError(ERRORS.get(rc, rc))
    return {n: int(getattr(out, n)) for n, _ in _Layout._fields_}


class Oracle:
    """Sequential restatement of one reference heap (one GPU thread (tid, bid))."""

    def __init__(self, variant: str, heap_bytes: int, tid: int = 0, bid: int = 0):
        self.variant = variant
        self._lib = _olib()
        self._h = self._lib.orc_create(VARIANTS.index(variant), heap_bytes, tid, bid)
        if not self._h:
            raise OracleError("orc_create failed")

    def close(self):
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def malloc(self, size: int):
        res, off = ctypes.c_uint64(), ctypes.c_int64()
        rc = self._lib.orc_malloc(self._h, size, ctypes.byref(res), ctypes.byref(off))
        if rc:
            raise OracleError(ERRORS.get(rc, rc))
        return int(res.value), int(off.value)

    def free(self, res: int):
        rc = self._lib.orc_free(self._h, res)
        if rc:
            raise OracleError(ERRORS.get(rc, rc))

    def run_trace(self, ops: np.ndarray):
        ops = np.ascontiguousarray(ops, dtype=np.uint32)
        n = ops.size // 2
        res = np.zeros(n, dtype=np.uint64)
        off = np.zeros(n, dtype=np.int64)
        failed = ctypes.c_uint64(0)
        rc = self._lib.orc_run_trace(self._h, ops.ctypes.data, n, res.ctypes.data, off.ctypes.data,
                                     ctypes.byref(failed))
        if rc:
            raise OracleError(f"{ERRORS.get(rc, rc)} at op {failed.value}")
        return res, off

    def state(self) -> np.ndarray:
        out = np.zeros(STATE_WORDS, dtype=np.uint64)
        self._lib.orc_state(self._h, out.ctypes.data)
        return out

    def next_free_chunk(self) -> int:
        return int(self._lib.orc_next_free_chunk(self._h))


_ref_lib = None


def _rlib():
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(REF_SO):
            raise OracleError(f"{REF_SO} missing: run `make -C oracle ref` where the reference is mounted")
        lib = ctypes.CDLL(REF_SO)
        u64, u32, p, i = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int
        lib.ref_create.argtypes = [i, u64, ctypes.POINTER(p)]
        lib.ref_destroy.argtypes = [p]
        lib.ref_trace.argtypes = [p, p, u64, p, u32, u32]
        lib.ref_state.argtypes = [p, p]
        lib.ref_info.argtypes = [p, p]
        lib.ref_alloc.argtypes = [p, u32, u32, p, p, i, p]
        lib.ref_free.argtypes = [p, u32, p, i, p]
        lib.ref_write.argtypes = [p, u32, u32, p, u32, p]
        lib.ref_sanitize.argtypes = [p, p, u32, u32, p, p, p]
        lib.ref_verify.argtypes = [p, u32, u32, p, u32, p, p]
        lib.ref_run_cell.argtypes = [p, u32, u32, i, i, p, u32, p, p]
        _ref_lib = lib
    return _ref_lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class RefDriver:
    """The reference allocator itself (sm_100a build), one heap on the current GPU."""

    def __init__(self, variant: str, heap_bytes: int):
        self.variant = variant
        self._lib = _rlib()
        h = ctypes.c_void_p()
        rc = self._lib.ref_create(VARIANTS.index(variant), heap_bytes, ctypes.byref(h))
        if rc:
            raise OracleError(f"ref_create failed ({rc})")
        self._h = h

    def close(self):
        if self._h:
            self._lib.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        out = np.zeros(4, dtype=np.uint64)
        self._lib.ref_info(self._h, out.ctypes.data)
        return {"max_chunks": int(out[0]), "allocation_bytes": int(out[1]), "d_memory": int(out[2]),
                "d_data": int(out[3])}

    def run_trace(self, ops: np.ndarray, tid: int = 0, bid: int = 0) -> np.ndarray:
        ops = np.ascontiguousarray(ops, dtype=np.uint32)
        n = ops.size // 2
        off = np.zeros(n, dtype=np.int64)
        rc = self._lib.ref_trace(self._h, ops.ctypes.data, n, off.ctypes.data, tid, bid)
        if rc:
            raise OracleError(f"ref_trace failed ({rc})")
        return off

    def state(self) -> np.ndarray:
        out = np.zeros(STATE_WORDS, dtype=np.uint64)
        rc = self._lib.ref_state(self._h, out.ctypes.data)
        if rc:
            raise OracleError(f"ref_state failed ({rc})")
        return out

    def alloc(self, n, size, d_ptrs, d_sizes=0, block=256, stream=0):
        rc = self._lib.ref_alloc(self._h, n, size, d_sizes or None, d_ptrs, block, stream or None)
        if rc:
            raise OracleError(f"ref_alloc failed ({rc})")

    def free(self, n, d_ptrs, block=256, stream=0):
        rc = self._lib.ref_free(self._h, n, d_ptrs, block, stream or None)
        if rc:
            raise OracleError(f"ref_free failed ({rc})")

    def sanitize(self, n, size, d_ptrs, d_counters, d_sizes=0, stream=0):
        """Null (and count in d_counters[1]) every pointer the reference returned
        outside its chunk region, before anything writes through or frees it."""
        rc = self._lib.ref_sanitize(self._h, d_ptrs, n, size, d_sizes or None, d_counters, stream or None)
        if rc:
            raise OracleError(f"ref_sanitize failed ({rc})")

    def run_cell(self, n, size, reps, d_ptrs, d_counters, seed=0x9E3779B9, block=256):
        ms = np.zeros(2, dtype=np.float32)
        rc = self._lib.ref_run_cell(self._h, n, size, block, reps, d_ptrs, seed, d_counters, ms.ctypes.data)
        if rc:
            raise OracleError(f"ref_run_cell failed ({rc})")
        return float(ms[0]), float(ms[1])


def ref_write(d_ptrs, n, size, seed, d_sizes=0, stream=0):
    _rlib().ref_write(d_ptrs, n, size, d_sizes or None, seed, stream or None)


def ref_verify(d_ptrs, n, size, seed, d_counters, d_sizes=0, stream=0):
    _rlib().ref_verify(d_ptrs, n, size, d_sizes or None, seed, d_counters, stream or None)


def decode(res: int):
    """Encoded result -> (class id, chunk, page) or None for failures / device heap."""
    if res & (RES_FAIL | RES_DEVHEAP):
        return None
    return (res >> 32) & 0xFF, (res & 0xFFFFFFFF) >> 9, res & 511
