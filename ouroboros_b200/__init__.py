"""ouroboros_b200 -- the Ouroboros device allocator, re-designed for B200.

Host-side mirror of the reference's interface (GPUPeople/Ouroboros,
include/device/Ouroboros.cuh:247-297): an :class:`Ouroboros` heap is created with
``initialize(heap_bytes)``, its device object (``getDeviceMemoryManager()``) is
what kernels call ``malloc``/``free`` on, and the six instantiations of
include/InstanceDefinitions.cuh:16-34 are available under their reference names
(``MultiOuroPQ`` ... ``MultiOuroVLCQ``).  Everything runs through the CUDA
library ``_lib/libouroboros_b200.so`` (C ABI: include/ouroboros_b200.h); there
is no CPU fallback -- without the library every call raises.

Device buffers are passed as integers (device addresses) or torch tensors.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libouroboros_b200.so")

VARIANTS = ("P", "C", "VAP", "VAC", "VLP", "VLC")
VARIANT_NAMES = {
    "P": "MultiOuroPQ", "C": "MultiOuroCQ", "VAP": "MultiOuroVAPQ",
    "VAC": "MultiOuroVACQ", "VLP": "MultiOuroVLPQ", "VLC": "MultiOuroVLCQ",
}
STATE_WORDS = 151
NUM_CLASSES = 12
RES_FAIL = 1 << 63
RES_DEVHEAP = 1 << 62

FLAG_OOM, FLAG_TIMEOUT, FLAG_CORRUPT, FLAG_QUEUE_FULL = 1, 2, 4, 8

# Every symbol declared in include/ouroboros_b200.h
EXPORTS = (
    "ouro_create", "ouro_destroy", "ouro_device_handle", "ouro_get_info", "ouro_alloc", "ouro_free",
    "ouro_trace", "ouro_state", "ouro_get_status", "ouro_write_pattern", "ouro_verify_pattern",
    "ouro_check_allocations", "ouro_check_heap", "ouro_measure_atomics", "ouro_scan_stats",
    "ouro_status_string", "ouro_check_allocations_noalloc", "ouro_free_resources", "ouro_prefill",
    "ouro_alloc_batch", "ouro_free_batch", "ouro_realloc_batch", "ouro_autotune_batch",
    "ouro_graph_init", "ouro_graph_grow", "ouro_graph_check", "ouro_free_bytes_to",
    "ouro_allocate_chunk", "ouro_enqueue_initial_chunk", "ouro_batch_reserve",
    "ouro_serve_start", "ouro_serve_submit", "ouro_serve_poll", "ouro_serve_stop", "ouro_serve_close",
    "ouro_config_default", "ouro_create_config", "ouro_get_config", "ouro_autotune_config",
    "ouro_alloc_host", "ouro_free_host", "ouro_host_reserve",
)


class OuroError(RuntimeError):
    pass


class _Info(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int32), ("heap_bytes", ctypes.c_uint64), ("max_chunks", ctypes.c_uint64),
                ("alloc_bytes", ctypes.c_uint64), ("data_base", ctypes.c_uint64), ("data_end", ctypes.c_uint64)]


class Config(ctypes.Structure):
    """ouro_config: run-time parameters of a heap (defaults: the reference's
    compile-time ones, include/Parameters.h:9-18)."""
    _fields_ = [("chunk_bytes", ctypes.c_uint32), ("page_queue_entries", ctypes.c_uint32),
                ("virtual_queue_entries", ctypes.c_uint32), ("agg_width", ctypes.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class TunePoint(ctypes.Structure):
    _fields_ = [("cfg", Config), ("block", ctypes.c_int), ("ok", ctypes.c_int), ("mops", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {**self.cfg.as_dict(), "block": int(self.block), "ok": bool(self.ok), "mops": float(self.mops)}


def autotune_config(variant: str, heap_bytes: int, n: int, lo: int = 16, hi: int = 8192, reps: int = 2,
                    queue_entries=(1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20), agg_widths=(8, 16, 32),
                    blocks=(128, 256, 512, 1024)) -> dict:
    """ouro_autotune_config: every (queue capacity, aggregation width, block
    size) candidate on a fresh heap, batched alloc + free of n log-uniform
    sizes; returns {"best": ..., "points": [...]}."""
    q = np.asarray(queue_entries, dtype=np.uint32)
    a = np.asarray(agg_widths, dtype=np.uint32)
    b = np.asarray(blocks, dtype=np.int32)
    pts = (TunePoint * (len(q) * len(a) * len(b)))()
    best = TunePoint()
    _check(lib().ouro_autotune_config(VARIANTS.index(variant), int(heap_bytes), n, lo, hi, reps,
                                      q.ctypes.data, len(q), a.ctypes.data, len(a), b.ctypes.data, len(b),
                                      pts, ctypes.byref(best)), "ouro_autotune_config")
    return {"best": best.as_dict(), "points": [p.as_dict() for p in pts]}


def default_config(**overrides) -> Config:
    c = Config()
    _check(lib().ouro_config_default(ctypes.byref(c)), "ouro_config_default")
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise ValueError(f"unknown config field {k}")
        setattr(c, k, int(v))
    return c


class _Status(ctypes.Structure):
    _fields_ = [("flags", ctypes.c_uint32), ("null_results", ctypes.c_uint64), ("timeouts", ctypes.c_uint64),
                ("chunk_allocs", ctypes.c_uint64), ("next_free_chunk", ctypes.c_uint64),
                ("timeout_sites", ctypes.c_uint32)]


class _AllocReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("checked", "nulls", "out_of_heap", "misaligned", "overlaps")]


class _SizeDist(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("lo", ctypes.c_uint32), ("hi", ctypes.c_uint32), ("zipf_s", ctypes.c_float)]


class _FreeReport(ctypes.Structure):
    _fields_ = [("page_size", ctypes.c_uint32 * 12), ("free_pages", ctypes.c_int64 * 12),
                ("queue_entries", ctypes.c_uint64 * 12), ("chunks_in_use", ctypes.c_uint64),
                ("chunks_untouched", ctypes.c_uint64), ("chunks_pooled", ctypes.c_uint64),
                ("free_bytes", ctypes.c_uint64), ("heap_chunks", ctypes.c_uint64)]


class _HeapReport(ctypes.Structure):
    _fields_ = [("owned_pages", ctypes.c_uint64 * 12), ("free_pages_meta", ctypes.c_uint64 * 12),
                ("sem_count", ctypes.c_int64 * 12), ("sem_expected", ctypes.c_uint64 * 12),
                ("sem_reserved", ctypes.c_uint64 * 12), ("data_chunks", ctypes.c_uint64), ("bad", ctypes.c_uint64)]


class ServeConfig(ctypes.Structure):
    _fields_ = [("ring", ctypes.c_uint32), ("max_inflight", ctypes.c_uint32), ("blocks_per_sm", ctypes.c_int),
                ("watermark", ctypes.c_double), ("idle_seconds", ctypes.c_double)]


class ServeResult(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_uint64), ("client", ctypes.c_uint32), ("n", ctypes.c_uint32),
                ("t_seen_ns", ctypes.c_uint64), ("t_start_ns", ctypes.c_uint64), ("t_done_ns", ctypes.c_uint64),
                ("failed_allocs", ctypes.c_uint64), ("lock_giveups", ctypes.c_uint64), ("held_back", ctypes.c_uint32)]


class ServeStats(ctypes.Structure):
    _fields_ = [("batches_seen", ctypes.c_uint64), ("batches_admitted", ctypes.c_uint64),
                ("held_back", ctypes.c_uint64), ("status", ctypes.c_uint32)]


OURO_ERR_FULL = 6

_lib = None


def lib():
    """The loaded CUDA library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OuroError(f"{LIB_PATH} is missing: build it with `python -m ouroboros_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        p, u32, u64, i = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        L.ouro_create.argtypes = [i, u64, ctypes.POINTER(p)]
        L.ouro_config_default.argtypes = [ctypes.POINTER(Config)]
        L.ouro_create_config.argtypes = [i, u64, ctypes.POINTER(Config), ctypes.POINTER(p)]
        L.ouro_get_config.argtypes = [p, ctypes.POINTER(Config)]
        L.ouro_autotune_config.argtypes = [i, u64, u32, u32, u32, u32, p, u32, p, u32, p, u32,
                                           ctypes.POINTER(TunePoint), ctypes.POINTER(TunePoint)]
        L.ouro_destroy.argtypes = [p]
        L.ouro_device_handle.argtypes = [p]
        L.ouro_device_handle.restype = p
        L.ouro_get_info.argtypes = [p, ctypes.POINTER(_Info)]
        L.ouro_alloc.argtypes = [p, u32, u32, p, p, i, p]
        L.ouro_free.argtypes = [p, u32, p, i, p]
        L.ouro_alloc_host.argtypes = [p, u32, u32, p, p, p, i, i, p]
        L.ouro_free_host.argtypes = [p, u32, p, i, i, p]
        L.ouro_host_reserve.argtypes = [p, u32]
        L.ouro_trace.argtypes = [p, p, u64, p, u32, u32]
        L.ouro_state.argtypes = [p, p]
        L.ouro_get_status.argtypes = [p, ctypes.POINTER(_Status), i]
        L.ouro_write_pattern.argtypes = [p, u32, u32, p, u32, p]
        L.ouro_verify_pattern.argtypes = [p, u32, u32, p, u32, p, p]
        L.ouro_check_allocations.argtypes = [p, p, u32, u32, p, ctypes.POINTER(_AllocReport)]
        L.ouro_check_heap.argtypes = [p, ctypes.POINTER(_HeapReport)]
        L.ouro_measure_atomics.argtypes = [i, ctypes.POINTER(ctypes.c_double)]
        L.ouro_scan_stats.argtypes = [p, p, i]
        L.ouro_check_allocations_noalloc.argtypes = [p, p, u32, u32, p, p, p]
        L.ouro_free_resources.argtypes = [p, ctypes.POINTER(_FreeReport)]
        L.ouro_prefill.argtypes = [p, u64, u64, ctypes.POINTER(ctypes.c_uint64), p]
        L.ouro_allocate_chunk.argtypes = [p, ctypes.POINTER(ctypes.c_uint32)]
        L.ouro_serve_start.argtypes = [p, p, p, u32, u64, ctypes.POINTER(ServeConfig), ctypes.POINTER(p)]
        L.ouro_serve_submit.argtypes = [p, p, u32, u32, ctypes.POINTER(ctypes.c_uint64)]
        L.ouro_serve_poll.argtypes = [p, ctypes.POINTER(ServeResult), u32, ctypes.POINTER(ctypes.c_uint32)]
        L.ouro_serve_stop.argtypes = [p, ctypes.POINTER(ServeStats)]
        L.ouro_serve_close.argtypes = [p]
        L.ouro_enqueue_initial_chunk.argtypes = [p, u32, u32, u32]
        L.ouro_alloc_batch.argtypes = [p, p, p, u32, i, p]
        L.ouro_batch_reserve.argtypes = [p, u32]
        L.ouro_free_batch.argtypes = [p, p, u32, i, p]
        L.ouro_realloc_batch.argtypes = [p, p, p, u32, u64, u32, u32, ctypes.POINTER(_SizeDist), i, p]
        L.ouro_graph_init.argtypes = [p, p, p, p, u32, u64, ctypes.c_float, p, p]
        L.ouro_graph_grow.argtypes = [p, p, p, p, u32, u32, u64, p, p]
        L.ouro_graph_check.argtypes = [p, p, p, u32, u32, u64, p, p]
        L.ouro_free_bytes_to.argtypes = [p, p, p]
        L.ouro_autotune_batch.argtypes = [p, u32, u32, u32, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double)]
        L.ouro_status_string.argtypes = [i]
        L.ouro_status_string.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc:
        raise OuroError(f"{what}: {lib().ouro_status_string(rc).decode()} ({rc})")


def _addr(x) -> int | None:
    """Address of a tensor (device or host), a numpy array, an int, or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x or None
    if isinstance(x, np.ndarray):
        return x.ctypes.data or None
    return x.data_ptr()


def _stream(s) -> int | None:
    if s is None:
        return None
    if isinstance(s, int):
        return s or None
    return s.cuda_stream or None


class Ouroboros:
    """One heap of one instantiation on the current device."""

    def __init__(self, variant: str = "P", heap_bytes: int | None = None, config: Config | dict | None = None):
        if variant not in VARIANTS:
            raise ValueError(f"variant must be one of {VARIANTS}")
        self.variant = variant
        self._h = None
        self._config = default_config(**config) if isinstance(config, dict) else config
        if heap_bytes is not None:
            self.initialize(heap_bytes)

    # -- reference interface ------------------------------------------------
    def initialize(self, heap_bytes: int) -> "Ouroboros":
        """Ouroboros<...>::initialize (MemoryInitialization.cuh:123-219); idempotent."""
        if self._h is not None:
            return self
        h = ctypes.c_void_p()
        if self._config is None:
            _check(lib().ouro_create(VARIANTS.index(self.variant), int(heap_bytes), ctypes.byref(h)), "ouro_create")
        else:
            _check(lib().ouro_create_config(VARIANTS.index(self.variant), int(heap_bytes), ctypes.byref(self._config),
                                            ctypes.byref(h)), "ouro_create_config")
        self._h = h
        return self

    def config(self) -> dict:
        c = Config()
        _check(lib().ouro_get_config(self._handle(), ctypes.byref(c)), "ouro_get_config")
        return c.as_dict()

    def getDeviceMemoryManager(self) -> int:  # noqa: N802 (reference name)
        return int(lib().ouro_device_handle(self._handle()))

    # -- lifetime -------------------------------------------------------------
    def _handle(self):
        if self._h is None:
            raise OuroError("heap not initialized")
        return self._h

    def close(self):
        if self._h is not None:
            lib().ouro_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- launches ---------------------------------------------------------------
    def alloc(self, out_ptrs, n: int, size: int = 0, sizes=None, block: int = 256, stream=None):
        """Thread i of one launch: out_ptrs[i] = malloc(size or sizes[i])."""
        _check(lib().ouro_alloc(self._handle(), n, size, _addr(sizes), _addr(out_ptrs), block, _stream(stream)),
               "ouro_alloc")

    def free(self, ptrs, n: int, block: int = 256, stream=None):
        _check(lib().ouro_free(self._handle(), n, _addr(ptrs), block, _stream(stream)), "ouro_free")

    def alloc_host(self, out_host, n: int, size: int = 0, sizes_host=None, out_device=None, block: int = 256,
                   slices: int = 0, stream=None):
        """alloc() for requests and results in host memory (pinned for
        overlapped copies): out_host[i] = malloc(size or sizes_host[i]), and
        out_device[i] too when given.  Asynchronous on `stream`."""
        _check(lib().ouro_alloc_host(self._handle(), n, size, _addr(sizes_host), _addr(out_host), _addr(out_device),
                                     block, slices, _stream(stream)), "ouro_alloc_host")

    def host_reserve(self, n: int):
        """Streams, events and device staging of the host-buffer calls for up
        to n requests, made now rather than by the first call."""
        _check(lib().ouro_host_reserve(self._handle(), n), "ouro_host_reserve")

    def free_host(self, ptrs_host, n: int, block: int = 256, slices: int = 0, stream=None):
        """free() of a host-memory pointer array.  Asynchronous on `stream`."""
        _check(lib().ouro_free_host(self._handle(), n, _addr(ptrs_host), block, slices, _stream(stream)),
               "ouro_free_host")

    def allocate_chunk(self) -> int:
        """allocateChunk<false> of the first instance (Ouroboros.cuh:108-136): an
        8 KiB chunk index, or 0xFFFFFFFF when none is left."""
        out = ctypes.c_uint32()
        _check(lib().ouro_allocate_chunk(self._handle(), ctypes.byref(out)), "ouro_allocate_chunk")
        return int(out.value)

    def enqueue_initial_chunk(self, queue_index: int, chunk_index: int, available_pages: int):
        """enqueueInitialChunk (Ouroboros.cuh:291-295): the chunk joins class
        queue_index with its last available_pages pages free."""
        _check(lib().ouro_enqueue_initial_chunk(self._handle(), queue_index, chunk_index, available_pages),
               "ouro_enqueue_initial_chunk")

    def trace(self, ops: np.ndarray, tid: int = 0, bid: int = 0) -> np.ndarray:
        ops = np.ascontiguousarray(ops, dtype=np.uint32)
        res = np.zeros(ops.size // 2, dtype=np.uint64)
        _check(lib().ouro_trace(self._handle(), ops.ctypes.data, ops.size // 2, res.ctypes.data, tid, bid),
               "ouro_trace")
        return res

    # -- introspection --------------------------------------------------------
    def info(self) -> dict:
        out = _Info()
        _check(lib().ouro_get_info(self._handle(), ctypes.byref(out)), "ouro_get_info")
        return {n: int(getattr(out, n)) for n, _ in _Info._fields_}

    def state(self) -> np.ndarray:
        out = np.zeros(STATE_WORDS, dtype=np.uint64)
        _check(lib().ouro_state(self._handle(), out.ctypes.data), "ouro_state")
        return out

    def status(self, clear: bool = False) -> dict:
        out = _Status()
        _check(lib().ouro_get_status(self._handle(), ctypes.byref(out), int(clear)), "ouro_get_status")
        return {n: int(getattr(out, n)) for n, _ in _Status._fields_}

    def check_allocations(self, ptrs, n: int, size: int = 0, sizes=None) -> dict:
        out = _AllocReport()
        _check(lib().ouro_check_allocations(self._handle(), _addr(ptrs), n, size, _addr(sizes), ctypes.byref(out)),
               "ouro_check_allocations")
        return {k: int(getattr(out, k)) for k, _ in _AllocReport._fields_}

    def scan_stats(self, clear: bool = False) -> dict:
        out = np.zeros(12, dtype=np.uint64)
        _check(lib().ouro_scan_stats(self._handle(), out.ctypes.data, int(clear)), "ouro_scan_stats")
        names = ("groups", "probes", "misses", "runs", "slow_cyc_sem", "slow_cyc_scan", "slow_cyc_dequeue",
                 "slow_cyc_claim", "slow_groups", "cyc_max", "slow_probes", "slow_misses")
        return {k: int(x) for k, x in zip(names, out)}

    # -- batched path ---------------------------------------------------------
    def batch_reserve(self, n: int):
        """Scratch for batches of up to n requests (call before capturing batch calls in a graph)."""
        _check(lib().ouro_batch_reserve(self._handle(), n), "ouro_batch_reserve")

    def alloc_batch(self, sizes, out_ptrs, n: int, block: int = 0, stream=None):
        """out_ptrs[i] = malloc(sizes[i]), binned by size class per tile."""
        _check(lib().ouro_alloc_batch(self._handle(), _addr(sizes), _addr(out_ptrs), n, block, _stream(stream)),
               "ouro_alloc_batch")

    def free_batch(self, ptrs, n: int, block: int = 0, stream=None):
        _check(lib().ouro_free_batch(self._handle(), _addr(ptrs), n, block, _stream(stream)), "ouro_free_batch")

    def realloc_batch(self, ptrs, sizes, n: int, seed: int, cycle: int, fraction_permille: int,
                      dist=("loguniform", 16, 8192), block: int = 0, stream=None):
        """One churn cycle: a hashed fraction of the requests frees and reallocates
        with a new size drawn from dist = ("loguniform", lo, hi) or ("zipf", s)."""
        d = _SizeDist(0, dist[1], dist[2], 0.0) if dist[0] == "loguniform" else _SizeDist(1, 16, 8192, float(dist[1]))
        _check(lib().ouro_realloc_batch(self._handle(), _addr(ptrs), _addr(sizes), n, seed & (2**64 - 1), cycle,
                                        fraction_permille, ctypes.byref(d), block, _stream(stream)),
               "ouro_realloc_batch")

    def autotune_batch(self, n: int = 1 << 20, lo: int = 16, hi: int = 8192) -> dict:
        b, s, m = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().ouro_autotune_batch(self._handle(), n, lo, hi, ctypes.byref(b), ctypes.byref(s), ctypes.byref(m)),
               "ouro_autotune_batch")
        return {"block": b.value, "blocks_per_sm": s.value, "mops": m.value}

    def prefill(self, size: int, pages: int, stream=None) -> int:
        """preFillQueue: add enough fresh chunks to the class of `size` for
        `pages` free pages; returns the pages added."""
        out = ctypes.c_uint64()
        _check(lib().ouro_prefill(self._handle(), int(size), int(pages), ctypes.byref(out), _stream(stream)),
               "ouro_prefill")
        return int(out.value)

    def free_resources(self) -> dict:
        """printFreeResources (MemoryQueries.cuh:8-88) as numbers: per class
        page size, free pages, queue entries; chunks in use / untouched /
        pooled and the free bytes an admission watermark compares against."""
        out = _FreeReport()
        _check(lib().ouro_free_resources(self._handle(), ctypes.byref(out)), "ouro_free_resources")
        return {
            "page_size": list(out.page_size), "free_pages": list(out.free_pages),
            "queue_entries": list(out.queue_entries), "chunks_in_use": int(out.chunks_in_use),
            "chunks_untouched": int(out.chunks_untouched), "chunks_pooled": int(out.chunks_pooled),
            "free_bytes": int(out.free_bytes), "heap_chunks": int(out.heap_chunks),
        }

    def check_heap(self) -> dict:
        out = _HeapReport()
        _check(lib().ouro_check_heap(self._handle(), ctypes.byref(out)), "ouro_check_heap")
        return {
            "owned_pages": list(out.owned_pages), "free_pages_meta": list(out.free_pages_meta),
            "sem_count": list(out.sem_count), "sem_expected": list(out.sem_expected),
            "sem_reserved": list(out.sem_reserved), "data_chunks": int(out.data_chunks), "bad": int(out.bad),
        }


def write_pattern(ptrs, n: int, size: int = 0, seed: int = 0x9E3779B9, sizes=None, stream=None):
    _check(lib().ouro_write_pattern(_addr(ptrs), n, size, _addr(sizes), seed & 0xFFFFFFFF, _stream(stream)),
           "ouro_write_pattern")


def verify_pattern(ptrs, n: int, counters, size: int = 0, seed: int = 0x9E3779B9, sizes=None, stream=None):
    _check(lib().ouro_verify_pattern(_addr(ptrs), n, size, _addr(sizes), seed & 0xFFFFFFFF, _addr(counters),
                                     _stream(stream)), "ouro_verify_pattern")


def measure_atomics(mode: int) -> float:
    """G L2 atomic operations per second: 0 distinct addresses, 1 / 2 one hot 32 / 64-bit address,
    3 / 4 two hot 32-bit addresses 128 B / 256 B apart."""
    out = ctypes.c_double()
    _check(lib().ouro_measure_atomics(mode, ctypes.byref(out)), "ouro_measure_atomics")
    return float(out.value)


def _named(variant):
    def make(heap_bytes: int | None = None) -> Ouroboros:
        return Ouroboros(variant, heap_bytes)
    make.__name__ = VARIANT_NAMES[variant]
    return make


MultiOuroPQ = _named("P")
MultiOuroCQ = _named("C")
MultiOuroVAPQ = _named("VAP")
MultiOuroVACQ = _named("VAC")
MultiOuroVLPQ = _named("VLP")
MultiOuroVLCQ = _named("VLC")
