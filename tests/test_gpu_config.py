"""The run-time configuration (ouro_config) and its autotuner.

The reference fixes its parameters at compile time (include/Parameters.h:9-18);
here a heap takes them at creation.  The defaults must be the reference's and
give the reference's capacity; other queue sizes and aggregation widths must
keep every invariant of the per-thread and batched paths."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import ouroboros_b200 as ob

from tests.test_gpu_concurrent import _idle, _ptrs, _round

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def test_default_config_is_the_reference_parameters():
    c = ob.default_config().as_dict()
    assert c == {"chunk_bytes": 8192, "page_queue_entries": 1 << 23, "virtual_queue_entries": 16384, "agg_width": 32}
    for v in ob.VARIANTS:
        with ob.Ouroboros(v, GiB, config=ob.default_config()) as heap:
            assert heap.info()["max_chunks"] == oracle.layout(v, GiB)["max_chunks"]
            assert heap.config() == c


def test_bad_configs_are_refused():
    out = ctypes.c_void_p()
    for bad in ({"chunk_bytes": 4096}, {"chunk_bytes": 16384}, {"page_queue_entries": 3 << 16},
                {"page_queue_entries": 1 << 15}, {"page_queue_entries": 1 << 24}, {"virtual_queue_entries": 16},
                {"virtual_queue_entries": 1 << 15}, {"agg_width": 3}, {"agg_width": 64}, {"agg_width": 0}):
        cfg = ob.default_config(**bad)
        assert ob.lib().ouro_create_config(0, GiB, ctypes.byref(cfg), ctypes.byref(out)) == 1, bad


def test_smaller_queues_leave_more_chunks():
    """The capacity formula on the configured queue sizes: 2^16-entry rings free
    the standard variants' queue region for chunks."""
    with ob.Ouroboros("P", GiB) as a, ob.Ouroboros("P", GiB, config={"page_queue_entries": 1 << 16}) as b:
        assert b.info()["max_chunks"] > a.info()["max_chunks"]
        q = (1 << 23) - (1 << 16)
        # 12 rings of 4-byte entries fewer, in 8320-byte reference chunks
        assert b.info()["max_chunks"] - a.info()["max_chunks"] == pytest.approx(12 * 4 * q / 8320, abs=2)


@pytest.mark.parametrize("v,cfg", [
    ("P", {"page_queue_entries": 1 << 16}),
    ("C", {"page_queue_entries": 1 << 16}),
    ("VAP", {"virtual_queue_entries": 32}),
    ("VAC", {"virtual_queue_entries": 32}),
    ("P", {"agg_width": 1}),
    ("VAP", {"agg_width": 8}),
    ("C", {"agg_width": 4}),
    ("VLP", {"agg_width": 16}),
    ("VLC", {"agg_width": 8}),
    ("VAC", {"agg_width": 2, "virtual_queue_entries": 64}),
])
def test_configured_heaps_keep_the_invariants(v, cfg):
    """Fixed and mixed sizes through the per-thread path, three rounds each,
    on a heap with small queues or narrow aggregation: no nulls, no overlap,
    aligned, in the heap, accounting idle after every round."""
    n = 1 << 15
    rng = np.random.default_rng(5)
    mixed = torch.from_numpy(rng.choice([16, 48, 100, 512, 2048, 8192], n).astype(np.uint32).view(np.int32)).cuda()
    with ob.Ouroboros(v, GiB, config=cfg) as heap:
        ptrs = _ptrs(n)
        for r in range(3):
            for size, sizes in ((64, None), (0, mixed)):
                rep, nulls, bad = _round(heap, ptrs, n, size, sizes, seed=r + 3)
                assert nulls == 0 and bad == 0, (r, size, nulls, bad)
                assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep
                _idle(heap, v)
        assert heap.status()["flags"] == 0


@pytest.mark.parametrize("v", ["P", "VAP"])
def test_small_queues_fill_up_cleanly(v):
    """A page-based class that would need more queue entries than its
    configured queue holds (2^16: a 2^16-entry ring, or 32 queue chunks of
    2048) is refused the chunks beyond it (nullptr, the queue-full flag), never
    corrupted: what was served is valid, at most 2^16 pages are handed out, and
    after the frees the accounting is idle."""
    cfg = {"page_queue_entries": 1 << 16} if v == "P" else {"virtual_queue_entries": 32}
    n = 1 << 17   # 2^17 x 16 B pages of one class > 2^16 queue entries
    with ob.Ouroboros(v, GiB, config=cfg) as heap:
        ptrs = _ptrs(n)
        heap.alloc(ptrs, n, 16)
        torch.cuda.synchronize()
        rep = heap.check_allocations(ptrs, n, 16)
        assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep
        st = heap.status()
        assert n - (1 << 16) <= rep["nulls"] < n, rep
        assert st["flags"] & ob.FLAG_QUEUE_FULL and not st["flags"] & ob.FLAG_TIMEOUT, st
        heap.free(ptrs, n)
        torch.cuda.synchronize()
        _idle(heap, v)


@pytest.mark.parametrize("v", ["VAC", "P"])
def test_batched_path_on_configured_heaps(v):
    n = 1 << 18
    rng = np.random.default_rng(8)
    sizes = torch.from_numpy((np.ceil(np.exp(rng.uniform(np.log(16), np.log(8192), n)) / 16) * 16)
                             .astype(np.uint32).view(np.int32)).cuda()
    cfg = {"agg_width": 16, "page_queue_entries": 1 << 20, "virtual_queue_entries": 512}
    with ob.Ouroboros(v, 4 * GiB, config=cfg) as heap:
        ptrs = _ptrs(n)
        for _ in range(2):
            heap.alloc_batch(sizes, ptrs, n)
            torch.cuda.synchronize()
            rep = heap.check_allocations(ptrs, n, sizes=sizes)
            assert rep["nulls"] == 0 and rep["overlaps"] == 0 and rep["misaligned"] == 0, rep
            heap.free_batch(ptrs, n)
            torch.cuda.synchronize()
            _idle(heap, v)
        assert heap.status()["flags"] == 0


def test_autotune_config_picks_an_accepted_candidate():
    res = ob.autotune_config("VAC", 2 * GiB, 1 << 18, queue_entries=(1 << 16, 1 << 20), agg_widths=(8, 32),
                             blocks=(256, 1024), reps=1)
    pts = res["points"]
    assert len(pts) == 8
    best = res["best"]
    assert best["ok"] and best["mops"] == max(p["mops"] for p in pts if p["ok"])
    assert best["virtual_queue_entries"] in (32, 512) and best["agg_width"] in (8, 32)
