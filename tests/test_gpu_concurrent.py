"""Concurrent correctness of the per-thread path: every pointer in the heap and
aligned to its size class, no two live allocations overlapping (ownership
bitmap + seeded pattern), and after all frees the heap accounting back at its
idle state (every owned page free and queued, no expected or reserved pages,
chunk bitmasks full)."""
import numpy as np
import pytest
import torch

import oracle
import ouroboros_b200 as ob

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _ptrs(n):
    return torch.zeros(n, dtype=torch.int64, device="cuda")


def _idle(heap, v):
    rep = heap.check_heap()
    assert rep["bad"] == 0, rep
    for c in range(12):
        assert rep["sem_expected"][c] == 0 and rep["sem_reserved"][c] == 0, (c, rep)
        assert rep["sem_count"][c] == rep["owned_pages"][c], (c, rep["sem_count"][c], rep["owned_pages"][c])
        assert rep["free_pages_meta"][c] == rep["owned_pages"][c], (c, rep["free_pages_meta"][c], rep["owned_pages"][c])
    return rep


def _round(heap, ptrs, n, size=0, sizes=None, seed=1):
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    heap.alloc(ptrs, n, size, sizes)
    torch.cuda.synchronize()
    rep = heap.check_allocations(ptrs, n, size, sizes)
    ob.write_pattern(ptrs, n, size, seed, sizes)
    ob.verify_pattern(ptrs, n, cnt, size, seed, sizes)
    torch.cuda.synchronize()
    nulls, bad = cnt.tolist()
    heap.free(ptrs, n)
    torch.cuda.synchronize()
    return rep, nulls, bad


@pytest.mark.parametrize("size", [16, 64, 100, 1024, 8192, 16384, 32768])
@pytest.mark.parametrize("v", ob.VARIANTS)
def test_fixed_size_rounds(v, size):
    n = 1 << 16
    if size > 8192:
        n = 1 << 13
    with ob.Ouroboros(v, GiB) as heap:
        ptrs = _ptrs(n)
        for r in range(3):
            rep, nulls, bad = _round(heap, ptrs, n, size, seed=r + 7)
            assert nulls == 0 and bad == 0, (r, nulls, bad)
            assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep
            _idle(heap, v)
        assert heap.status()["flags"] == 0


@pytest.mark.parametrize("v", ob.VARIANTS)
def test_mixed_sizes(v):
    n = 1 << 16
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(0, np.log(32768), n)).astype(np.uint32)
    d_sizes = torch.from_numpy(sizes.astype(np.int32)).cuda()
    with ob.Ouroboros(v, 2 * GiB) as heap:
        ptrs = _ptrs(n)
        for r in range(3):
            rep, nulls, bad = _round(heap, ptrs, n, sizes=d_sizes, seed=r)
            assert nulls == 0 and bad == 0, (r, nulls, bad)
            assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep
            _idle(heap, v)
        assert heap.status()["flags"] == 0


@pytest.mark.parametrize("v", ["P", "C"])
def test_out_of_memory_exact_count(v):
    # A heap of a few hundred chunks, asked for more 8 KiB pages than it has:
    # exactly max_chunks - 1 requests succeed (the reference's bound
    # index + 1 < maxChunks), the rest get nullptr; freeing restores the heap.
    heap_bytes = oracle.layout(v, GiB)["total_required"] + 300 * 8320
    with ob.Ouroboros(v, heap_bytes) as heap:
        mc = heap.info()["max_chunks"]
        n = 4096
        ptrs = _ptrs(n)
        for r in range(2):
            rep, nulls, bad = _round(heap, ptrs, n, 8192, seed=r)
            assert n - nulls == mc - 1, (n - nulls, mc)
            assert bad == 0 and rep["overlaps"] == 0
            _idle(heap, v)
        st = heap.status(clear=True)
        assert st["flags"] == ob.FLAG_OOM and st["null_results"] == 2 * (n - (mc - 1))


def _budget_chunks(v, mc, ppc):
    """Data chunks a virtualized heap of mc chunks grants one class before its
    chunk budget is spent: budget = data chunks + the queue chunks for the
    class's entries (pages, or three per chunk for chunk queues) + per class one
    initial queue chunk and a margin (4 for array queues, 14 for linked)."""
    margin = 4 if v.startswith("VA") else 14
    committed = 12 * (1 + margin)
    per = ppc if v.endswith("P") else 3
    m = 0
    while committed + (m + 1) + -(-(m + 1) * per // 2048) <= mc - 1:
        m += 1
    return m


@pytest.mark.parametrize("size", [8192, 4096])
@pytest.mark.parametrize("v", ["VAP", "VAC", "VLP", "VLC"])
def test_out_of_memory_virtualized(v, size):
    # Queue chunks come from the same pool as data chunks: the budget stops a
    # class from taking the chunks its queue still needs, so running out of
    # memory ends in nullptr results, never in a wait that times out.
    heap_bytes = oracle.layout(v, GiB)["total_required"] + 400 * 8320
    ppc = 8192 // size
    with ob.Ouroboros(v, heap_bytes) as heap:
        mc = heap.info()["max_chunks"]
        n = 4096
        cap = _budget_chunks(v, mc, ppc) * ppc
        ptrs = _ptrs(n)
        oks = []
        for r in range(3):
            rep, nulls, bad = _round(heap, ptrs, n, size, seed=r)
            ok = n - nulls
            oks.append(ok)
            # one group of 32 may find the budget momentarily full; the budget's
            # queue-chunk term is computed on reserved page counts that may still
            # hold releases in flight, so it can be one queue chunk short (the
            # per-class margin absorbs that): at most one chunk's pages above cap
            assert cap - 32 * ppc <= ok <= cap + ppc, (r, ok, cap, mc)
            assert bad == 0 and rep["overlaps"] == 0 and rep["misaligned"] == 0
            _idle(heap, v)
        assert oks[1] == oks[2], oks
        st = heap.status(clear=True)
        assert st["flags"] == ob.FLAG_OOM and st["timeouts"] == 0, st


@pytest.mark.parametrize("size", [16, 32, 64])
@pytest.mark.parametrize("v", ["VAP", "VLP"])
def test_burst_grows_past_one_queue_chunk(v, size):
    # 2^20 threads on a cold heap: the semaphore elects groups to grow many
    # chunks at once (waiting groups' reservations add to the deficit), so one
    # publish covers more than two 2048-entry queue chunks.  Every wait must
    # end and every page must be handed out exactly once.
    n = 1 << 20
    with ob.Ouroboros(v, 4 * GiB) as heap:
        ptrs = _ptrs(n)
        for r in range(3):
            rep, nulls, bad = _round(heap, ptrs, n, size, seed=r + 3)
            assert nulls == 0 and bad == 0, (r, nulls, bad)
            assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep
            _idle(heap, v)
        st = heap.status()
        assert st["flags"] == 0 and st["timeouts"] == 0, st


@pytest.mark.parametrize("v,reps", [("C", 72), ("VAC", 140), ("VLC", 40)])
def test_chunk_queue_wraps_around(v, reps):
    # Bursts of 2^20 requests of 2 KiB: every free phase re-enqueues 262,144
    # chunks, so the back of the class's queue moves 262,144 positions per
    # burst.  The standard ring (2^23 entries) wraps every 32 bursts and the
    # virtualized-array index (16,384 queue chunks of 2048 entries) every 128;
    # the front passes fully removed ring segments and queue chunks on their
    # removal counts, which must start every lap clean.  Checked rounds along
    # the way: every page handed out once, every wait ended.
    n, size, cls = 1 << 20, 2048, 7
    with ob.Ouroboros(v, 4 * GiB) as heap:
        ptrs = _ptrs(n)
        back0 = int(heap.state()[7 + 12 * cls + 4])
        for r in range(reps):
            if r % 16 == 15 or r == reps - 1:
                rep, nulls, bad = _round(heap, ptrs, n, size, seed=r)
                assert nulls == 0 and bad == 0, (r, nulls, bad)
                assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, (r, rep)
            else:
                heap.alloc(ptrs, n, size)
                heap.free(ptrs, n)
        torch.cuda.synchronize()
        moved = int(heap.state()[7 + 12 * cls + 4]) - back0
        laps = {"C": 1 << 23, "VAC": 16384 * 2048, "VLC": 0}[v]
        assert moved > laps, (moved, laps)
        st = heap.status()
        assert st["flags"] == 0 and st["timeouts"] == 0, st
        _idle(heap, v)


@pytest.mark.parametrize("v", ob.VARIANTS)
def test_free_resources_accounting(v):
    # free bytes = free pages x page size + chunks never handed out or pooled
    # x 8 KiB: an allocation of n pages of one class takes exactly n x page
    # size (plus, for the virtualized variants, the queue chunks it needed)
    # and freeing them gives it all back
    size, n = 256, 1 << 16
    with ob.Ouroboros(v, GiB) as heap:
        r0 = heap.free_resources()
        assert r0["chunks_in_use"] == (0 if v in ("P", "C") else 12)   # one queue chunk per class
        assert r0["free_bytes"] == (r0["heap_chunks"] - r0["chunks_in_use"]) * 8192
        ptrs = _ptrs(n)
        heap.alloc(ptrs, n, size)
        torch.cuda.synchronize()
        r1 = heap.free_resources()
        assert r1["page_size"][4] == 256 and r1["free_pages"][4] >= 0
        extra = r0["free_bytes"] - r1["free_bytes"] - n * size   # queue chunks the entries needed
        assert extra % 8192 == 0 and 0 <= extra // 8192 <= (0 if v in ("P", "C") else 64), (r0, r1)
        heap.free(ptrs, n)
        torch.cuda.synchronize()
        r2 = heap.free_resources()
        back = r2["free_bytes"] - r1["free_bytes"]    # the pages, less queue chunks the frees needed
        assert back % 8192 == 0 and 0 <= (n * size - back) // 8192 <= (0 if v in ("P", "C") else 64), (r1, r2)
        assert r2["free_pages"][4] == r1["free_pages"][4] + n and r2["queue_entries"][4] > 0


@pytest.mark.parametrize("v", ob.VARIANTS)
def test_prefill_serves_a_burst_without_new_chunks(v):
    # preFillQueue at scale: the class's pages are published up front, so the
    # burst that follows takes no new data chunk
    size, n = 128, 1 << 18
    with ob.Ouroboros(v, GiB) as heap:
        added = heap.prefill(size, n)
        assert added == n, added                       # 128 B: 64 pages per chunk, n a multiple
        r = heap.free_resources()
        assert r["free_pages"][3] == n and r["queue_entries"][3] == (n if v.endswith("P") else n // 64)
        used = r["chunks_in_use"]
        ptrs = _ptrs(n)
        rep, nulls, bad = _round(heap, ptrs, n, size, seed=5)
        assert nulls == 0 and bad == 0 and rep["overlaps"] == 0 and rep["misaligned"] == 0
        r2 = heap.free_resources()
        assert r2["chunks_in_use"] - used <= (0 if v in ("P", "C") else 32), (used, r2["chunks_in_use"])
        assert r2["free_pages"][3] == n
        _idle(heap, v)
        assert heap.status()["flags"] == 0
        with pytest.raises(ob.OuroError):
            heap.prefill(1 << 20, 1)                  # above 32 KiB: the CUDA device heap's
