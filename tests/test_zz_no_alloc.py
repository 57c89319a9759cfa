"""The allocation-free checker, ouro_check_allocations_noalloc, against the
allocating one, ouro_check_allocations, through the C ABI.

Callers that cannot allocate device memory -- a serving loop that must not let
cudaFree stall its other streams, or a process whose heap already holds nearly
all of HBM -- use the no-alloc entry point, whose ownership bitmap is a fixed
8 MiB array inside the library.  Its reports must equal the allocating
checker's exactly (integer counts), on two calls in a row, including after a
call that left the shared array full of bits.  This file is collected last so
that a run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest
import torch

import ouroboros_b200 as ob

pytestmark = pytest.mark.gpu

FIELDS = ("checked", "nulls", "out_of_heap", "misaligned", "overlaps")


def _noalloc(heap, ptrs, n, sizes, size=0, stream=None):
    rep = torch.full((5,), -1, dtype=torch.int64, device="cuda")   # garbage: the call must clear it
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    rc = ob.lib().ouro_check_allocations_noalloc(heap._handle(), ptrs.data_ptr(), n, size,
                                                 sizes.data_ptr() if sizes is not None else None,
                                                 rep.data_ptr(), stream)
    assert rc == 0, ob.lib().ouro_status_string(rc)
    torch.cuda.synchronize()
    return dict(zip(FIELDS, rep.tolist()))


@pytest.mark.parametrize("v", ["P", "VLC"])
def test_noalloc_checker_matches_allocating_checker(v):
    n = 30000
    rng = np.random.default_rng(11)
    sizes = torch.from_numpy(rng.choice([16, 48, 100, 512, 2048, 8192], n).astype(np.uint32).view(np.int32)).cuda()
    with ob.Ouroboros(v, 1 << 30) as heap:
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        heap.alloc(ptrs, n, sizes=sizes)
        torch.cuda.synchronize()
        # a second pointer set with planted faults: duplicates (overlaps), a
        # null, a misaligned pointer and one outside the heap
        bad = ptrs.clone()
        bad[1000:1500] = ptrs[0:500]
        bad[2000] = 0
        bad[2001] = bad[2001] + 8
        bad[2002] = heap.info()["data_end"] + 4096
        for arr in (bad, bad, ptrs, ptrs):
            want = heap.check_allocations(arr, n, sizes=sizes)
            got = _noalloc(heap, arr, n, sizes)
            assert got == want
        assert want["overlaps"] == 0 and want["checked"] == n
        assert _noalloc(heap, bad, n, sizes)["overlaps"] > 0
        heap.free(ptrs, n)
        torch.cuda.synchronize()


# Heap sizes whose chunk data is exactly the scratch's limit of 131,072 chunks
# (VAP layout), and one chunk more.
AT_LIMIT_BYTES = 1091837824
OVER_LIMIT_BYTES = AT_LIMIT_BYTES + 8320


def test_noalloc_checker_uniform_size_at_the_limit():
    """One size for every pointer (no size array), on a heap whose chunk data
    is exactly the 8 MiB bitmap's reach.  A pointer to the heap's last chunk
    puts bits into the bitmap's last words.  Two calls in a row on a side
    stream, after one that left the array full of bits."""
    with ob.Ouroboros("VAP", AT_LIMIT_BYTES) as heap:
        assert heap.info()["max_chunks"] == 131072
        n = 60000
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        heap.alloc(ptrs, n, 8192)
        torch.cuda.synchronize()
        assert int((ptrs == 0).sum()) == 0
        # the start of the heap's highest chunk: its 8 KiB are the bitmap's
        # last 16 words
        last = torch.tensor([heap.info()["data_end"] - 8192], dtype=torch.int64, device="cuda")
        arr = torch.cat([ptrs, ptrs[:100], last])
        side = torch.cuda.Stream()
        for a in (arr, ptrs, ptrs):
            want = heap.check_allocations(a, a.numel(), 8192)
            with torch.cuda.stream(side):
                got = _noalloc(heap, a, a.numel(), None, size=8192, stream=side.cuda_stream)
            assert got == want
        assert want == {"checked": n, "nulls": 0, "out_of_heap": 0, "misaligned": 0, "overlaps": 0}
        heap.free(ptrs, n)
        torch.cuda.synchronize()
    with ob.Ouroboros("VAP", OVER_LIMIT_BYTES) as heap:
        assert heap.info()["max_chunks"] == 131073
        rep = torch.zeros(5, dtype=torch.int64, device="cuda")
        ptrs = torch.zeros(4, dtype=torch.int64, device="cuda")
        rc = ob.lib().ouro_check_allocations_noalloc(heap._handle(), ptrs.data_ptr(), 4, 16, None,
                                                     rep.data_ptr(), None)
        assert rc == 5


def test_noalloc_checker_refuses_heaps_beyond_its_scratch():
    with ob.Ouroboros("P", 2 << 30) as heap:
        rep = torch.zeros(5, dtype=torch.int64, device="cuda")
        ptrs = torch.zeros(4, dtype=torch.int64, device="cuda")
        sizes = torch.full((4,), 16, dtype=torch.int32, device="cuda")
        rc = ob.lib().ouro_check_allocations_noalloc(heap._handle(), ptrs.data_ptr(), 4, 0, sizes.data_ptr(),
                                                     rep.data_ptr(), None)
        assert rc == 5
        assert b"1 GiB" in ob.lib().ouro_status_string(rc)
