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


def _noalloc(heap, ptrs, n, sizes):
    rep = torch.full((5,), -1, dtype=torch.int64, device="cuda")   # garbage: the call must clear it
    stream = torch.cuda.current_stream().cuda_stream
    rc = ob.lib().ouro_check_allocations_noalloc(heap._handle(), ptrs.data_ptr(), n, 0, sizes.data_ptr(),
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


def test_noalloc_checker_refuses_heaps_beyond_its_scratch():
    with ob.Ouroboros("P", 2 << 30) as heap:
        rep = torch.zeros(5, dtype=torch.int64, device="cuda")
        ptrs = torch.zeros(4, dtype=torch.int64, device="cuda")
        sizes = torch.full((4,), 16, dtype=torch.int32, device="cuda")
        rc = ob.lib().ouro_check_allocations_noalloc(heap._handle(), ptrs.data_ptr(), 4, 0, sizes.data_ptr(),
                                                     rep.data_ptr(), None)
        assert rc == 5
        assert b"1 GiB" in ob.lib().ouro_status_string(rc)
