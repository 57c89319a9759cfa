"""The host-buffer entry points (ouro_alloc_host / ouro_free_host): requests
and results in host memory, cut into slices whose copies overlap the other
slices' launches.  The pointers they return obey the same invariants as the
device-buffer path (in the heap, aligned, no overlaps), the device copy equals
the host copy, and after ouro_free_host the heap accounting is idle."""
import numpy as np
import pytest
import torch

import ouroboros_b200 as ob

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _idle(heap):
    rep = heap.check_heap()
    assert rep["bad"] == 0, rep
    for c in range(12):
        assert rep["sem_expected"][c] == 0 and rep["sem_reserved"][c] == 0, (c, rep)
        assert rep["sem_count"][c] == rep["owned_pages"][c], (c, rep)
        assert rep["free_pages_meta"][c] == rep["owned_pages"][c], (c, rep)


def _checked(heap, ptrs_h, n, size=0, sizes_h=None):
    ptrs_d = ptrs_h.to("cuda")
    sizes_d = None if sizes_h is None else torch.from_numpy(np.asarray(sizes_h).astype(np.int32)).to("cuda")
    rep = heap.check_allocations(ptrs_d, n, size, sizes_d)
    assert rep["nulls"] == 0 and rep["out_of_heap"] == 0 and rep["misaligned"] == 0 and rep["overlaps"] == 0, rep
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    ob.write_pattern(ptrs_d, n, size, 5, sizes_d)
    ob.verify_pattern(ptrs_d, n, cnt, size, 5, sizes_d)
    torch.cuda.synchronize()
    assert cnt.tolist() == [0, 0]


@pytest.mark.parametrize("slices", [0, 1, 3, 8])
@pytest.mark.parametrize("v", ob.VARIANTS)
def test_fixed_size_through_host_buffers(v, slices):
    n = (1 << 18) + 5   # slices of unequal length
    size = 256
    stream = torch.cuda.Stream()
    with ob.Ouroboros(v, 2 * GiB) as heap:
        ptrs_h = torch.zeros(n, dtype=torch.int64).pin_memory()
        ptrs_d = torch.zeros(n, dtype=torch.int64, device="cuda")
        for _ in range(2):
            heap.alloc_host(ptrs_h, n, size, out_device=ptrs_d, slices=slices, stream=stream)
            stream.synchronize()
            assert torch.equal(ptrs_h, ptrs_d.cpu())
            _checked(heap, ptrs_h, n, size)
            heap.free_host(ptrs_h, n, slices=slices, stream=stream)
            stream.synchronize()
            _idle(heap)
        assert heap.status()["flags"] == 0


@pytest.mark.parametrize("v", ["P", "VAC", "VLC"])
def test_mixed_sizes_from_pageable_memory(v):
    # per-request sizes in a numpy array (pageable memory), pointers to a numpy array
    n = 300_001
    rng = np.random.default_rng(3)
    sizes = np.exp(rng.uniform(np.log(16), np.log(8192), n)).astype(np.uint32)
    with ob.Ouroboros(v, 4 * GiB) as heap:
        ptrs = np.zeros(n, dtype=np.int64)
        heap.alloc_host(ptrs, n, 0, sizes_host=sizes)
        torch.cuda.synchronize()
        _checked(heap, torch.from_numpy(ptrs), n, 0, sizes)
        heap.free_host(ptrs, n)
        torch.cuda.synchronize()
        _idle(heap)
        assert heap.status()["flags"] == 0


def test_back_to_back_calls_share_the_staging():
    # two allocations queued without a synchronisation between them: the
    # second call's copies wait for the first call's, which read the same
    # device staging; then both sets are freed in one queued sequence
    n = 1 << 18
    stream = torch.cuda.Stream()
    with ob.Ouroboros("VAP", 2 * GiB) as heap:
        a = torch.zeros(n, dtype=torch.int64).pin_memory()
        b = torch.zeros(n, dtype=torch.int64).pin_memory()
        sa = torch.full((n,), 64, dtype=torch.int32).pin_memory()
        sb = torch.full((n,), 1024, dtype=torch.int32).pin_memory()
        heap.alloc_host(a, n, 0, sizes_host=sa, stream=stream)
        heap.alloc_host(b, n, 0, sizes_host=sb, stream=stream)
        stream.synchronize()
        both = torch.cat([a, b])
        sizes = np.concatenate([sa.numpy(), sb.numpy()])
        _checked(heap, both, 2 * n, 0, sizes)
        heap.free_host(a, n, stream=stream)
        heap.free_host(b, n, stream=stream)
        stream.synchronize()
        _idle(heap)


@pytest.mark.parametrize("n,slices", [(1, 8), (10, 8), (7, 3), (33, 0)])
def test_fewer_requests_than_slices(n, slices):
    # slices hold ceil(n / slices) requests, and only as many slices as that
    # takes run (10 requests in 8 wanted slices: 5 slices of 2)
    with ob.Ouroboros("VAP", GiB) as heap:
        ptrs = torch.zeros(n, dtype=torch.int64).pin_memory()
        heap.alloc_host(ptrs, n, 128, slices=slices)
        torch.cuda.synchronize()
        _checked(heap, ptrs, n, 128)
        heap.free_host(ptrs, n, slices=slices)
        torch.cuda.synchronize()
        _idle(heap)
        assert heap.status()["flags"] == 0


def test_reserve_then_calls_of_that_size():
    n = 1 << 17
    with ob.Ouroboros("VLC", GiB) as heap:
        heap.host_reserve(n)
        ptrs = torch.zeros(n, dtype=torch.int64).pin_memory()
        sizes = torch.full((n,), 512, dtype=torch.int32).pin_memory()
        heap.alloc_host(ptrs, n, 0, sizes_host=sizes)
        torch.cuda.synchronize()
        _checked(heap, ptrs, n, 0, sizes.numpy())
        heap.free_host(ptrs, n)
        torch.cuda.synchronize()
        _idle(heap)


def test_arguments_are_checked():
    with ob.Ouroboros("P", GiB) as heap:
        ptrs = torch.zeros(16, dtype=torch.int64).pin_memory()
        heap.alloc_host(ptrs, 0, 64)   # nothing to do
        with pytest.raises(ob.OuroError):
            heap.alloc_host(ptrs, 16, 64, slices=9)
        with pytest.raises(ob.OuroError):
            heap.alloc_host(None, 16, 64)
        with pytest.raises(ob.OuroError):
            heap.free_host(ptrs, 16, block=2048)
        with pytest.raises(ob.OuroError):
            heap.free_host(None, 16)
