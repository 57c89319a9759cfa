"""The batched path: persistent alloc / free / churn kernels with shared-memory
binning by size class.  Same invariants as the per-thread path: every pointer
in the heap and aligned to its class, no two live allocations overlapping
(ownership bitmap + seeded pattern), and after all frees the accounting back
at idle."""
import numpy as np
import pytest
import torch

import ouroboros_b200 as ob
from tests.test_gpu_concurrent import _idle, _ptrs

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _loguniform(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.uint32)
    return torch.from_numpy(s.astype(np.int32)).cuda()


def _check_live(heap, ptrs, sizes, n, seed):
    rep = heap.check_allocations(ptrs, n, sizes=sizes)
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    ob.write_pattern(ptrs, n, 0, seed, sizes)
    ob.verify_pattern(ptrs, n, cnt, 0, seed, sizes)
    torch.cuda.synchronize()
    nulls, bad = cnt.tolist()
    assert nulls == 0 and bad == 0, (nulls, bad)
    assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0, rep


@pytest.mark.parametrize("block", [128, 256])
@pytest.mark.parametrize("v", ob.VARIANTS)
def test_batch_alloc_free_mixed_sizes(v, block):
    n = 1 << 18
    sizes = _loguniform(n, 16, 32768, seed=3)
    with ob.Ouroboros(v, 2 * GiB) as heap:
        ptrs = _ptrs(n)
        for r in range(2):
            heap.alloc_batch(sizes, ptrs, n, block=block)
            torch.cuda.synchronize()
            _check_live(heap, ptrs, sizes, n, seed=r + 11)
            heap.free_batch(ptrs, n, block=block)
            torch.cuda.synchronize()
            _idle(heap, v)
        assert heap.status()["flags"] == 0


@pytest.mark.parametrize("dist,frac", [(("loguniform", 16, 8192), 500), (("zipf", 1.2), 300)])
@pytest.mark.parametrize("v", ["C", "VAC", "VLC", "VLP"])
def test_batch_churn_cycles(v, dist, frac):
    # a live set churned by realloc cycles stays consistent cycle after cycle
    n = 1 << 17
    with ob.Ouroboros(v, 2 * GiB) as heap:
        ptrs = _ptrs(n)
        sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
        heap.realloc_batch(ptrs, sizes, n, seed=7, cycle=0, fraction_permille=1000, dist=dist)   # initial live set
        for cycle in range(1, 9):
            heap.realloc_batch(ptrs, sizes, n, seed=7, cycle=cycle, fraction_permille=frac, dist=dist)
            if cycle % 4 == 0:
                torch.cuda.synchronize()
                _check_live(heap, ptrs, sizes, n, seed=cycle)
        torch.cuda.synchronize()
        s = sizes.cpu().numpy().view(np.uint32)
        assert s.min() >= 16 and s.max() <= 8192 and np.all(s % 16 == 0)
        heap.free_batch(ptrs, n)
        torch.cuda.synchronize()
        _idle(heap, v)
        assert heap.status()["flags"] == 0


def test_batch_realloc_picks_the_requested_fraction():
    n = 1 << 18
    with ob.Ouroboros("VAC", GiB) as heap:
        ptrs = _ptrs(n)
        sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
        heap.realloc_batch(ptrs, sizes, n, seed=1, cycle=0, fraction_permille=1000, dist=("loguniform", 16, 16))
        torch.cuda.synchronize()
        assert int((sizes == 16).sum()) == n
        heap.realloc_batch(ptrs, sizes, n, seed=1, cycle=1, fraction_permille=300, dist=("loguniform", 32, 32))
        torch.cuda.synchronize()
        picked = int((sizes == 32).sum())
        assert abs(picked / n - 300 / 1024 * 1024 / 1000) < 0.01, picked
        heap.free_batch(ptrs, n)
        torch.cuda.synchronize()
        _idle(heap, "VAC")


def test_batch_autotune_picks_a_shape():
    with ob.Ouroboros("VAC", GiB) as heap:
        best = heap.autotune_batch(n=1 << 16, lo=16, hi=8192)
        assert best["block"] in (128, 256, 512, 1024) and best["blocks_per_sm"] in (0, 1, 2, 4)
        assert best["mops"] > 0
        _idle(heap, "VAC")
        n = 1 << 16
        sizes = _loguniform(n, 16, 8192, seed=9)
        ptrs = _ptrs(n)
        heap.alloc_batch(sizes, ptrs, n)   # the tuned shape
        torch.cuda.synchronize()
        _check_live(heap, ptrs, sizes, n, seed=4)
        heap.free_batch(ptrs, n)
        torch.cuda.synchronize()
        assert heap.status()["flags"] == 0
