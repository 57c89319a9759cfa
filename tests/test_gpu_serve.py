"""The serving loop: continuous batching of dynamic-graph growth batches by
the device-resident loop (ouro_serve_*).

Each batch's result -- the edge blocks of the vertices it grew -- must be the
same when the batch runs alone and when it runs in the mix with the others,
admitted concurrently by the loop (exact: integer content checksums); the heap
holds no overlapping or misplaced block afterwards.  A C++ client drives the
same loop through the C ABI."""
import os
import subprocess

import pytest
import torch

import ouroboros_b200 as ob
from ouroboros_b200 import serve

pytestmark = pytest.mark.gpu

GiB = 1 << 30


def _batches(nv, sizes, seed):
    perm = torch.randperm(nv, generator=torch.Generator().manual_seed(seed)).to(torch.int32).cuda()
    out, o = [], 0
    for k, n in enumerate(sizes):
        out.append((0.0, k, perm[o:o + n].contiguous()))   # disjoint vertex sets
        o += n
    return out


@pytest.mark.parametrize("v", ["VAP", "P", "VLC"])
def test_each_batch_same_alone_and_in_the_mix(v):
    nv = 1 << 17
    sizes = [1000, 3000, 5000, 8000, 12000, 2000, 7000, 4000, 9000, 6000, 11000, 1500]
    batches = _batches(nv, sizes, seed=3)
    # alone: one batch at a time on the device
    with ob.Ouroboros(v, 2 * GiB) as heap:
        g = serve.Graph(heap, nv, seed=5)
        alone = []
        for _, _, verts in batches:
            g.grow(verts)
            torch.cuda.synchronize()
            alone.append(g.check(verts))
        assert g.failed.tolist() == [0, 0]
    # in the mix: all arrive at once and run concurrently in 8 slots, three times
    with ob.Ouroboros(v, 2 * GiB) as heap:
        g = serve.Graph(heap, nv, seed=5)
        srv = serve.Server(g, max_inflight=8, watermark=0.05)
        rep = srv.run(batches)
        srv.close()
        assert rep["batches"] == len(batches) and rep["left_pending"] == 0 and rep["loop_status"] == 0, rep
        assert rep["peak_inflight"] > 1, rep
        assert rep["failed_allocs"] == 0 and rep["lock_giveups"] == 0, rep
        mixed = [g.check(verts) for _, _, verts in batches]
        assert mixed == alone
        for s, bad in mixed:
            assert bad == 0
        # every vertex's block: in the heap, aligned, not overlapping another
        sizes_t = (g.degree.to(torch.int64) * 4).to(torch.int32)
        rep = heap.check_allocations(g.vptr, nv, sizes=sizes_t)
        assert rep["overlaps"] == 0 and rep["misaligned"] == 0 and rep["out_of_heap"] == 0 and rep["nulls"] == 0
        assert heap.status()["flags"] == 0


def test_repeated_vertices_are_serialised():
    # the same vertex named many times within and across concurrent batches:
    # its final degree reflects every growth, its edges follow the recipe
    nv = 1 << 12
    with ob.Ouroboros("VAP", GiB) as heap:
        g = serve.Graph(heap, nv, seed=9)
        d0 = g.degree.clone()
        verts = torch.arange(nv, dtype=torch.int32, device="cuda").repeat(2)   # each vertex twice
        batches = [(0.0, k, verts) for k in range(3)]
        srv = serve.Server(g, max_inflight=3, watermark=0.0)
        rep = srv.run(batches)
        srv.close()
        assert rep["batches"] == 3 and rep["lock_giveups"] == 0 and rep["failed_allocs"] == 0, rep
        expect = torch.clamp(d0.to(torch.int64) * 64, max=2048)   # six doublings, capped
        assert torch.equal(g.degree.to(torch.int64), expect)
        s, bad = g.check(torch.arange(nv, dtype=torch.int32, device="cuda"))
        assert bad == 0


def test_watermark_holds_batches_back():
    # A heap that the graph fills past the watermark: admission waits while
    # a batch runs, every batch still completes (one is always admitted when
    # none runs), and the held-back batches are counted.
    nv = 1 << 16
    with ob.Ouroboros("VAP", GiB) as heap:
        g = serve.Graph(heap, nv, seed=11)
        free_frac = heap.free_resources()["free_bytes"] / heap.info()["heap_bytes"]
        batches = _batches(nv, [4000] * 16, seed=4)
        srv = serve.Server(g, max_inflight=16, watermark=min(0.99, free_frac + 0.05))
        rep = srv.run(batches)
        srv.close()
        assert rep["batches"] == 16 and rep["left_pending"] == 0, rep
        assert rep["held_back"] > 0 and rep["peak_inflight"] == 1, rep


HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLIENT = os.path.join(ROOT, "ouroboros_b200", "_lib", "serve_client")


def test_cpp_client_through_the_c_abi():
    from ouroboros_b200 import build
    lib = build.build()
    src = os.path.join(HERE, "serve", "serve_client.cpp")
    if not os.path.exists(CLIENT) or os.path.getmtime(CLIENT) < max(os.path.getmtime(lib), os.path.getmtime(src)):
        cmd = [build.nvcc(), "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), src, "-L", os.path.dirname(lib),
               "-louroboros_b200", f"-Xlinker=-rpath,{os.path.dirname(lib)}", "-o", CLIENT]
        res = subprocess.run(cmd, capture_output=True, text=True)
        assert res.returncode == 0, res.stderr[-3000:]
    res = subprocess.run([CLIENT], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert '"ok": true' in res.stdout, res.stdout
