"""The multi-GPU path of bench.py runs one independent replica per rank (the
allocator has no exchange step).  Its only collective is the MAX all-reduce of
the ranks' kernel times; the job value is all ranks' operations over the
slowest rank's time.  Checked here with two gloo ranks on CPU."""
import os
import sys

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        total_ms = 10.0 if rank == 0 else 25.0          # rank 1 is the slow one
        e2e_ms = 40.0 if rank == 0 else 30.0
        value, t, e = bench.replica_value(total_ms, e2e_ms, ops_per_rank=1e6, world=world, dist=dist, device="cpu")
        q.put((rank, value, t, e))
    finally:
        dist.destroy_process_group()


def test_replica_value_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, value, t, e in out:
        assert t == 25.0 and e == 40.0                  # MAX over ranks
        assert abs(value - 2e6 / 25e-3 / 1e6) < 1e-9    # both ranks' ops over the slowest time


def test_replica_value_single_rank():
    sys.path.insert(0, ROOT)
    import bench
    value, t, e = bench.replica_value(10.0, 5.0, ops_per_rank=1e6, world=1)
    assert (t, e) == (10.0, 5.0) and abs(value - 100.0) < 1e-9
