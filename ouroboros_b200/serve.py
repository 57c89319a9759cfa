"""Serving loop over the allocator: continuous batching of dynamic-graph growth.

Clients send batches of vertex-growth requests (each request frees a vertex's
edge block of 4 x d bytes and allocates one of 8 x d bytes, at most 8 KiB,
through ``ouro_graph_grow``).  The state -- heap and graph -- stays on the
device.  The scheduler admits batches as they arrive into a fixed number of
stream slots, so batches that arrive while others run start as soon as a slot
is free and their kernels overlap on the GPU; a client's next batch waits for
its previous one.  Admission is deferred while the heap's free bytes -- read
from allocator state by a small kernel on a side stream and copied to pinned
host memory asynchronously, never synchronizing the device -- are below a
watermark fraction of the heap.
Latency of a batch = completion (its stream event seen done) - arrival.
"""
from __future__ import annotations

import collections
import time

import numpy as np
import torch

from . import Ouroboros, _addr, _check, lib


class Graph:
    """A power-law graph whose adjacency lists live in an Ouroboros heap."""

    def __init__(self, heap: Ouroboros, num_vertices: int, seed: int = 1, alpha: float = 2.1, stream=None):
        self.heap, self.nv, self.seed = heap, int(num_vertices), int(seed)
        self.vptr = torch.zeros(self.nv, dtype=torch.int64, device="cuda")
        self.degree = torch.zeros(self.nv, dtype=torch.int32, device="cuda")
        self.failed = torch.zeros(2, dtype=torch.int64, device="cuda")
        scratch = torch.empty(self.nv, dtype=torch.int32, device="cuda")
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _check(lib().ouro_graph_init(heap._handle(), _addr(self.vptr), _addr(self.degree), _addr(scratch), self.nv,
                                     self.seed, float(alpha), _addr(self.failed), s), "ouro_graph_init")
        torch.cuda.synchronize()
        del scratch

    def grow(self, vertices: torch.Tensor, stream=None):
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        _check(lib().ouro_graph_grow(self.heap._handle(), _addr(self.vptr), _addr(self.degree), _addr(vertices),
                                     vertices.numel(), self.nv, self.seed, _addr(self.failed), s), "ouro_graph_grow")

    def check(self, vertices: torch.Tensor) -> tuple[int, int]:
        """(checksum of the vertices' edges, vertices whose edges break the recipe)."""
        out = torch.zeros(2, dtype=torch.int64, device="cuda")
        _check(lib().ouro_graph_check(_addr(self.vptr), _addr(self.degree), _addr(vertices), vertices.numel(), self.nv,
                                      self.seed, _addr(out), torch.cuda.current_stream().cuda_stream),
               "ouro_graph_check")
        torch.cuda.synchronize()
        s, bad = out.tolist()
        return s & (2**64 - 1), bad


class Server:
    """Continuous batching of graph-growth batches into `slots` streams."""

    def __init__(self, graph: Graph, slots: int = 16, watermark: float = 0.10):
        self.g, self.slots, self.watermark = graph, int(slots), float(watermark)
        self.streams = [torch.cuda.Stream() for _ in range(self.slots)]
        self.query_stream = torch.cuda.Stream()
        self.free_bytes_dev = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.free_bytes = torch.zeros(1, dtype=torch.int64).pin_memory()   # copied from the device, no sync
        self.heap_bytes = graph.heap.info()["heap_bytes"]

    def _refresh_free_bytes(self):
        _check(lib().ouro_free_bytes_to(self.g.heap._handle(), _addr(self.free_bytes_dev),
                                        self.query_stream.cuda_stream), "ouro_free_bytes_to")
        with torch.cuda.stream(self.query_stream):
            self.free_bytes.copy_(self.free_bytes_dev, non_blocking=True)

    def run(self, batches, poll_s: float = 20e-6) -> dict:
        """batches: list of (arrival_s, client, vertices tensor on the device),
        sorted by arrival.  Returns latencies and counters."""
        pending = collections.deque()
        arrivals = collections.deque(batches)
        free_slots = list(range(self.slots))
        busy_clients = set()
        inflight = {}   # slot -> (event, arrival, client, requests)
        lat, requests, deferred, peak = [], 0, 0, 0
        self._refresh_free_bytes()
        t0 = time.perf_counter()
        while arrivals or pending or inflight:
            now = time.perf_counter() - t0
            while arrivals and arrivals[0][0] <= now:
                pending.append(arrivals.popleft())
            for slot, (ev, arr, client, nreq) in list(inflight.items()):
                if ev.query():
                    lat.append(time.perf_counter() - t0 - arr)
                    requests += nreq
                    busy_clients.discard(client)
                    free_slots.append(slot)
                    del inflight[slot]
            self._refresh_free_bytes()
            held = False
            for _ in range(len(pending)):
                if not free_slots:
                    break
                arr, client, verts = pending[0]
                if client in busy_clients:   # a client's batches run in order
                    pending.rotate(-1)
                    continue
                if int(self.free_bytes[0]) < self.watermark * self.heap_bytes:
                    held = True
                    break
                pending.popleft()
                slot = free_slots.pop()
                st = self.streams[slot]
                self.g.grow(verts, stream=st)
                ev = torch.cuda.Event()
                ev.record(st)
                inflight[slot] = (ev, arr, client, verts.numel())
                busy_clients.add(client)
            deferred += int(held)
            peak = max(peak, len(inflight))
            if held and not inflight:
                break   # the heap stays below the watermark: nothing in flight can free memory
            if not inflight or not free_slots:
                time.sleep(poll_s)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        lat_ms = np.array(lat) * 1e3
        failed = self.g.failed.tolist()
        return {
            "batches": len(lat), "requests": requests, "wall_s": wall,
            "ops_per_s": 2.0 * requests / wall,   # each request is one free and one malloc
            "p50_ms": float(np.percentile(lat_ms, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat_ms, 99)) if len(lat) else None,
            "deferred_polls": deferred, "peak_inflight": peak, "left_pending": len(pending) + len(arrivals),
            "failed_allocs": failed[0], "lock_giveups": failed[1],
        }


def poisson_batches(num_clients: int, rate_per_s: float, duration_s: float, nv: int, lo: int, hi: int, seed: int):
    """Arrivals of `num_clients` clients, each a Poisson process (the total
    rate is rate_per_s); batch sizes log-uniform in [lo, hi]; vertices drawn
    uniformly (the growth kernel serialises repeats)."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(num_clients):
        t = 0.0
        while True:
            t += rng.exponential(num_clients / rate_per_s)
            if t >= duration_s:
                break
            size = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
            out.append((t, c, size, int(rng.integers(0, 2**62))))
    out.sort()
    batches = []
    gen = torch.Generator(device="cuda")
    for t, c, size, s in out:
        gen.manual_seed(s)
        verts = torch.randint(0, nv, (size,), generator=gen, device="cuda", dtype=torch.int64).to(torch.int32)
        batches.append((t, c, verts))
    torch.cuda.synchronize()
    return batches
