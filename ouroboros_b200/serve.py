"""Serving loop over the allocator: continuous batching of dynamic-graph growth.

Clients send batches of vertex-growth requests (each request frees a vertex's
edge block of 4 x d bytes and allocates one of 8 x d bytes, at most 8 KiB).
The state -- heap and graph -- stays on the device, and so does the loop: a
persistent kernel (``ouro_serve_start``) takes batches from a ring in pinned,
mapped host memory as clients submit them, admits them in arrival order while
the heap's free bytes (computed on the device from allocator state) stay above
a watermark fraction of the heap, and runs the tiles of every admitted batch
side by side on all SMs.  Submitting is a host store, not a CUDA call.  This
module is a thin client: it replays arrivals, submits, polls completions and
reports latencies from the device's own timestamps (seen -> done).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import OURO_ERR_FULL, Ouroboros, ServeConfig, ServeResult, ServeStats, _addr, _check, lib


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
    """Client of the device-resident serving loop (ouro_serve_* of the C ABI)."""

    def __init__(self, graph: Graph, max_inflight: int = 64, watermark: float = 0.10, ring: int = 4096,
                 idle_seconds: float = 10.0, blocks_per_sm: int = 0):
        self.g = graph
        # the loop occupies the device until it is stopped: pending work is
        # finished first, and nothing while it runs may synchronize the device
        torch.cuda.synchronize()
        cfg = ServeConfig(int(ring), int(max_inflight), int(blocks_per_sm), float(watermark), float(idle_seconds))
        h = ctypes.c_void_p()
        _check(lib().ouro_serve_start(graph.heap._handle(), _addr(graph.vptr), _addr(graph.degree), graph.nv,
                                      graph.seed, ctypes.byref(cfg), ctypes.byref(h)), "ouro_serve_start")
        self._s = h
        self._buf = (ServeResult * 1024)()
        self._live = {}        # seq -> vertices tensor (kept alive until the batch is done)
        self.done = []
        self.stats = None

    def submit(self, vertices: torch.Tensor, client: int = 0):
        """Submit one batch; returns its sequence number, or None when the ring is full."""
        seq = ctypes.c_uint64()
        rc = lib().ouro_serve_submit(self._s, _addr(vertices), vertices.numel(), int(client), ctypes.byref(seq))
        if rc == OURO_ERR_FULL:
            return None
        _check(rc, "ouro_serve_submit")
        self._live[int(seq.value)] = vertices
        return int(seq.value)

    def poll(self) -> int:
        """Collect finished batches; returns how many came in."""
        got = ctypes.c_uint32()
        total = 0
        while True:
            _check(lib().ouro_serve_poll(self._s, self._buf, len(self._buf), ctypes.byref(got)), "ouro_serve_poll")
            for i in range(got.value):
                r = self._buf[i]
                self._live.pop(int(r.seq), None)
                self.done.append({f: getattr(r, f) for f, _ in ServeResult._fields_})
            total += got.value
            if got.value < len(self._buf):
                return total

    def stop(self) -> dict:
        st = ServeStats()
        rc = lib().ouro_serve_stop(self._s, ctypes.byref(st))
        self.poll()
        self.stats = {f: getattr(st, f) for f, _ in ServeStats._fields_}
        if rc not in (0, 4):
            _check(rc, "ouro_serve_stop")
        return self.stats

    def close(self):
        if self._s:
            lib().ouro_serve_close(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, batches, poll_s: float = 20e-6) -> dict:
        """batches: list of (arrival_s, client, vertices tensor on the device),
        sorted by arrival (all at 0 for a saturating load).  Submits each at its
        arrival time, polls completions meanwhile, stops after the last one and
        reports latencies from the device timestamps (seen -> done).  The
        batches' vertex tensors must be ready on the caller's stream; only that
        stream is synchronized (a device-wide synchronize would wait for the
        loop itself)."""
        torch.cuda.current_stream().synchronize()
        requests = sum(int(b[2].numel()) for b in batches)
        t0 = time.perf_counter()
        full_waits = 0
        for arr, client, verts in batches:
            while time.perf_counter() - t0 < arr:
                if not self.poll():
                    time.sleep(poll_s)
            while self.submit(verts, client) is None:
                full_waits += 1
                if not self.poll():
                    time.sleep(poll_s)
        deadline = time.perf_counter() + 120.0
        while len(self.done) < len(batches) and time.perf_counter() < deadline:
            if not self.poll():
                time.sleep(poll_s)
        stats = self.stop()
        wall = time.perf_counter() - t0
        d = self.done
        lat = np.array([(r["t_done_ns"] - r["t_seen_ns"]) * 1e-6 for r in d]) if d else np.zeros(0)
        queue = np.array([(r["t_start_ns"] - r["t_seen_ns"]) * 1e-6 for r in d]) if d else np.zeros(0)
        span_s = (max(r["t_done_ns"] for r in d) - min(r["t_seen_ns"] for r in d)) * 1e-9 if d else 0.0
        done_requests = sum(r["n"] for r in d)
        # batches running at once on the device: the most [start, done] intervals that overlap
        ev = sorted([(r["t_start_ns"], 1) for r in d] + [(r["t_done_ns"], -1) for r in d])
        peak = cur = 0
        for _, step in ev:
            cur += step
            peak = max(peak, cur)
        return {
            "batches": len(d), "requests": done_requests, "wall_s": wall, "device_span_s": span_s,
            "ops_per_s": 2.0 * done_requests / span_s if span_s > 0 else None,   # a request: one free, one malloc
            "batches_per_s": len(d) / span_s if span_s > 0 else None,
            "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
            "queue_p50_ms": float(np.percentile(queue, 50)) if queue.size else None,
            "queue_p99_ms": float(np.percentile(queue, 99)) if queue.size else None,
            "held_back": int(stats["held_back"]), "left_pending": len(batches) - len(d),
            "ring_full_waits": full_waits, "loop_status": int(stats["status"]), "peak_inflight": peak,
            "failed_allocs": int(sum(r["failed_allocs"] for r in d)),
            "lock_giveups": int(sum(r["lock_giveups"] for r in d)),
            "offered_requests": requests,
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
