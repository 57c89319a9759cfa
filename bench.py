#!/usr/bin/env python
"""Alloc+free throughput of the Ouroboros allocator on B200.

Workload (the all-six-instantiations configuration): every instantiation
(P, C, VAP, VAC, VLP, VLC) on a 4 GiB heap; one launch of 2^20 threads, each
mallocs one fixed size, then (untimed) a seeded uint32 pattern is written and
verified, then one launch frees everything.  Sizes are the powers of two
16 B .. 2048 B: the reference runs out of chunks at 4096 B and 8192 B
(2^20 x 4 KiB exceeds a 4 GiB heap), so those cells are timed for this build
only and reported under "extra".  A step is one pass over the 48 cells; the
metric is (mallocs + frees) / (alloc kernel time + free kernel time), timed with
CUDA events around each launch as src/main.cu:146-164 of the reference does,
with L2 flushed (256 MiB written) before every timed launch.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference runs the reference's own CUDA code (oracle/_ref, built from the
reference's sources for sm_100a) on the same cells, launch shape and timing.
Under torchrun every rank runs its own replica (the allocator does not shard);
value sums ranks over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# Load every kernel's module when the context is created, not at its first
# launch: otherwise the first (cold) repetition of each cell would include
# loading the alloc/free kernels of its instantiation, in both arms.
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

import numpy as np  # noqa: E402
import torch  # noqa: E402

VARIANTS = ("P", "C", "VAP", "VAC", "VLP", "VLC")
HEADLINE_SIZES = (16, 32, 64, 128, 256, 512, 1024, 2048)
EXTRA_SIZES = (4096, 8192)
GiB = 1 << 30
SEED = 0x9E3779B9
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "roofline_traffic.json")
REFERENCE_CELLS = os.path.join(ROOT, "profiles", "reference_cells.json")
# Instantiations whose reference code faulted on the GPU on a cell of this
# benchmark that its capacity model admits; the reference arm does not run
# them again.
REFERENCE_FAULTED = {
    "VAC": "the reference's own code raised 'an illegal memory access was encountered' on the VAC 1024 B cell "
           "(2^20 threads, 4 GiB heap, 131,072 of 516,064 chunks needed); its VAC code also faulted on the "
           "batched trace; it is not run again",
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--variants", default=",".join(VARIANTS))
    ap.add_argument("--sizes", default=",".join(map(str, HEADLINE_SIZES)))
    ap.add_argument("--extra-sizes", default=",".join(map(str, EXTRA_SIZES)))
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--heap-gib", type=int, default=4)
    ap.add_argument("--block", type=int, default=256)
    ap.add_argument("--flush-mib", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-path measurement")
    ap.add_argument("--batched-n", type=int, default=1 << 22)
    ap.add_argument("--batched-cycles", type=int, default=100)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-churn", action="store_true", help="skip the churn measurement")
    ap.add_argument("--churn-rounds", type=int, default=1000)
    ap.add_argument("--serving-seconds", type=float, default=0.5)
    ap.add_argument("--no-config1", action="store_true", help="skip the 65,536 x 64 B page-based configuration")
    ap.add_argument("--no-traces", action="store_true",
                    help="skip the per-thread replays of the batched, churn and serving traces")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, enabled: bool = True):
        self.device = device
        self.proc = None
        self.path = None
        if not enabled:
            return
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "samples": len(rows), "reasons": sorted(reasons)}


# ------------------------------------------------------------- the arms
class OursArm:
    name = "ours"

    def __init__(self, heap_bytes: int):
        import ouroboros_b200 as ob
        self.ob = ob
        self.heap_bytes = heap_bytes
        self.heap = None

    def open(self, v):
        self.heap = self.ob.Ouroboros(v, self.heap_bytes)

    def close(self):
        if self.heap is not None:
            self.heap.close()
            self.heap = None

    def alloc(self, n, size, ptrs, block, stream, sizes=None):
        self.heap.alloc(ptrs, n, size, sizes, block, stream)

    def free(self, n, ptrs, block, stream):
        self.heap.free(ptrs, n, block, stream)

    def alloc_host(self, n, sizes_h, ptrs_h, ptrs, block, slices, stream):
        self.heap.alloc_host(ptrs_h, n, 0, sizes_h, ptrs, block, slices, stream)

    def host_reserve(self, n):
        self.heap.host_reserve(n)

    def write(self, ptrs, n, size, seed, stream):
        self.ob.write_pattern(ptrs, n, size, seed, None, stream)

    def verify(self, ptrs, n, size, seed, counters, stream):
        self.ob.verify_pattern(ptrs, n, counters, size, seed, None, stream)

    def flags(self):
        return self.heap.status()["flags"]

    def sanitize(self, ptrs, n, size, counters, stream, sizes=None):
        pass   # this build's pointers are checked by the tests; nothing to guard in the timed loop

    def verify_nulls(self, ptrs, n, counters, stream):
        # counters[0] += null pointers (size 0: no payload is read)
        self.ob.verify_pattern(ptrs, n, counters, 0, SEED, None, stream)

    def detail(self) -> str:
        st = self.heap.status()
        return f"timeouts {st['timeouts']} at wait sites {st['timeout_sites']:#x}, nulls {st['null_results']}"


class ReferenceArm:
    name = "reference"

    def __init__(self, heap_bytes: int):
        import oracle
        self.oracle = oracle
        self.heap_bytes = heap_bytes
        self.heap = None

    def open(self, v):
        self.heap = self.oracle.RefDriver(v, self.heap_bytes)

    def close(self):
        if self.heap is not None:
            self.heap.close()
            self.heap = None

    def alloc(self, n, size, ptrs, block, stream, sizes=None):
        self.heap.alloc(n, size, ptrs.data_ptr(), sizes.data_ptr() if sizes is not None else 0, block,
                        stream.cuda_stream)

    def free(self, n, ptrs, block, stream):
        self.heap.free(n, ptrs.data_ptr(), block, stream.cuda_stream)

    def sanitize(self, ptrs, n, size, counters, stream, sizes=None):
        self.heap.sanitize(n, size, ptrs.data_ptr(), counters.data_ptr(),
                           sizes.data_ptr() if sizes is not None else 0, stream.cuda_stream)

    def write(self, ptrs, n, size, seed, stream):
        self.oracle.ref_write(ptrs.data_ptr(), n, size, seed, 0, stream.cuda_stream)

    def verify(self, ptrs, n, size, seed, counters, stream):
        self.oracle.ref_verify(ptrs.data_ptr(), n, size, seed, counters.data_ptr(), 0, stream.cuda_stream)

    def flags(self):
        return 0

    def verify_nulls(self, ptrs, n, counters, stream):
        self.oracle.ref_verify(ptrs.data_ptr(), n, 0, SEED, counters.data_ptr(), 0, stream.cuda_stream)


class StdoutToStderr:
    """The reference prints banners with printf from initialize(); keep them
    (and anything else C code writes to fd 1) off stdout, which carries only
    the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


def fits_reference(v: str, size: int, n: int, heap_bytes: int) -> bool:
    """Capacity model: chunks the cell needs against the reference's maxChunks."""
    import oracle
    need = -(-n * size // 8192)
    return need + 64 < oracle.layout(v, heap_bytes)["max_chunks"]


# ----------------------------------------------------------- measurement
class BenchAbort(RuntimeError):
    pass


def run_cells(arm, cells, n, block, stream, ptrs, counters, flush, steps, warmup, e2e=False, tag="cells"):
    """Every cell on a fresh heap (the reference benchmarks one size per process):
    `warmup` untimed repetitions, then `steps` timed ones, each a flushed,
    event-timed alloc launch, an untimed pattern write + verify, and a flushed,
    event-timed free launch.  Optionally one end-to-end repetition through the
    C ABI with host buffers.  Returns {cell: (alloc_ms list, free_ms list, e2e_ms,
    (cold alloc_ms, cold free_ms))}: the cold pair is repetition 0, the first
    burst on the fresh heap (it is also the first warm-up repetition)."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    res = {}
    if e2e:
        sizes_h = torch.empty(n, dtype=torch.int32).pin_memory()
        ptrs_h = torch.empty(n, dtype=torch.int64).pin_memory()
    for (v, size) in cells:
        t0 = time.perf_counter()
        arm.open(v)
        a_ms, f_ms = [], []
        cold = None
        for rep in range(warmup + steps):
            with torch.cuda.stream(stream):
                flush.add_(1)
                ev[0].record(stream)
                arm.alloc(n, size, ptrs, block, stream)
                ev[1].record(stream)
                arm.sanitize(ptrs, n, size, counters, stream)
                arm.write(ptrs, n, size, SEED + rep, stream)
                arm.verify(ptrs, n, size, SEED + rep, counters, stream)
                flush.add_(1)
                ev[2].record(stream)
                arm.free(n, ptrs, block, stream)
                ev[3].record(stream)
            stream.synchronize()
            if rep >= warmup:
                a_ms.append(ev[0].elapsed_time(ev[1]))
                f_ms.append(ev[2].elapsed_time(ev[3]))
            if rep == 0:
                cold = (ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3]))
                flags = arm.flags()
                if flags & ~1:
                    why = arm.detail() if hasattr(arm, "detail") else ""
                    arm.close()
                    raise BenchAbort(f"device error flags {flags} after {v}:{size} (first repetition) {why}")
        e2e_ms = None
        if e2e:
            sizes_h.fill_(size)
            arm.host_reserve(n)   # the heap's copy streams and staging, made once per heap, untimed
            e2e_ms = e2e_host(arm, n, block, stream, sizes_h, ptrs, ptrs_h)
        flags = arm.flags()
        why = arm.detail() if hasattr(arm, "detail") and flags & ~1 else ""
        arm.close()
        if flags & ~1:
            raise BenchAbort(f"device error flags {flags} after {v}:{size} {why}")
        res[(v, size)] = (a_ms, f_ms, e2e_ms, cold)
        print(f"[bench] {tag} {v}:{size} alloc {np.mean(a_ms):.4f} ms free {np.mean(f_ms):.4f} ms "
              f"cold alloc {cold[0]:.4f} ms free {cold[1]:.4f} ms ({time.perf_counter() - t0:.2f}s)",
              file=sys.stderr, flush=True)
    return res


E2E_SLICES = 4


def e2e_host(arm, n, block, stream, sizes_h, ptrs, ptrs_h, slices=E2E_SLICES) -> float:
    """One end-to-end repetition through the C ABI with host buffers, as a
    caller with host-side requests runs it: one ouro_alloc_host call (the
    request sizes host->device from pinned memory, the allocation and the
    pointers device->host, in `slices` slices whose copies overlap the other
    slices' launches, with the pointers also left in a device array), then
    ouro_free of that device array (all 2^20 allocations are live at once, as
    in the timed repetitions).  Returns the device time from the call to the
    end of the free, ms."""
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    arm.alloc_host(n, sizes_h, ptrs_h, ptrs, block, slices, stream)
    arm.free(n, ptrs, block, stream)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def wake_up(arm_cls, v, stream):
    """An untimed alloc + free pass on a scratch heap before the timed region:
    otherwise the first cell's first (cold) repetition also times the GPU
    leaving idle."""
    n = 1 << 16
    arm = arm_cls(GiB)
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    counters = torch.zeros(2, dtype=torch.int64, device="cuda")
    with StdoutToStderr():
        arm.open(v)
        try:
            for _ in range(3):
                with torch.cuda.stream(stream):
                    arm.alloc(n, 64, ptrs, 256, stream)
                    arm.sanitize(ptrs, n, 64, counters, stream)
                    arm.free(n, ptrs, 256, stream)
                stream.synchronize()
        finally:
            arm.close()


def size_classes(sizes: np.ndarray) -> np.ndarray:
    """Queue index of each request size (Helper.cuh:42-45): max(ceil_log2(size) - 4, 0), sizes <= 8 KiB."""
    s = np.maximum(sizes.astype(np.int64), 1)
    return np.maximum(np.ceil(np.log2(s)).astype(np.int64) - 4, 0)


def chunks_for(class_pages: np.ndarray) -> int:
    """Base chunks a set of live pages per class (first instance) needs: ceil(pages / pages-per-chunk)."""
    ppc = 512 >> np.arange(10)
    return int(np.sum(-(-class_pages // ppc)))


def trace_configs(arm_cls, stream, is_reference: bool, churn_rounds: int = 10, serve_seconds: float = 0.25) -> dict:
    """The batched, churn and serving configurations replayed through the plain
    per-thread path (one launch of n threads for the allocations, one for the
    frees, as src/main.cu does), with the same seeded traces for both arms:
      batched_trace: VAC 8 GiB, 2^22 sizes log-uniform in [16, 8192] rounded
        up to 16 B; a cold repetition then 3 warm ones (alloc all, free all);
      churn_trace: VLC 16 GiB, a live set of 2^21 Zipf(1.2) sizes over the ten
        16 B .. 8 KiB classes, then `churn_rounds` rounds, each freeing a
        seeded 30% and allocating replacements;
      serving_trace: VAP 32 GiB, the allocation trace of the serving workload
        -- a 10M-vertex power-law graph's edge blocks (4 x degree bytes), then
        `serve_seconds` of its batches (2,000 batches/s, 1k..256k requests
        log-uniform, a batch's distinct vertices), each batch one launch that
        allocates the doubled blocks (8 x degree bytes, at most 8 KiB) and one
        that frees the old ones.
    Only the allocation and free launches are timed (CUDA events, L2 flushed
    before each launch of the batched trace).  The reference is run only where
    a capacity model of the trace says it stays below maxChunks (its behaviour
    past that is undefined), never on the batched or churn traces (its own code
    faulted on each once, in launches of 2^22 and 2^21 threads of mixed sizes,
    so it is not run on them again), and with launches of at most 2^20
    threads, the concurrency its benchmark configuration runs at; the
    launches of this build are split the same way."""
    import oracle
    out = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    flush = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")

    def timed(fn):
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            fn()
            ev[1].record(stream)
        stream.synchronize()
        return ev[0].elapsed_time(ev[1])

    # ---------------------------------------------------------------- batched
    n = 1 << 22
    rng = np.random.default_rng(2024)
    sizes_np = (np.ceil(np.exp(rng.uniform(np.log(16), np.log(8192), n)) / 16) * 16).astype(np.uint32)
    cls = size_classes(sizes_np)
    need = chunks_for(np.bincount(cls, minlength=10)) + 12 * 8 + (3 * n) // 2048
    mc = oracle.layout("VAC", 8 * GiB)["max_chunks"]
    rec = {"workload": "VAC 8 GiB, 2^22 requests log-uniform 16..8192 B (rounded up to 16 B), per-thread alloc "
                       "launch + free launch", "chunks_needed": need, "max_chunks": mc}
    if is_reference:
        rec["unavailable"] = ("the reference's own CUDA code faulted on this trace (unspecified launch failure in "
                              "its alloc launch of 2^22 threads on a VAC heap 90% full); it is not run again")
    else:
        arm = arm_cls(8 * GiB)
        sizes_d = torch.from_numpy(sizes_np.view(np.int32)).cuda()
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        ms = []
        with StdoutToStderr():
            arm.open("VAC")
            try:
                for rep in range(4):
                    flush.add_(1)
                    a = timed(lambda: arm.alloc(n, 0, ptrs, 256, stream, sizes=sizes_d))
                    if rep == 0:
                        cnt.zero_()
                        arm.verify_nulls(ptrs, n, cnt, stream)
                    flush.add_(1)
                    f = timed(lambda: arm.free(n, ptrs, 256, stream))
                    ms.append((a, f))
                flags = arm.flags()
            finally:
                arm.close()
        warm = float(np.mean([a + f for a, f in ms[1:]]))
        rec.update({"cold_mops": round(2.0 * n / ((ms[0][0] + ms[0][1]) * 1e-3) / 1e6, 2),
                    "warm_mops": round(2.0 * n / (warm * 1e-3) / 1e6, 2),
                    "cold_ms": [round(ms[0][0], 3), round(ms[0][1], 3)],
                    "warm_ms": [round(float(np.mean([a for a, _ in ms[1:]])), 3),
                                round(float(np.mean([f for _, f in ms[1:]])), 3)],
                    "null_results_first_rep": int(cnt[0].item()), "flags": flags})
    out["batched_trace"] = rec

    # ------------------------------------------------------------------ churn
    n = 1 << 21
    rng = np.random.default_rng(99)
    w = 1.0 / np.arange(1, 11) ** 1.2
    w /= w.sum()
    live_cls = rng.choice(10, size=n, p=w)
    rounds_sizes, rounds_idx = [], []
    for r in range(churn_rounds):
        idx = np.nonzero(rng.random(n) < 0.3)[0]
        rounds_idx.append(idx)
        rounds_sizes.append(rng.choice(10, size=idx.size, p=w))
    # capacity: live pages per class at their peak (allocations of a round come before nothing is freed? frees first)
    peak = np.bincount(live_cls, minlength=10).astype(np.int64)
    cur_cls = live_cls.copy()
    for idx, new in zip(rounds_idx, rounds_sizes):
        cur_cls[idx] = new
        peak = np.maximum(peak, np.bincount(cur_cls, minlength=10))
    need = chunks_for(peak) * 2 + 12 * 16
    mc = oracle.layout("VLC", 16 * GiB)["max_chunks"]
    rec = {"workload": "VLC 16 GiB, live set 2^21 Zipf(1.2) over 16 B..8 KiB, %d rounds of 30%% free + "
                       "re-allocation, per-thread free launch + alloc launch" % churn_rounds,
           "chunks_needed_bound": need, "max_chunks": mc}
    if is_reference:
        rec["unavailable"] = ("the reference's own CUDA code faulted on this trace (misaligned address in its first "
                              "alloc launch, 2^21 threads of mixed sizes on a VLC heap); it is not run again")
    else:
        arm = arm_cls(16 * GiB)
        ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
        sizes_d = torch.from_numpy((16 << live_cls).astype(np.uint32).view(np.int32)).cuda()
        ms, ops = 0.0, 0
        with StdoutToStderr():
            arm.open("VLC")
            try:
                timed(lambda: arm.alloc(n, 0, ptrs, 256, stream, sizes=sizes_d))
                for idx, new in zip(rounds_idx, rounds_sizes):
                    m = idx.size
                    idx_d = torch.from_numpy(idx).cuda()
                    sub = ptrs[idx_d].contiguous()
                    nsz = torch.from_numpy((16 << new).astype(np.uint32).view(np.int32)).cuda()
                    ms += timed(lambda: arm.free(m, sub, 256, stream))
                    ms += timed(lambda: arm.alloc(m, 0, sub, 256, stream, sizes=nsz))
                    ptrs[idx_d] = sub
                    ops += 2 * m
                flags = arm.flags()
            finally:
                arm.close()
        rec.update({"mops": round(ops / (ms * 1e-3) / 1e6, 2), "ms": round(ms, 3), "ops": ops, "flags": flags})
    out["churn_trace"] = rec

    # ---------------------------------------------------------------- serving
    nv = 10_000_000
    rng = np.random.default_rng(17)
    u = rng.random(nv)
    deg = np.minimum(np.maximum(np.floor(u ** (-1.0 / 1.1)), 1), 1024).astype(np.int64)   # P(d) ~ d^-2.1
    batches = []
    t, rate, clients = 0.0, 2000.0, 256
    arr = []
    for c in range(clients):
        tt = 0.0
        while True:
            tt += rng.exponential(clients / rate)
            if tt >= serve_seconds:
                break
            arr.append((tt, int(np.exp(rng.uniform(np.log(1000), np.log(256000))))))
    arr.sort()
    for _, size in arr:
        batches.append(np.unique(rng.integers(0, nv, size)))
    # capacity: page-based classes keep their chunks; live pages per class after each batch's allocations
    cur = deg.copy()
    cls_of = lambda d: size_classes(np.minimum(4 * d, 8192))
    live = np.bincount(cls_of(cur), minlength=10).astype(np.int64)
    peak = live.copy()
    for v in batches:
        d = cur[v]
        g = v[d < 2048]
        nd = np.minimum(2 * cur[g], 2048)
        live_with_new = live + np.bincount(cls_of(nd), minlength=10)
        peak = np.maximum(peak, live_with_new)
        live = live_with_new - np.bincount(cls_of(cur[g]), minlength=10)
        cur[g] = nd
    need = chunks_for(peak) + sum(int(-(-p // 2048)) for p in peak) + 12 * 8
    mc = oracle.layout("VAP", 32 * GiB)["max_chunks"]
    rec = {"workload": "VAP 32 GiB, 10M-vertex power-law graph (alpha 2.1) edge blocks, then %.2f s of serving "
                       "batches at 2,000 batches/s (%d batches, distinct vertices per batch): per batch one alloc "
                       "launch (8 x degree bytes, at most 8 KiB) and one free launch of the old blocks"
                       % (serve_seconds, len(batches)), "chunks_needed": need, "max_chunks": mc}
    if is_reference and need + 1024 >= mc:
        rec["skipped"] = "capacity model: the trace needs %d of %d chunks" % (need, mc)
    else:
        arm = arm_cls(32 * GiB)
        vptr = torch.zeros(nv, dtype=torch.int64, device="cuda")
        degree = torch.from_numpy(deg).cuda()
        scnt = torch.zeros(2, dtype=torch.int64, device="cuda")
        ms, ops = 0.0, 0
        with StdoutToStderr():
            arm.open("VAP")
            try:
                sz = (4 * degree).to(torch.int32)
                for o in range(0, nv, 1 << 20):   # the initial blocks, 2^20 threads per launch
                    m = min(1 << 20, nv - o)
                    timed(lambda: arm.alloc(m, 0, vptr[o:o + m], 256, stream, sizes=sz[o:o + m]))
                    with torch.cuda.stream(stream):
                        arm.sanitize(vptr[o:o + m], m, 0, scnt, stream, sizes=sz[o:o + m])
                for v in batches:
                    vd = torch.from_numpy(v).cuda()
                    d = degree[vd]
                    vd = vd[d < 2048]
                    m = int(vd.numel())
                    if m == 0:
                        continue
                    nd = torch.clamp(2 * degree[vd], max=2048)
                    nsz = (4 * nd).to(torch.int32)
                    newp = torch.zeros(m, dtype=torch.int64, device="cuda")
                    old = vptr[vd].contiguous()
                    ms += timed(lambda: arm.alloc(m, 0, newp, 256, stream, sizes=nsz))
                    with torch.cuda.stream(stream):
                        arm.sanitize(newp, m, 0, scnt, stream, sizes=nsz)
                    ms += timed(lambda: arm.free(m, old, 256, stream))
                    vptr[vd] = newp
                    degree[vd] = nd
                    ops += 2 * m
                flags = arm.flags()
            finally:
                arm.close()
        rec.update({"mops": round(ops / (ms * 1e-3) / 1e6, 2), "ms": round(ms, 3), "ops": ops, "flags": flags,
                    "pointers_outside_heap": int(scnt[1].item())})
    out["serving_trace"] = rec
    return out


def cold_summary(res, n) -> dict:
    """The first burst on every fresh heap: repetition 0 of each cell, the case
    where every request must create chunks."""
    per, ops, ms = {}, 0.0, 0.0
    for (v, s), (_, _, _, (ca, cf)) in res.items():
        per[f"{v}:{s}"] = {"alloc_ms": round(ca, 4), "free_ms": round(cf, 4),
                           "mops": round(2.0 * n / ((ca + cf) * 1e-3) / 1e6, 2)}
        ops += 2.0 * n
        ms += ca + cf
    worst = max(per.items(), key=lambda kv: kv[1]["alloc_ms"])
    return {"value": round(ops / (ms * 1e-3) / 1e6, 3), "unit": "Mops/s", "ms_total": round(ms, 3),
            "worst_alloc": {"cell": worst[0], "alloc_ms": worst[1]["alloc_ms"]},
            "what": "repetition 0 of every cell: one alloc launch of n threads on a fresh heap (every chunk is "
                    "created in it) and the free launch after it, event-timed, L2 flushed before each",
            "per_cell": per}


def config1_bench(arm_cls, stream, steps=10) -> dict:
    """The single-instantiation configuration: page-based standard queues, 1 GiB
    heap, one launch of 65,536 threads (256 per block) each allocating 64 B;
    after each alloc launch the payload is written and verified (untimed), then
    one launch frees everything; 10 repetitions on one heap.  Reported the way
    the reference's harness reports it (src/main.cu:146-167): the mean over all
    repetitions, the first (cold) one included; the warm mean beside it."""
    n, size, block = 1 << 16, 64, 256
    arm = arm_cls(GiB)
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    counters = torch.zeros(2, dtype=torch.int64, device="cuda")
    flush = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    a_ms, f_ms = [], []
    with StdoutToStderr():
        arm.open("P")
        try:
            for rep in range(steps):
                with torch.cuda.stream(stream):
                    flush.add_(1)
                    ev[0].record(stream)
                    arm.alloc(n, size, ptrs, block, stream)
                    ev[1].record(stream)
                    arm.sanitize(ptrs, n, size, counters, stream)
                    arm.write(ptrs, n, size, SEED + rep, stream)
                    arm.verify(ptrs, n, size, SEED + rep, counters, stream)
                    flush.add_(1)
                    ev[2].record(stream)
                    arm.free(n, ptrs, block, stream)
                    ev[3].record(stream)
                stream.synchronize()
                a_ms.append(ev[0].elapsed_time(ev[1]))
                f_ms.append(ev[2].elapsed_time(ev[3]))
            flags = arm.flags()
        finally:
            arm.close()
    nulls, bad = counters.tolist()
    mean = float(np.mean(a_ms) + np.mean(f_ms))
    warm = float(np.mean(a_ms[1:]) + np.mean(f_ms[1:]))
    return {"workload": "P, 1 GiB heap, 65,536 threads x 64 B (256 per block), 10 repetitions on one heap",
            "value": round(2.0 * n / (mean * 1e-3) / 1e6, 3), "unit": "Mops/s",
            "what": "mean over all 10 repetitions, the first (cold) one included, as src/main.cu:146-167 averages",
            "warm_mops": round(2.0 * n / (warm * 1e-3) / 1e6, 3),
            "cold_ms": {"alloc": round(a_ms[0], 4), "free": round(f_ms[0], 4)},
            "alloc_ms": [round(x, 4) for x in a_ms], "free_ms": [round(x, 4) for x in f_ms],
            "null_results": nulls, "bad_words": bad, "flags": flags}


def against_reference_cells(per_cell: dict, cold: dict) -> dict | None:
    """Per-instantiation geometric-mean and smallest per-cell ratios of this
    run's cells against a recorded reference-arm run (warm and cold); reported
    beside the headline, which the driver compares with its own reference run."""
    try:
        ref = json.load(open(REFERENCE_CELLS))
    except Exception:
        return None
    out = {}
    for key, mine, theirs in (("warm", per_cell, ref["per_cell"]), ("cold", cold, ref["cold_per_cell"])):
        by = {}
        for cell, r in theirs.items():
            if cell in mine and r["mops"] > 0:
                by.setdefault(cell.split(":")[0], []).append(mine[cell]["mops"] / r["mops"])
        out[key] = {v: {"geomean": round(float(np.exp(np.mean(np.log(x)))), 2), "min": round(min(x), 2)}
                    for v, x in by.items()}
    out["source"] = "profiles/reference_cells.json (" + ref.get("command", "") + ")"
    return out


def cpu_baseline(cells, n, heap_bytes) -> dict:
    """The oracle port (one host thread) over every cell, 2^20 requests each,
    one alloc pass and one free pass; plus glibc malloc/free on all host cores."""
    import oracle
    t_total, ops = 0.0, 0
    for v, size in cells:
        ops_arr = np.empty(4 * n, dtype=np.uint32)
        ops_arr[0:2 * n:2] = 0
        ops_arr[1:2 * n:2] = size
        ops_arr[2 * n::2] = 1
        ops_arr[2 * n + 1::2] = np.arange(n, dtype=np.uint32)
        o = oracle.Oracle(v, heap_bytes)
        t0 = time.perf_counter()
        o.run_trace(ops_arr)
        t_total += time.perf_counter() - t0
        ops += 2 * n
        o.close()
    out = {"value": ops / t_total / 1e6, "unit": "Mops/s", "cores": 1, "kind": "port",
           "sample": f"{len(cells)} cells x {n} requests, one malloc pass and one free pass each, "
                     f"sequential C restatement of the reference (oracle/ouro_oracle.c)"}
    so = os.path.join(ROOT, "oracle", "_build", "libhost_replay.so")
    if os.path.exists(so):
        lib = ctypes.CDLL(so)
        lib.host_replay.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32,
                                    ctypes.c_int, ctypes.c_void_p]
        threads = os.cpu_count() or 1
        tot, hops = 0.0, 0
        r = np.zeros(3)
        for v, size in cells[: len(HEADLINE_SIZES)]:
            lib.host_replay(n, size, None, SEED, threads, r.ctypes.data)
            tot += r[0]
            hops += 2 * n
        out["host_malloc"] = {"value": hops / tot / 1e6, "unit": "Mops/s", "cores": threads,
                              "sample": f"glibc malloc/free, {len(HEADLINE_SIZES)} sizes x {n} requests "
                                        f"(the same requests for every instantiation)"}
    return out


# Hot-line RMWs per warp group that every group of a class serialises on: the
# class semaphore plus the front ticket (page alloc), back ticket (page free) or
# scan cursor (chunk alloc); chunk free only signals the semaphore.
HOT_RMW = {("page", "alloc"): 2, ("page", "free"): 2, ("chunk", "alloc"): 2, ("chunk", "free"): 1}
# Per-lane L2 atomics per alloc+free pair of the reference's algorithm (g = 32 lanes per group).
REF_ATOMICS_PER_PAIR = {"P": 2 + 4 / 32, "VAP": 4 + 4 / 32, "VLP": 4 + 4 / 32,
                        "C": 4 + 2 / 32, "VAC": 4 + 2 / 32, "VLC": 4 + 2 / 32}


def roofline(res, n, steps) -> dict:
    """Roofline of the dominant kernel: the (kernel, instantiation) pair with the
    largest share of the timed kernel time.  The path is bound by L2 atomic
    throughput.  achieved = the per-lane L2 atomics of the reference's algorithm
    for one launch (per alloc+free pair: P 2 + 4/g, VAP and VLP 4 + 4/g,
    chunk-based 4 + 2/g, g = 32 lanes per class group; half of it per launch)
    over the average launch time; peak = the distinct-address atomic rate of
    this GPU, measured live (every lane of all SMs, one atomicAdd each on an
    L2-resident array).  Beside it: the rate on the lines every group of a
    class serialises on (semaphore + ticket or cursor) against the measured
    single-address rate, and the DRAM traffic of the kernel from ncu."""
    import ouroboros_b200 as ob
    per = {}
    for (v, size), (a, f, _, _) in res.items():
        for kern, ms in (("alloc", a), ("free", f)):
            t = per.setdefault((v, kern), [0.0, 0])
            t[0] += float(np.sum(ms))
            t[1] += len(ms)
    total = sum(t[0] for t in per.values())
    (v, kern), (ms_sum, launches) = max(per.items(), key=lambda kv: kv[1][0])
    avg_ms = ms_sum / launches
    kind = "page" if v in ("P", "VAP", "VLP") else "chunk"
    hot_lines = HOT_RMW[(kind, kern)]
    groups = n / 32.0
    hot_achieved = hot_lines * groups / (avg_ms * 1e-3) / 1e9
    hot = ob.measure_atomics(1)
    two_lines = {"one_256B_block": ob.measure_atomics(3), "separate_256B_blocks": ob.measure_atomics(4)}
    distinct = ob.measure_atomics(0)
    vidx = VARIANTS.index(v)
    traffic, traffic_cell = None, None
    try:
        t = json.load(open(TRAFFIC_FILE)).get(f"k_{kern}<{vidx}>")
        if t:
            traffic, traffic_cell = t["bytes"], t["cell"]
    except Exception:
        pass
    peaks = measured_peaks()
    if peaks.get("hbm_gbs"):
        hbm_peak, hbm_source = float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    else:
        hbm_peak, hbm_source = FALLBACK_HBM_GBS, "no MEASURED_PEAKS.json: 6.65 TB/s copy bandwidth (of fallback)"
    atomics = REF_ATOMICS_PER_PAIR[v] / 2.0 * n
    achieved = atomics / (avg_ms * 1e-3) / 1e9
    return {
        "bound": "l2_atomic", "kernel": f"k_{kern}<{vidx}> ({v})", "share": round(ms_sum / total, 4),
        "achieved": round(achieved, 4), "peak": round(distinct, 2), "unit": "G atomics/s",
        "frac": round(achieved / distinct, 5), "traffic": traffic,
        "traffic_unit": "bytes per launch (dram read + write, ncu)", "traffic_cell": traffic_cell,
        "algorithmic_atomics_per_launch": atomics,
        "peak_source": "measured live by ouro_measure_atomics(0): distinct addresses, every lane of all SMs "
                       "(builder-measured; the driver's peaks file has no atomic figure)",
        "avg_launch_ms": round(avg_ms, 5), "launches": launches,
        "hot_line": {
            "what": "RMWs on the lines every group of the class serialises on (semaphore + front/back ticket or "
                    "scan cursor), one per warp group",
            "rmw_per_launch": hot_lines * groups, "achieved_gops": round(hot_achieved, 4),
            "peak_gops": round(hot_lines * hot, 4),
            "peak_source": f"measured live: one hot 32-bit address, one RMW per warp, x{hot_lines} independent lines",
            "frac": round(hot_achieved / (hot_lines * hot), 4),
            "two_hot_lines_gops": {k: round(x, 4) for k, x in two_lines.items()},
            "note": "two hot lines in one 256 B block share an L2 slice; the allocator's hot counters each "
                    "have a 256 B block of their own"},
        "hbm": {"bytes_per_launch": 16.0 * n, "achieved_gbs": round(16.0 * n / (avg_ms * 1e-3) / 1e9, 2),
                "peak_gbs": hbm_peak, "peak_source": hbm_source,
                "frac": round(16.0 * n / (avg_ms * 1e-3) / 1e9 / hbm_peak, 5),
                "note": "per request 8 B pointer + 4 B entry read + 4 B entry write"},
    }


def batched_bench(n: int, cycles: int, stream) -> dict:
    """The batched configuration: chunk-based virtualized-array heap of 8 GiB,
    n requests with sizes log-uniform in [16, 8192] B rounded up to 16 B
    (seeded).  Phase 1: all n allocated, then all freed -- by the batched
    kernels and, for comparison, by the per-thread kernels on the same sizes
    (warm heap, L2 flushed).  Phase 2: `cycles` churn cycles, each freeing a
    hashed 50% and re-allocating new log-uniform sizes, captured as one CUDA
    graph and replayed.  Launch shape from the autotuner."""
    import ouroboros_b200 as ob
    rng = np.random.default_rng(2024)
    sz = np.exp(rng.uniform(np.log(16), np.log(8192), n))
    sizes = torch.from_numpy(((np.ceil(sz / 16) * 16).astype(np.uint32)).view(np.int32)).cuda()
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    flush = torch.zeros(64 << 20, dtype=torch.int32, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    out = {"workload": "VAC, 8 GiB heap, %d requests log-uniform 16..8192 B (rounded up to 16 B)" % n}
    # the run-time configuration: queue capacity x aggregation width x block
    # size, each candidate on a fresh heap (ouro_autotune_config)
    try:
        tc = ob.autotune_config("VAC", 8 * GiB, min(n, 1 << 20), 16, 8192, reps=2)
        pts = tc["points"]
        dflt = [p for p in pts if p["virtual_queue_entries"] == 512 and p["agg_width"] == 32]
        out["autotune_config"] = {
            "best": tc["best"], "candidates": len(pts), "accepted": sum(p["ok"] for p in pts),
            "swept": {"queue_entries_per_class": [1 << 16, 1 << 17, 1 << 18, 1 << 19, 1 << 20],
                      "agg_width": [8, 16, 32], "block": [128, 256, 512, 1024]},
            "best_at_2e20_entries_agg32": max((p["mops"] for p in dflt if p["ok"]), default=None)}
    except Exception as exc:   # reported, the rest stands
        out["autotune_config"] = {"error": str(exc)[:300]}
    with ob.Ouroboros("VAC", 8 * GiB) as heap:
        out["autotune"] = heap.autotune_batch(n=min(n, 1 << 20), lo=16, hi=8192)
        res = {}
        for name, alloc, free in (
                ("batched", lambda: heap.alloc_batch(sizes, ptrs, n, stream=stream),
                 lambda: heap.free_batch(ptrs, n, stream=stream)),
                ("per_thread", lambda: heap.alloc(ptrs, n, 0, sizes, stream=stream),
                 lambda: heap.free(ptrs, n, stream=stream))):
            times = []
            for rep in range(4):
                with torch.cuda.stream(stream):
                    flush.add_(1)
                    ev[0].record(stream)
                    alloc()
                    ev[1].record(stream)
                    flush.add_(1)
                    ev[2].record(stream)
                    free()
                    ev[3].record(stream)
                stream.synchronize()
                if rep:   # the first repetition warms the heap
                    times.append(ev[0].elapsed_time(ev[1]) + ev[2].elapsed_time(ev[3]))
            res[name] = 2.0 * n / (np.mean(times) * 1e-3) / 1e6
        st1 = heap.status(clear=True)
        out["phase1_status"] = {"flags": st1["flags"], "timeout_sites": st1["timeout_sites"],
                                "null_results": st1["null_results"]}
        out["phase1_mops"] = {k: round(v, 1) for k, v in res.items()}
        out["phase1_speedup"] = round(res["batched"] / res["per_thread"], 3)
        # phase 2: the live set, then `cycles` churn cycles replayed from one graph
        with torch.cuda.stream(stream):
            heap.alloc_batch(sizes, ptrs, n, stream=stream)
        stream.synchronize()
        sizes_live = sizes.clone()
        heap.batch_reserve(n)   # the batch scratch exists before capture (no allocation inside the graph)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            for c in range(cycles):
                heap.realloc_batch(ptrs, sizes_live, n, seed=77, cycle=c + 1, fraction_permille=500,
                                   dist=("loguniform", 16, 8192), stream=torch.cuda.current_stream())
        for _ in range(2):   # replays keep churning the same live set
            g.replay()
        torch.cuda.synchronize()
        st0 = heap.status()
        ev[0].record(stream)
        with torch.cuda.stream(stream):
            g.replay()
        ev[1].record(stream)
        stream.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        ops = 2.0 * 0.5 * n * cycles   # a picked request is one free and one malloc
        st = heap.status()
        out["phase2"] = {"cycles": cycles, "ms": round(ms, 3), "mops": round(ops / (ms * 1e-3) / 1e6, 1),
                         "ms_per_cycle": round(ms / cycles, 4), "null_results": st["null_results"] - st0["null_results"],
                         "flags": st["flags"], "timeout_sites": st["timeout_sites"], "timeouts": st["timeouts"]}
        del g
        with torch.cuda.stream(stream):
            heap.free_batch(ptrs, n, stream=stream)
        stream.synchronize()
    return out


def churn_bench(rounds: int, stream) -> dict:
    """The churn configuration: chunk-based virtualized linked-list heap of
    16 GiB; an initial live set of 2^21 allocations; `rounds` rounds, each
    freeing a hashed 30% of the live set and allocating replacements with sizes
    Zipf(1.2) over the ten 16 B..8 KiB classes (rank 1 = 16 B), through the
    batched churn kernel.  Tracks failed allocations, chunk reuse and peak
    occupancy; ownership / alignment / heap-bounds checks and a seeded payload
    every 10 rounds and at the end, the accounting check at the end."""
    import ouroboros_b200 as ob
    n = 1 << 21
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    sizes = torch.zeros(n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    dist = ("zipf", 1.2)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {"workload": "VLC 16 GiB, live set 2^21, %d rounds of 30%% free + Zipf(1.2) re-allocation" % rounds}
    with ob.Ouroboros("VLC", 16 * GiB) as heap:
        with torch.cuda.stream(stream):
            heap.realloc_batch(ptrs, sizes, n, seed=99, cycle=0, fraction_permille=1000, dist=dist, stream=stream)
        stream.synchronize()
        st0 = heap.status()
        peak, checked, bad, overlaps, ms = 0, 0, 0, 0, 0.0
        for r in range(1, rounds + 1):
            ev[0].record(stream)
            heap.realloc_batch(ptrs, sizes, n, seed=99, cycle=r, fraction_permille=300, dist=dist, stream=stream)
            ev[1].record(stream)
            stream.synchronize()
            ms += ev[0].elapsed_time(ev[1])
            if r % 10 == 0 or r == rounds:
                peak = max(peak, heap.free_resources()["chunks_in_use"])
                rep = heap.check_allocations(ptrs, n, sizes=sizes)
                ob.write_pattern(ptrs, n, 0, r, sizes)
                ob.verify_pattern(ptrs, n, cnt, 0, r, sizes)
                torch.cuda.synchronize()
                overlaps += rep["overlaps"] + rep["misaligned"] + rep["out_of_heap"]
                checked += 1
        st = heap.status()
        nulls, badw = cnt.tolist()
        with torch.cuda.stream(stream):
            heap.free_batch(ptrs, n, stream=stream)
        stream.synchronize()
        hr = heap.check_heap()
        idle = all(hr["sem_count"][c] == hr["owned_pages"][c] == hr["free_pages_meta"][c] and
                   hr["sem_expected"][c] == 0 and hr["sem_reserved"][c] == 0 for c in range(12)) and hr["bad"] == 0
        fr = heap.free_resources()
    ops = 2.0 * 0.3 * n * rounds
    out.update({
        "rounds": rounds, "ms": round(ms, 2), "mops": round(ops / (ms * 1e-3) / 1e6, 1),
        "failed_allocs": st["null_results"] - st0["null_results"], "flags": st["flags"],
        "chunk_allocs_after_warmup": st["chunk_allocs"] - st0["chunk_allocs"],
        "peak_chunks_in_use": peak, "heap_chunks": fr["heap_chunks"], "checks": checked,
        "overlap_or_bounds_violations": overlaps, "payload_nulls": nulls, "payload_bad_words": badw,
        "accounting_idle_after_free": bool(idle),
    })
    return out


def serving_bench(seconds: float) -> dict:
    """The serving configuration: page-based virtualized-array heap of 32 GiB
    holding a 10M-vertex power-law graph (degree exponent 2.1, uint32 ids);
    256 clients with Poisson arrivals; batch sizes log-uniform in 1k..256k
    requests, each request moving a vertex's edge block from 4 x d to 8 x d
    bytes (at most 8 KiB); admission deferred while free bytes are below 10%
    of the heap.  Served by the device-resident loop (ouro_serve_*): three
    rows, each on a fresh heap and graph with `seconds` of arrivals --
    saturation (every batch at t = 0: the service rate), the configured
    2,000 batches/s, and 80% of the measured service rate.  Latency = device
    time from the loop seeing a batch to its last request done."""
    from ouroboros_b200 import serve
    import ouroboros_b200 as ob
    nv = 10_000_000
    rows = {}

    def one(name, rate, seed, at_zero=False, span=None):
        with ob.Ouroboros("VAP", 32 * GiB) as heap:
            g = serve.Graph(heap, nv, seed=17, alpha=2.1)
            batches = serve.poisson_batches(256, rate, span or seconds, nv, 1000, 256_000, seed=seed)
            if at_zero:
                batches = [(0.0, c, v) for (_, c, v) in batches]
            srv = serve.Server(g, max_inflight=64, watermark=0.10)
            try:
                rep = srv.run(batches)
            finally:
                srv.close()
            rep["offered_batches_per_s"] = None if at_zero else rate
            rep["free_bytes_after"] = heap.free_resources()["free_bytes"]
            rep["flags"] = heap.status()["flags"]
        for k in list(rep):
            if isinstance(rep[k], float):
                rep[k] = round(rep[k], 4)
        rows[name] = rep
        return rep

    sat = one("saturated", 2000.0, 23, at_zero=True)
    one("rate_2000", 2000.0, 23)
    service = sat.get("batches_per_s") or 0.0
    if service > 0:
        # as many batches as the 2,000 batches/s row offers, arriving at 80% of
        # the service rate: the graph (and the heap) grows by the same amount
        one("rate_80pct_of_service", 0.8 * service, 29, span=seconds * 2000.0 / (0.8 * service))
    return {"workload": ("VAP 32 GiB, 10M-vertex power-law graph (alpha 2.1), 256 Poisson clients, batches of "
                         "1k-256k growth requests (log-uniform), %.2f s of arrivals at 2,000 batches/s (the 80%% row: "
                         "the same expected number of batches, arriving faster), device-resident loop "
                         "(64 batches in flight at most), 10%% free-byte watermark; fresh heap and graph per row"
                         % seconds),
            "service_batches_per_s": round(service, 1) if service else None,
            "rows": rows}


# Copy bandwidth measured earlier on B200s of the same kind, used when no
# measured peaks file is present.
FALLBACK_HBM_GBS = 6650.0


def measured_peaks() -> dict:
    try:
        return json.load(open(MEASURED_PEAKS))
    except Exception:
        return {}


def replica_value(total_ms: float, e2e_ms: float, ops_per_rank: float, world: int, dist=None, device="cuda"):
    """Replicas: every rank runs the whole workload on its own GPU.  The job's
    time is the slowest rank's (a MAX all-reduce of the summed kernel times)
    and its value all ranks' operations over that time.  Returns (Mops/s,
    max total ms, max end-to-end ms)."""
    if dist is not None and world > 1:
        t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_ms = float(t[0].item()), float(t[1].item())
    return ops_per_rank * world / (total_ms * 1e-3) / 1e6, total_ms, e2e_ms


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and world > 1:
        # the reference arm is measured by rank 0 alone; the other ranks have no work
        if rank != 0:
            return 0
        world = 1
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))

    variants = [v for v in args.variants.split(",") if v]
    sizes = [int(s) for s in args.sizes.split(",") if s]
    extra_sizes = [int(s) for s in args.extra_sizes.split(",") if s]
    heap_bytes = args.heap_gib * GiB
    n = args.n
    cells = [(v, s) for v in variants for s in sizes]
    stream = torch.cuda.Stream()
    ptrs = torch.zeros(n, dtype=torch.int64, device="cuda")
    counters = torch.zeros(2, dtype=torch.int64, device="cuda")
    flush = torch.zeros(args.flush_mib << 18, dtype=torch.int32, device="cuda")

    if args.impl == "reference":
        import oracle
        if not oracle.ref_available():
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libouro_ref.so was not built "
                                  "(the reference sources were not mounted at build time)"}))
            return 0
        skipped = {f"{v}:{sz}": ("capacity model: needs more chunks than the heap has" if v not in REFERENCE_FAULTED
                                 else REFERENCE_FAULTED[v])
                   for v, sz in cells if v in REFERENCE_FAULTED or not fits_reference(v, sz, n, heap_bytes)}
        cells = [c for c in cells if f"{c[0]}:{c[1]}" not in skipped]
        arm = ReferenceArm(heap_bytes)
        extra_cells = []
    else:
        arm = OursArm(heap_bytes)
        extra_cells = [(v, s) for v in variants for s in extra_sizes]

    wake_up(ReferenceArm if args.impl == "reference" else OursArm, "P", stream)

    # --- timed region: every cell, W warm-up + K timed repetitions on its own heap
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local, enabled=not args.no_clocks)
    t_wall = time.perf_counter()
    with StdoutToStderr():
        res = run_cells(arm, cells, n, args.block, stream, ptrs, counters, flush, args.steps, args.warmup,
                        e2e=(args.impl == "ours" and not args.no_e2e))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    if dist:
        dist.barrier()

    per_cell = {}
    total_ms = alloc_ms = free_ms = 0.0
    e2e_ms = 0.0
    for (v, s), (a, f, e, _) in res.items():
        per_cell[f"{v}:{s}"] = {"alloc_ms": round(float(np.mean(a)), 5), "free_ms": round(float(np.mean(f)), 5),
                                "mops": round(2.0 * n / ((np.mean(a) + np.mean(f)) * 1e-3) / 1e6, 2)}
        total_ms += float(np.sum(a) + np.sum(f))
        alloc_ms += float(np.sum(a))
        free_ms += float(np.sum(f))
        if e is not None:
            e2e_ms += e
    nulls, bad = counters.tolist()
    configured_cells = len(variants) * len(sizes)
    value, total_ms, e2e_ms = replica_value(total_ms, e2e_ms, 2.0 * n * len(cells) * args.steps, world, dist)
    # the same aggregate over the cells the reference arm measures
    ref_cells = [(v, s) for (v, s) in res if v not in REFERENCE_FAULTED]
    ref_ms = sum(float(np.sum(res[c][0]) + np.sum(res[c][1])) for c in ref_cells)
    value_ref_cells = 2.0 * n * len(ref_cells) * args.steps / (ref_ms * 1e-3) / 1e6 if ref_ms else None

    # --- extra cells (ours only): 4096 / 8192 B exceed the heap for 2^20 requests
    extra = {}
    if extra_cells:
        counters_x = torch.zeros(2, dtype=torch.int64, device="cuda")
        try:
            rx = run_cells(arm, extra_cells, n, args.block, stream, ptrs, counters_x, flush, 2, 1, tag="extra")
            for (v, s), (a, f, _, _) in rx.items():
                extra[f"{v}:{s}"] = {"alloc_ms": round(float(np.mean(a)), 5), "free_ms": round(float(np.mean(f)), 5)}
            extra["null_results_per_repetition"] = int(counters_x[0].item()) // 3
        except BenchAbort as exc:
            extra["error"] = str(exc)
        extra["note"] = ("2^20 x size exceeds the 4 GiB heap: the surplus requests get nullptr "
                         "(the reference's behaviour there is undefined, it is not run)")

    out = {
        "metric": "alloc+free Mops/s (6 instantiations x 16..2048 B, 2^20 threads, 4 GiB heaps)",
        "value": round(value, 3), "unit": "Mops/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (fixed-size requests, seeded pattern)",
        "config": {"workload": "all six instantiations, fixed size per launch",
                   "variants": variants, "sizes": sizes, "threads_per_launch": n, "block": args.block,
                   "heap_bytes": heap_bytes, "cells": configured_cells, "l2": f"flushed ({args.flush_mib} MiB) before every timed launch",
                   "parallelism": f"replicas x{world}"},
        "alloc_ms_total": round(alloc_ms, 3), "free_ms_total": round(free_ms, 3),
        "wall_s": round(wall, 3), "null_results": nulls, "bad_words": bad,
        "gpu_launches": 4 * len(cells) * args.steps if args.impl == "ours" else 0,
        "timed_region": "per cell: W warm-up + K timed repetitions on a fresh heap; value = all mallocs and frees / "
                        "summed alloc + free kernel time",
        "clocks": clocks, "per_cell": per_cell,
        "cells_measured": len(cells),
        "cold": cold_summary(res, n),
    }
    if args.impl == "reference":
        out["cells_unavailable"] = skipped
    else:
        vs = against_reference_cells(per_cell, out["cold"]["per_cell"])
        if vs:
            out["per_cell_vs_reference"] = vs
    if args.impl != "reference" and value_ref_cells:
        out["value_on_reference_cells"] = {
            "value": round(value_ref_cells, 3), "unit": "Mops/s", "cells": len(ref_cells),
            "what": "the same aggregate over the cells the reference arm measures (all but "
                    + ", ".join(sorted(REFERENCE_FAULTED)) + ", whose reference code faulted)"}
    if rank == 0 and not args.no_config1:
        try:
            out["config1"] = config1_bench(ReferenceArm if args.impl == "reference" else OursArm, stream)
        except Exception as exc:   # reported, the headline stands
            out["config1"] = {"error": str(exc)[:300]}
    if rank == 0 and not args.no_traces:
        try:
            out["per_thread_traces"] = trace_configs(ReferenceArm if args.impl == "reference" else OursArm, stream,
                                                     args.impl == "reference")
        except Exception as exc:   # reported, the headline stands
            out["per_thread_traces"] = {"error": str(exc)[:300]}
    if args.impl == "reference":
        out["impl"] = "reference"
        out["gpu_launches"] = 0
        out["e2e"] = {"value": out["value"], "unit": "Mops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        out["cpu_baseline"] = {"value": out["value"], "unit": "Mops/s", "cores": 1, "kind": "reference",
                               "sample": "the reference's own CUDA code (sm_100a build of its sources) on the "
                                         "same B200, the same cells, launch shape and timing; the reference "
                                         "has no host implementation"}
    else:
        out["extra"] = extra
        if e2e_ms:
            e2e_ops = 2.0 * n * len(cells) * world
            out["e2e"] = {"value": round(e2e_ops / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mops/s",
                          "h2d_bytes_per_step": 4 * n * len(cells), "d2h_bytes_per_step": 8 * n * len(cells),
                          "what": "per cell, after the timed repetitions, through the C ABI: one "
                                  "ouro_alloc_host call (request sizes host->device from pinned memory, alloc, "
                                  "pointer array device->host, in %d slices whose copies overlap the other "
                                  "slices' launches) and ouro_free of the device copy of the pointers"
                                  % E2E_SLICES}
        out["roofline"] = roofline(res, n, args.steps)
        extras = rank == 0   # the configurations beyond the headline: one replica measures them
        if extras and not args.no_churn:
            try:
                out["churn"] = churn_bench(args.churn_rounds, stream)
            except Exception as exc:   # reported, the headline stands
                out["churn"] = {"error": str(exc)[:300]}
        if extras and not args.no_serving:
            try:
                out["serving"] = serving_bench(args.serving_seconds)
            except Exception as exc:   # reported, the headline stands
                out["serving"] = {"error": str(exc)[:300]}
        if extras and not args.no_batched:
            try:
                out["batched"] = batched_bench(args.batched_n, args.batched_cycles, stream)
            except Exception as exc:   # reported, the headline stands
                out["batched"] = {"error": str(exc)[:300]}
        if not args.no_cpu and rank == 0:
            out["cpu_baseline"] = cpu_baseline(cells, n, heap_bytes)
    if rank == 0:
        print(json.dumps(out))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
