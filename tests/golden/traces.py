"""Deterministic request traces for the sequential parity checks.

A trace is a flat uint32 array of (kind, arg) pairs: kind 0 = malloc(arg bytes),
kind 1 = free(the pointer returned by op number arg), kind 2 = take a chunk from
the heap (the reference's allocateChunk), kind 3 = enqueue such a chunk as an
initial chunk (the reference's enqueueInitialChunk; arg = op << 14 |
available pages << 4 | queue index), kind 4 = free page (arg & 1023) of such a
chunk (arg = op << 10 | page).  The same traces are
replayed by one GPU thread through the reference build (make_golden.py), by the
C oracle and by the CUDA allocator of this repository.  Every trace stays far
from the heap's capacity and from the reference's queue limits, so that the
reference runs it with defined behaviour.
"""
from __future__ import annotations

import numpy as np

HEAP_BYTES = 1 << 30


class _Builder:
    def __init__(self):
        self.ops: list[int] = []
        self.live: list[int] = []

    def malloc(self, size: int) -> int:
        i = len(self.ops) // 2
        self.ops += [0, int(size)]
        self.live.append(i)
        return i

    def free(self, i: int):
        self.ops += [1, int(i)]
        self.live.remove(i)

    def alloc_chunk(self) -> int:
        i = len(self.ops) // 2
        self.ops += [2, 0]
        return i

    def enqueue_initial(self, chunk_op: int, queue_index: int, available: int):
        self.ops += [3, (chunk_op << 14) | (available << 4) | queue_index]

    def free_page(self, chunk_op: int, page: int):
        self.ops += [4, (chunk_op << 10) | page]

    def free_all(self, order=None):
        for i in list(self.live if order is None else order):
            self.free(i)

    def free_many(self, ids):
        """free(i) for every i of ids, in that order, with one pass over the
        live list (free() searches it once per call)."""
        ids = [int(i) for i in ids]
        for i in ids:
            self.ops += [1, i]
        gone = set(ids)
        assert len(gone) == len(ids) and gone <= set(self.live)
        self.live = [i for i in self.live if i not in gone]

    def array(self) -> np.ndarray:
        return np.asarray(self.ops, dtype=np.uint32)


def basic() -> np.ndarray:
    """Fixed 64 B requests: fill, free every other one, refill, free all."""
    b = _Builder()
    first = [b.malloc(64) for _ in range(300)]
    for i in first[::2]:
        b.free(i)
    for _ in range(200):
        b.malloc(64)
    b.free_all()
    return b.array()


def mixed(seed: int = 1, n_ops: int = 3000) -> np.ndarray:
    """Random mix: log-uniform sizes up to 8 KiB, some 8-32 KiB (second
    instance), a few above 32 KiB (CUDA device heap), one size 0; frees of
    random live allocations; everything freed at the end."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    b.malloc(0)
    tier2 = 0
    for _ in range(n_ops):
        if b.live and rng.random() < 0.4:
            b.free(b.live[int(rng.integers(len(b.live)))])
            continue
        u = rng.random()
        if u < 0.90 or tier2 >= 300:
            size = int(np.exp(rng.uniform(0.0, np.log(8192.0))))
        elif u < 0.99:
            size = int(rng.integers(8193, 32769))
            tier2 += 1
        else:
            size = int(rng.integers(32769, 65537))
        b.malloc(max(size, 1))
    order = list(b.live)
    rng.shuffle(order)
    b.free_all(order)
    return b.array()


def churn(size: int = 16, n: int = 5000, rounds: int = 6) -> np.ndarray:
    """Many same-class requests: enough queue traffic to allocate, drain and
    recycle queue chunks of the virtualized variants (2048 entries each)."""
    b = _Builder()
    for r in range(rounds):
        ids = [b.malloc(size) for _ in range(n)]
        b.free_all(ids if r % 2 == 0 else ids[::-1])
    return b.array()


def chunk_fifo() -> np.ndarray:
    """Chunk-queue order: fill three 1 KiB chunks (8 pages each), free pages in
    C, A, B order so they re-enter the queue in that order, then reallocate."""
    b = _Builder()
    ids = [b.malloc(1024) for _ in range(24)]
    a, bb, c = ids[0:8], ids[8:16], ids[16:24]
    for i in (c[3], a[5], bb[0], a[7], c[6]):
        b.free(i)
    for _ in range(7):
        b.malloc(1000)
    b.free_all()
    return b.array()


def tier2() -> np.ndarray:
    """Second instance only: 16 KiB and 32 KiB pages in 4-base-chunk chunks."""
    b = _Builder()
    ids = [b.malloc(16384 if i % 3 else 32768) for i in range(60)]
    for i in ids[::2]:
        b.free(i)
    for i in range(40):
        b.malloc(12000 if i % 2 else 30000)
    b.free_all()
    return b.array()


def initial() -> np.ndarray:
    """Initial chunks (enqueueInitialChunk): on a fresh heap one chunk each for
    64 B, 512 B and 2 KiB pages joins its class with its first pages in the
    caller's use; mallocs take the initial pages first and then grow; the
    caller's pages are freed along the way; everything freed at the end.  One
    initial chunk per class: the reference's standard and virtualized-array
    chunk queues accept it only as a class's first operation."""
    b = _Builder()
    c64, c512, c2k = b.alloc_chunk(), b.alloc_chunk(), b.alloc_chunk()
    b.enqueue_initial(c64, 2, 125)     # pages 0..2 held by the caller
    b.enqueue_initial(c512, 5, 10)     # pages 0..5 held
    b.enqueue_initial(c2k, 7, 3)       # page 0 held
    m64 = [b.malloc(64) for _ in range(200)]
    m512 = [b.malloc(512) for _ in range(20)]
    m2k = [b.malloc(2048) for _ in range(5)]
    b.free_page(c64, 1)
    b.free_page(c512, 0)
    b.free_page(c512, 5)
    b.free_page(c2k, 0)
    for i in m64[::2]:
        b.free(i)
    for _ in range(50):
        b.malloc(64)
    b.free_page(c64, 0)
    b.free_page(c64, 2)
    for p in range(1, 5):
        b.free_page(c512, p)
    for i in m512[3:9] + m2k[1:3]:
        b.free(i)
    b.malloc(512)
    b.malloc(2048)
    b.free_all()
    return b.array()


def large(seed: int = 3) -> np.ndarray:
    """At scale, on a 4 GiB heap: 2^15 requests of 2 KiB, 2^16 of 64 B and
    2^14 of 8 KiB (about 25,000 chunks; the 64 B page queue passes through 32
    queue chunks), then a third of the small requests and all the 8 KiB ones
    freed in a random order (chunk-based queues re-enqueue partly used chunks
    and return the emptied ones to the reuse queue), 2^15 re-allocations of
    64 B .. 8 KiB that take those pages and chunks again, and everything freed
    in the reverse order of allocation."""
    rng = np.random.default_rng(seed)
    b = _Builder()
    k2 = [b.malloc(2048) for _ in range(1 << 15)]
    s64 = [b.malloc(64) for _ in range(1 << 16)]
    k8 = [b.malloc(8192) for _ in range(1 << 14)]
    victims = np.asarray(k2[::3] + s64[1::3] + k8)
    b.free_many(victims[rng.permutation(victims.size)])
    for size in rng.choice(np.asarray([64, 1024, 2048, 8192]), size=1 << 15):
        b.malloc(int(size))
    b.free_many(b.live[::-1])
    return b.array()


# name -> (builder, tid, bid): the GPU thread that replays the trace
TRACES = {
    "basic": (basic, 0, 0),
    "mixed": (lambda: mixed(1), 0, 0),
    "mixed_t37b5": (lambda: mixed(2), 37, 5),
    "churn16": (lambda: churn(16), 0, 0),
    "churn512": (lambda: churn(512, 2500, 4), 0, 0),
    "chunk_fifo": (chunk_fifo, 0, 0),
    "tier2": (tier2, 0, 0),
    "initial": (initial, 0, 0),
    "large4g": (large, 0, 0),
}

# traces replayed on a heap other than HEAP_BYTES
HEAPS = {"large4g": 4 << 30}

# traces whose reference offsets are pinned by their SHA-256 instead of being
# stored whole (the fixture would hold about 200,000 of them per variant)
DIGEST_ONLY = {"large4g"}


def heap_bytes(name: str) -> int:
    return HEAPS.get(name, HEAP_BYTES)


def build(name: str):
    fn, tid, bid = TRACES[name]
    return fn(), tid, bid
