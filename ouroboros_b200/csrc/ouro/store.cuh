// store.cuh -- the three queue storages behind both queue families.
//
//  FlatStore  standard array queues: one ring per class (PageQueue.cuh /
//             ChunkQueue.cuh: 2^23 entries).
//  VaStore    virtualized array (PageQueueVA.cuh / ChunkQueueVA.cuh): 2048-entry
//             queue chunks taken from the heap, found through a 16384-entry
//             index array; a queue chunk returns to the chunk pool once drained.
//  VlStore    virtualized linked list (PageQueueVL.cuh / ChunkQueueVL.cuh):
//             queue chunks linked through their metadata; the ten most recently
//             drained ones are held back before reuse (QueueChunk_impl.cuh:494-551).
//
// Positions are virtual (monotone u32).  Page queues hand out entries by
// position (consume_lane); chunk queues scan them (peek / remove).  Groups of
// lanes always own contiguous positions, so every slot access of a warp is one
// coalesced request.
#pragma once

#include "heap.cuh"

namespace ouro {

__device__ __forceinline__ int lane_of_rank(uint32_t mask, int r) {
  return static_cast<int>(__fns(mask, 0u, r + 1));
}

// Wait until a slot holds `want` (kEmpty before writing) -- bounded.
__device__ __forceinline__ bool wait_slot_empty(HeapCore* h, uint32_t* s) {
  uint32_t it = 0;
  while (ld_relaxed(s) != kEmpty) {
    if (it >= kSpinLimit) { note_timeout(h); return false; }
    backoff(it);
  }
  return true;
}

// Take the value of a slot once it is there and clear the slot -- bounded.
__device__ __forceinline__ uint32_t take_slot(HeapCore* h, uint32_t* s) {
  uint32_t v, it = 0;
  while ((v = ld_acquire(s)) == kEmpty) {
    if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
    backoff(it);
  }
  st_relaxed(s, kEmpty);
  return v;
}

// ================================================================= flat
struct FlatStore {
  static constexpr int kKind = 0;

  __device__ static uint32_t* slot(ClassState* q, uint32_t pos) { return q->ring + (pos & q->ring_mask); }

  // Group writes E entries at [b, b + E); value(j, cj) computes entry j from
  // the chunk held by group rank j / per_lane_chunk.
  template <bool PageQueue, typename Value>
  __device__ static void publish_range(HeapCore* h, ClassState* q, const Group& g, uint32_t b, uint32_t E,
                                       uint32_t chunk, uint32_t entries_per_chunk, Value&& value) {
    const uint32_t n = static_cast<uint32_t>(g.size);
    const uint32_t rounds = (E + n - 1u) / n;
    for (uint32_t i = 0; i < rounds; ++i) {
      uint32_t j = static_cast<uint32_t>(g.rank) + i * n;
      int src = j < E ? lane_of_rank(g.mask, static_cast<int>(j / entries_per_chunk)) : g.leader;
      uint32_t cj = __shfl_sync(g.mask, chunk, src);
      if (j < E) {
        uint32_t* s = slot(q, b + j);
        if (wait_slot_empty(h, s)) st_relaxed(s, value(j, cj));
      }
    }
  }

  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    uint32_t* s = slot(q, pos);
    if (wait_slot_empty(h, s)) st_relaxed(s, v);
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    return take_slot(h, slot(q, pos));
  }

  // ---- chunk-queue side
  __device__ static bool enqueue_one(HeapCore* h, ClassState* q, uint32_t c, uint32_t* qpos) {
    uint32_t b = atomicAdd(&q->back.v, 1u);
    uint32_t* s = slot(q, b);
    if (!wait_slot_empty(h, s)) return false;
    st_relaxed(qpos, b);
    __threadfence();
    st_release(s, c);
    return true;
  }
  struct Cursor { uint32_t unused; };
  __device__ static Cursor cursor(ClassState*) { return Cursor{0}; }
  __device__ static uint32_t peek(HeapCore* h, ClassState* q, uint32_t pos, Cursor&) { return ld_acquire(slot(q, pos)); }
  __device__ static void remove(HeapCore* h, ClassState* q, uint32_t pos) { st_relaxed(slot(q, pos), kTomb); }

  // Move the front past removed entries, freeing their slots for the next lap.
  __device__ static void advance_front(HeapCore* h, ClassState* q) {
    for (uint32_t i = 0; i < 64u; ++i) {
      uint32_t f = ld_relaxed(&q->front.v);
      if (static_cast<int32_t>(ld_relaxed(&q->back.v) - f) <= 0) return;
      uint32_t* s = slot(q, f);
      if (ld_relaxed(s) != kTomb) return;
      if (atomicCAS(&q->front.v, f, f + 1u) == f) st_relaxed(s, kEmpty);
    }
  }
};

// ==================================================== virtualized array
struct VaStore {
  static constexpr int kKind = 1;

  __device__ static uint32_t vid(uint32_t pos) { return (pos / kQcSpots) & (kVqSize - 1u); }

  // The queue chunk holding pos (spins while its pre-allocation is in flight).
  __device__ static uint32_t qchunk(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t* e = q->ring + vid(pos);
    uint32_t c, it = 0;
    while ((c = ld_acquire(e)) == kEmpty) {
      if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
      backoff(it);
    }
    if (ld_relaxed(&h->meta[c].vstart) / kQcSpots != pos / kQcSpots) {
      set_status(h, kErrCorrupt);
      return kEmpty;
    }
    return c;
  }

  // The producer of a position at the start of a queue chunk allocates the
  // next queue chunk (PageQueueVA_impl.cuh:45-56, :202-212).
  __device__ static void preallocate(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t nq = new_queue_chunk(h, q->inst, pos + kQcSpots);
    if (nq != kEmpty) st_release(q->ring + vid(pos + kQcSpots), nq);
  }

  // Drained queue chunk back to the chunk pool (PageQueueVA_impl.cuh:159-166).
  __device__ static void recycle(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t c = atomicExch(q->ring + vid(pos), kEmpty);
    if (c != kEmpty) reuse_put(h, &h->reuse[0], c);
  }

  // Count update of a range: m entries enqueued into the chunk of pos.
  __device__ static void count_enqueued(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos, uint32_t m, bool recycle_ok) {
    uint32_t add = (m << 16) + m;
    uint32_t old = atomicAdd(&h->meta[c].qcount, add);
    if (recycle_ok && old + add == kQcSpots) recycle(h, q, pos);
  }

  template <bool PageQueue, typename Value>
  __device__ static void publish_range(HeapCore* h, ClassState* q, const Group& g, uint32_t b, uint32_t E,
                                       uint32_t chunk, uint32_t entries_per_chunk, Value&& value) {
    const uint32_t n = static_cast<uint32_t>(g.size);
    const uint32_t rounds = (E + n - 1u) / n;
    for (uint32_t i = 0; i < rounds; ++i) {
      uint32_t j = static_cast<uint32_t>(g.rank) + i * n;
      if (j < E && ((b + j) % kQcSpots) == 0u) preallocate(h, q, b + j);
    }
    uint32_t c1 = kEmpty, c2 = kEmpty;
    const uint32_t split = kQcSpots - (b % kQcSpots);   // entries that land in the first queue chunk
    for (uint32_t i = 0; i < rounds; ++i) {
      uint32_t j = static_cast<uint32_t>(g.rank) + i * n;
      int src = j < E ? lane_of_rank(g.mask, static_cast<int>(j / entries_per_chunk)) : g.leader;
      uint32_t cj = __shfl_sync(g.mask, chunk, src);
      if (j < E) {
        uint32_t p = b + j;
        uint32_t qc = qchunk(h, q, p);
        if (qc == kEmpty) continue;
        if (j < split) c1 = qc; else c2 = qc;
        uint32_t* s = queue_slots(h, qc) + (p % kQcSpots);
        if (wait_slot_empty(h, s)) st_relaxed(s, value(j, cj));
      }
    }
    __syncwarp(g.mask);
    __threadfence();
    // the leader may not have touched both chunks: take them from any lane
    c1 = __reduce_min_sync(g.mask, c1);
    c2 = __reduce_min_sync(g.mask, c2);
    if (g.is_leader()) {
      uint32_t m1 = E < split ? E : split;
      if (c1 != kEmpty && m1) count_enqueued(h, q, c1, b, m1, PageQueue);
      if (c2 != kEmpty && E > m1) count_enqueued(h, q, c2, b + m1, E - m1, PageQueue);
    }
  }

  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    if (pos % kQcSpots == 0u) preallocate(h, q, pos);
    uint32_t qc = qchunk(h, q, pos);
    if (qc != kEmpty) {
      uint32_t* s = queue_slots(h, qc) + (pos % kQcSpots);
      if (wait_slot_empty(h, s)) st_relaxed(s, v);
    }
    __syncwarp(g.mask);
    __threadfence();
    Group cg = group_by(g.mask, qc);
    if (cg.is_leader() && qc != kEmpty) count_enqueued(h, q, qc, pos, static_cast<uint32_t>(cg.size), true);
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    uint32_t qc = qchunk(h, q, pos);
    uint32_t v = kEmpty;
    if (qc != kEmpty) v = take_slot(h, queue_slots(h, qc) + (pos % kQcSpots));
    __syncwarp(g.mask);
    Group cg = group_by(g.mask, qc);
    if (cg.is_leader() && qc != kEmpty) {
      uint32_t sub = static_cast<uint32_t>(cg.size) << 16;
      uint32_t old = atomicSub(&h->meta[qc].qcount, sub);
      if (old - sub == kQcSpots) recycle(h, q, pos);
    }
    return v;
  }

  // ---- chunk-queue side (front-driven recycling, see advance_front)
  __device__ static bool enqueue_one(HeapCore* h, ClassState* q, uint32_t c, uint32_t* qpos) {
    uint32_t b = atomicAdd(&q->back.v, 1u);
    if (b % kQcSpots == 0u) preallocate(h, q, b);
    uint32_t qc = qchunk(h, q, b);
    if (qc == kEmpty) return false;
    uint32_t* s = queue_slots(h, qc) + (b % kQcSpots);
    if (!wait_slot_empty(h, s)) return false;
    st_relaxed(qpos, b);
    __threadfence();
    st_release(s, c);
    atomicAdd(&h->meta[qc].qcount, (1u << 16) + 1u);
    return true;
  }
  struct Cursor { uint32_t unused; };
  __device__ static Cursor cursor(ClassState*) { return Cursor{0}; }
  __device__ static uint32_t peek(HeapCore* h, ClassState* q, uint32_t pos, Cursor&) {
    uint32_t qc = ld_acquire(q->ring + vid(pos));
    if (qc == kEmpty) return kEmpty;
    if (ld_relaxed(&h->meta[qc].vstart) / kQcSpots != pos / kQcSpots) return kTomb;
    return ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
  }
  __device__ static void remove(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t qc = ld_acquire(q->ring + vid(pos));
    if (qc == kEmpty) return;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    atomicSub(&h->meta[qc].qcount, 1u << 16);
  }
  // Front moves over removed entries; passing the last entry of a queue chunk
  // returns that chunk to the pool (ChunkQueueVA_impl.cuh:144-156).
  __device__ static void advance_front(HeapCore* h, ClassState* q) {
    for (uint32_t i = 0; i < 64u; ++i) {
      uint32_t f = ld_relaxed(&q->front.v);
      if (static_cast<int32_t>(ld_relaxed(&q->back.v) - f) <= 0) return;
      uint32_t qc = ld_acquire(q->ring + vid(f));
      if (qc == kEmpty) return;
      if (ld_acquire(queue_slots(h, qc) + (f % kQcSpots)) != kTomb) return;
      if (atomicCAS(&q->front.v, f, f + 1u) == f && ((f + 1u) % kQcSpots) == 0u) {
        uint32_t c = atomicExch(q->ring + vid(f), kEmpty);
        if (c != kEmpty) reuse_put(h, &h->reuse[0], c);
      }
    }
  }
};

// ===================================================== virtualized linked
struct VlStore {
  static constexpr int kKind = 2;
  static constexpr uint32_t kBehind = 0xFFFFFFFDu;

  // Walk from `from` to the queue chunk holding pos (QueueChunk_impl.cuh:403-426).
  // Returns kBehind when pos precedes `from`, kEmpty on timeout.
  __device__ static uint32_t locate(HeapCore* h, uint32_t from, uint32_t pos) {
    uint32_t cur = from, it = 0;
    for (uint32_t hops = 0; hops < (1u << 20); ++hops) {
      uint32_t vs = ld_relaxed(&h->meta[cur].vstart) / kQcSpots;
      uint32_t want = pos / kQcSpots;
      if (vs == want) return cur;
      if (static_cast<int32_t>(want - vs) < 0) return kBehind;
      uint32_t nx;
      while ((nx = ld_acquire(&h->meta[cur].next)) == kEmpty) {
        if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
        backoff(it);
      }
      cur = nx;
    }
    note_timeout(h);
    return kEmpty;
  }

  __device__ static uint32_t next_of(HeapCore* h, uint32_t c) {
    uint32_t nx, it = 0;
    while ((nx = ld_acquire(&h->meta[c].next)) == kEmpty) {
      if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
      backoff(it);
    }
    return nx;
  }

  // QueueChunk_impl.cuh:440-463 setBackPointer
  __device__ static void set_back(HeapCore* h, ClassState* q, uint32_t cur) {
    for (uint32_t i = 0; i < (1u << 16); ++i) {
      uint32_t nx = ld_acquire(&h->meta[cur].next);
      if (nx == kEmpty) return;
      if (atomicCAS(&q->back_ptr, cur, nx) != cur) return;
      if ((ld_relaxed(&h->meta[nx].qcount) & 0xFFFFu) == kQcSpots) cur = nx;
      else return;
    }
  }

  // QueueChunk_impl.cuh:467-490 setFrontPointer
  __device__ static uint32_t set_front(HeapCore* h, ClassState* q, uint32_t cur) {
    uint32_t ret = 0;
    for (uint32_t i = 0; i < (1u << 16); ++i) {
      uint32_t nx = ld_acquire(&h->meta[cur].next);
      if (nx == kEmpty) break;
      if (atomicCAS(&q->front_ptr, cur, nx) != cur) break;
      ++ret;
      if (ld_relaxed(&h->meta[nx].qcount) == kQcSpots) cur = nx;
      else break;
    }
    return ret;
  }

  // QueueChunk_impl.cuh:494-551 setOldPointer: drained chunks are held back
  // (up to kOldHold) before they return to the pool, so that a lane that read
  // front/back a little while ago can still walk forward from it.
  __device__ static void set_old(HeapCore* h, ClassState* q, uint32_t freed) {
    uint32_t cur = ld_relaxed(&q->old_count);
    if (cur < kOldHold) {
      cur = atomicAdd(&q->old_count, freed);
      if (cur < kOldHold) {
        if (cur + freed > kOldHold) {
          freed = cur + freed - kOldHold;
          atomicSub(&q->old_count, freed);
        } else {
          freed = 0;
        }
      }
    }
    uint32_t old = ld_relaxed(&q->old_ptr);
    for (uint32_t guard = 0; freed > 0 && guard < (1u << 20); ++guard) {
      uint32_t nx = ld_acquire(&h->meta[old].next);
      uint32_t seen = atomicCAS(&q->old_ptr, old, nx);
      if (seen == old) {
        --freed;
        reuse_put(h, &h->reuse[0], old);
        old = nx;
      } else {
        old = seen;
      }
    }
  }

  __device__ static void on_empty(HeapCore* h, ClassState* q, uint32_t c) {
    uint32_t n = set_front(h, q, c);
    set_old(h, q, n);
  }

  // Count update of m enqueued entries into chunk c (QueueChunk_impl.cuh:160-182).
  __device__ static void count_enqueued(HeapCore* h, ClassState* q, uint32_t c, uint32_t m) {
    uint32_t add = (m << 16) + m;
    uint32_t old = atomicAdd(&h->meta[c].qcount, add);
    if ((old & 0xFFFFu) + m == kQcSpots) set_back(h, q, c);
    if (old + add == kQcSpots) on_empty(h, q, c);
  }

  __device__ static void count_removed(HeapCore* h, ClassState* q, uint32_t c, uint32_t m) {
    uint32_t sub = m << 16;
    uint32_t old = atomicSub(&h->meta[c].qcount, sub);
    if (old - sub == kQcSpots) on_empty(h, q, c);
  }

  // A producer at the start of a queue chunk links the next one (QueueChunk_impl.cuh:144-158).
  __device__ static void preallocate(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos) {
    uint32_t nq = new_queue_chunk(h, q->inst, pos + kQcSpots);
    if (nq != kEmpty) st_release(&h->meta[c].next, nq);
  }

  template <bool PageQueue, typename Value>
  __device__ static void publish_range(HeapCore* h, ClassState* q, const Group& g, uint32_t b, uint32_t E,
                                       uint32_t chunk, uint32_t entries_per_chunk, Value&& value) {
    const uint32_t n = static_cast<uint32_t>(g.size);
    const uint32_t rounds = (E + n - 1u) / n;
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate(h, ld_acquire(&q->back_ptr), b);
    c1 = bcast(g, c1);
    if (c1 == kEmpty || c1 == kBehind) { set_status(h, kErrCorrupt); return; }
    const uint32_t split = kQcSpots - (b % kQcSpots);
    // the lane holding the first position of a queue chunk links the next one
    for (uint32_t i = 0; i < rounds; ++i) {
      uint32_t j = static_cast<uint32_t>(g.rank) + i * n;
      if (j < E && ((b + j) % kQcSpots) == 0u) preallocate(h, q, j < split ? c1 : next_of(h, c1), b + j);
    }
    uint32_t c2 = E > split ? kEmpty : c1;
    for (uint32_t i = 0; i < rounds; ++i) {
      uint32_t j = static_cast<uint32_t>(g.rank) + i * n;
      int src = j < E ? lane_of_rank(g.mask, static_cast<int>(j / entries_per_chunk)) : g.leader;
      uint32_t cj = __shfl_sync(g.mask, chunk, src);
      if (j < E) {
        uint32_t qc = c1;
        if (j >= split) {
          if (c2 == kEmpty) c2 = next_of(h, c1);
          qc = c2;
        }
        if (qc == kEmpty) continue;
        uint32_t* s = queue_slots(h, qc) + ((b + j) % kQcSpots);
        st_relaxed(s, value(j, cj));   // linked slots are written once per lap (enqueueLinked)
      }
    }
    __syncwarp(g.mask);
    __threadfence();
    if (g.is_leader()) {
      uint32_t m1 = E < split ? E : split;
      count_enqueued(h, q, c1, m1);
      if (E > m1) {
        uint32_t cc = next_of(h, c1);
        if (cc != kEmpty) count_enqueued(h, q, cc, E - m1);
      }
    }
  }

  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate(h, ld_acquire(&q->back_ptr), first);
    c1 = bcast(g, c1);
    uint32_t qc = kEmpty;
    if (c1 != kEmpty && c1 != kBehind) {
      qc = (pos / kQcSpots == first / kQcSpots) ? c1 : next_of(h, c1);
      if (qc != kEmpty) {
        if (pos % kQcSpots == 0u) preallocate(h, q, qc, pos);
        st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), v);
      }
    } else {
      set_status(h, kErrCorrupt);
    }
    __syncwarp(g.mask);
    __threadfence();
    Group cg = group_by(g.mask, qc);
    if (cg.is_leader() && qc != kEmpty) count_enqueued(h, q, qc, static_cast<uint32_t>(cg.size));
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate(h, ld_acquire(&q->front_ptr), first);
    c1 = bcast(g, c1);
    uint32_t qc = kEmpty, v = kEmpty;
    if (c1 != kEmpty && c1 != kBehind) {
      qc = (pos / kQcSpots == first / kQcSpots) ? c1 : next_of(h, c1);
      if (qc != kEmpty) v = take_slot(h, queue_slots(h, qc) + (pos % kQcSpots));
    } else {
      set_status(h, kErrCorrupt);
    }
    __syncwarp(g.mask);
    Group cg = group_by(g.mask, qc);
    if (cg.is_leader() && qc != kEmpty) count_removed(h, q, qc, static_cast<uint32_t>(cg.size));
    return v;
  }

  // ---- chunk-queue side
  __device__ static bool enqueue_one(HeapCore* h, ClassState* q, uint32_t c, uint32_t* qpos) {
    uint32_t b = atomicAdd(&q->back.v, 1u);
    uint32_t qc = locate(h, ld_acquire(&q->back_ptr), b);
    if (qc == kEmpty || qc == kBehind) { set_status(h, kErrCorrupt); return false; }
    if (b % kQcSpots == 0u) preallocate(h, q, qc, b);
    st_relaxed(qpos, b);
    __threadfence();
    st_release(queue_slots(h, qc) + (b % kQcSpots), c);
    __threadfence();
    count_enqueued(h, q, qc, 1u);
    return true;
  }
  struct Cursor { uint32_t chunk; };
  __device__ static Cursor cursor(ClassState* q) { return Cursor{ld_acquire(&q->front_ptr)}; }
  __device__ static uint32_t peek(HeapCore* h, ClassState* q, uint32_t pos, Cursor& cur) {
    uint32_t qc = locate(h, cur.chunk, pos);
    if (qc == kBehind) {
      cur.chunk = ld_acquire(&q->front_ptr);
      return kTomb;
    }
    if (qc == kEmpty) return kEmpty;
    cur.chunk = qc;
    return ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
  }
  __device__ static void remove(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t qc = locate(h, ld_acquire(&q->front_ptr), pos);
    if (qc == kEmpty || qc == kBehind) return;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    __threadfence();
    count_removed(h, q, qc, 1u);
  }
  __device__ static void advance_front(HeapCore* h, ClassState* q) {
    uint32_t cur = ld_acquire(&q->front_ptr);
    for (uint32_t i = 0; i < 64u; ++i) {
      uint32_t f = ld_relaxed(&q->front.v);
      if (static_cast<int32_t>(ld_relaxed(&q->back.v) - f) <= 0) return;
      uint32_t qc = locate(h, cur, f);
      if (qc == kEmpty) return;
      if (qc == kBehind) {
        // front lags the first live queue chunk: everything before it is gone
        uint32_t start = ld_relaxed(&h->meta[cur].vstart);
        start -= start % kQcSpots;
        if (static_cast<int32_t>(start - f) > 0) atomicCAS(&q->front.v, f, start);
        continue;
      }
      cur = qc;
      if (ld_acquire(queue_slots(h, qc) + (f % kQcSpots)) != kTomb) return;
      atomicCAS(&q->front.v, f, f + 1u);
    }
  }
};

}  // namespace ouro
