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

// ------------------------------------------------ front advance (groups)
// The front of a chunk queue moves over removed entries (kTomb).  One group at
// a time does it (queues.cuh: help_front): its lanes read 4 consecutive
// entries each per round with one 16-byte load, so a round covers 4 x group
// size entries and the first live entry is found with one ballot.  Positions
// before `from` count as removed, positions at or after `back` as live.
// Rounds per advance: 256 (32768 entries for a full warp), and at least
// 8192 entries for small groups.
__device__ __forceinline__ uint32_t front_rounds(uint32_t n) { return 2048u / n > 256u ? 2048u / n : 256u; }

__device__ __forceinline__ bool first_live4(const Group& g, uint32_t p, uint4 e, uint32_t from, uint32_t back,
                                            uint32_t* stop) {
  const uint32_t v[4] = {e.x, e.y, e.z, e.w};
  uint32_t idx = 4u;
#pragma unroll
  for (int k = 3; k >= 0; --k) {
    const uint32_t pos = p + static_cast<uint32_t>(k);
    const bool behind = static_cast<int32_t>(pos - from) < 0;
    const bool beyond = static_cast<int32_t>(pos - back) >= 0;
    if (!behind && (beyond || v[k] != kTomb)) idx = static_cast<uint32_t>(k);
  }
  const uint32_t m = __ballot_sync(g.mask, idx < 4u);
  if (!m) return false;
  *stop = __shfl_sync(g.mask, p + idx, __ffs(m) - 1);
  return true;
}

// Claim [from, stop) for the front with one CAS (from = the front we read).
// Returns the start of the part this group moved the front over (== stop when
// another group got at least as far).
__device__ __forceinline__ uint32_t claim_front(ClassState* q, uint32_t from, uint32_t stop) {
  uint32_t cur = from;
  for (;;) {
    const uint32_t seen = atomicCAS(&q->front.v, cur, stop);
    if (seen == cur) return cur;
    if (static_cast<int32_t>(seen - stop) >= 0) return stop;   // someone else moved it at least as far
    cur = seen;                                                 // [seen, stop) is still ours to pass
  }
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
  __device__ static void advance_front(HeapCore* h, ClassState* q, const Group& g) {
    uint32_t f = 0, back = 0;
    if (g.is_leader()) {
      f = ld_relaxed(&q->front.v);
      back = ld_relaxed(&q->back.v);
    }
    f = bcast(g, f);
    back = bcast(g, back);
    if (static_cast<int32_t>(back - f) <= 0) return;
    const uint32_t n = static_cast<uint32_t>(g.size);
    uint32_t a = f & ~3u, stop = 0;
    bool found = false;
    for (uint32_t r = 0, rounds = front_rounds(n); r < rounds && !found; ++r, a += 4u * n) {
      const uint32_t p = a + 4u * static_cast<uint32_t>(g.rank);
      // ring positions are 4-aligned here and the ring size is a multiple of 4
      const uint4 e = static_cast<int32_t>(p - back) < 0 ? ld_relaxed_v4(slot(q, p)) : make_uint4(0, 0, 0, 0);
      found = first_live4(g, p, e, f, back, &stop);
      if (!found && static_cast<int32_t>(a + 4u * n - back) >= 0) {
        stop = back;
        found = true;
      }
    }
    if (!found) stop = a;
    if (static_cast<int32_t>(stop - f) <= 0) return;
    uint32_t cur = 0;
    if (g.is_leader()) cur = claim_front(q, f, stop);
    cur = bcast(g, cur);
    for (uint32_t p = cur + static_cast<uint32_t>(g.rank); p != stop && static_cast<int32_t>(p - stop) < 0; p += n)
      st_relaxed(slot(q, p), kEmpty);
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
    while ((c = ld_acquire(e)) == kEmpty || c == kInstalling) {
      if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
      if (c == kEmpty && it >= kInstallAfter && (it & 63u) == 0u)
        install_queue_chunk(h, e, q->inst, pos - pos % kQcSpots);
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
    offer_queue_chunk(h, q->ring + vid(pos + kQcSpots), new_queue_chunk(h, q->inst, pos + kQcSpots));
  }

  // Drained queue chunk back to the chunk pool (PageQueueVA_impl.cuh:159-166).
  __device__ static void recycle(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t c = atomicExch(q->ring + vid(pos), kEmpty);
    if (c < kInstalling) reuse_put(h, &h->reuse[0], c);
  }

  // Count update of a range: m entries enqueued into the chunk of pos.
  __device__ static void count_enqueued(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos, uint32_t m, bool recycle_ok) {
    uint32_t add = (m << 16) + m;
    uint32_t old = atomicAdd(&h->meta[c].qcount, add);
    if (recycle_ok && old + add == kQcSpots) recycle(h, q, pos);
  }

  // The lanes of a group hold contiguous positions that span at most two
  // queue chunks.  Each half is written and counted on its own, so the count
  // of the first chunk never waits for the second chunk to appear.
  __device__ static Group half_of(const Group& g, uint32_t pos, uint32_t first) {
    const bool second = pos / kQcSpots != first / kQcSpots;
    const uint32_t m2 = __ballot_sync(g.mask, second);
    return make_group(second ? m2 : (g.mask & ~m2));
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
    // A range may cover several queue chunks (a group that grew many chunks
    // of a small class); each queue chunk's segment is written and counted on
    // its own.
    for (uint32_t j0 = 0, j1; j0 < E; j0 = j1) {
      const uint32_t room = kQcSpots - ((b + j0) % kQcSpots);
      j1 = E - j0 < room ? E : j0 + room;
      uint32_t qc = kEmpty;
      if (g.is_leader()) qc = qchunk(h, q, b + j0);
      qc = bcast(g, qc);
      if (qc == kEmpty) continue;
      const uint32_t r2 = (j1 - j0 + n - 1u) / n;
      for (uint32_t i = 0; i < r2; ++i) {
        uint32_t j = j0 + static_cast<uint32_t>(g.rank) + i * n;
        int src = j < j1 ? lane_of_rank(g.mask, static_cast<int>(j / entries_per_chunk)) : g.leader;
        uint32_t cj = __shfl_sync(g.mask, chunk, src);
        if (j < j1) {
          uint32_t* s = queue_slots(h, qc) + ((b + j) % kQcSpots);
          if (wait_slot_empty(h, s)) st_relaxed(s, value(j, cj));
        }
      }
      __syncwarp(g.mask);
      __threadfence();
      if (g.is_leader()) count_enqueued(h, q, qc, b + j0, j1 - j0, PageQueue);
    }
  }

  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    const Group sg = half_of(g, pos, bcast(g, pos));
    if (pos % kQcSpots == 0u) preallocate(h, q, pos);
    uint32_t qc = kEmpty;
    if (sg.is_leader()) qc = qchunk(h, q, pos);
    qc = bcast(sg, qc);
    if (qc != kEmpty) {
      uint32_t* s = queue_slots(h, qc) + (pos % kQcSpots);
      if (wait_slot_empty(h, s)) st_relaxed(s, v);
    }
    __syncwarp(sg.mask);
    __threadfence();
    if (sg.is_leader() && qc != kEmpty) count_enqueued(h, q, qc, pos, static_cast<uint32_t>(sg.size), true);
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    const Group sg = half_of(g, pos, bcast(g, pos));
    uint32_t qc = kEmpty;
    if (sg.is_leader()) qc = qchunk(h, q, pos);
    qc = bcast(sg, qc);
    uint32_t v = kEmpty;
    if (qc != kEmpty) v = take_slot(h, queue_slots(h, qc) + (pos % kQcSpots));
    __syncwarp(sg.mask);
    if (sg.is_leader() && qc != kEmpty) {
      uint32_t sub = static_cast<uint32_t>(sg.size) << 16;
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
    if (qc >= kInstalling) return kEmpty;
    if (ld_relaxed(&h->meta[qc].vstart) / kQcSpots != pos / kQcSpots) return kTomb;
    return ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
  }
  __device__ static void remove(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t qc = ld_acquire(q->ring + vid(pos));
    if (qc >= kInstalling) return;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    atomicSub(&h->meta[qc].qcount, 1u << 16);
  }
  // Front moves over removed entries; passing the last entry of a queue chunk
  // returns that chunk to the pool (ChunkQueueVA_impl.cuh:144-156).  Each lane
  // keeps the queue chunk of its own positions and looks the next one up when
  // it crosses a 2048-entry boundary; a missing or reused queue chunk stops
  // the scan.
  __device__ static void advance_front(HeapCore* h, ClassState* q, const Group& g) {
    uint32_t f = 0, back = 0;
    if (g.is_leader()) {
      f = ld_relaxed(&q->front.v);
      back = ld_relaxed(&q->back.v);
    }
    f = bcast(g, f);
    back = bcast(g, back);
    if (static_cast<int32_t>(back - f) <= 0) return;
    const uint32_t n = static_cast<uint32_t>(g.size);
    uint32_t a = f & ~3u, stop = 0, range = kEmpty, qc = kEmpty;
    bool found = false;
    for (uint32_t r = 0, rounds = front_rounds(n); r < rounds && !found; ++r, a += 4u * n) {
      const uint32_t p = a + 4u * static_cast<uint32_t>(g.rank);
      uint4 e = make_uint4(0, 0, 0, 0);
      if (static_cast<int32_t>(p - back) < 0) {
        if (p / kQcSpots != range) {
          range = p / kQcSpots;
          qc = ld_acquire(q->ring + vid(p));
          if (qc >= kInstalling || ld_relaxed(&h->meta[qc].vstart) / kQcSpots != range) qc = kEmpty;
        }
        if (qc != kEmpty) e = ld_relaxed_v4(queue_slots(h, qc) + (p % kQcSpots));
      }
      found = first_live4(g, p, e, f, back, &stop);
      if (!found && static_cast<int32_t>(a + 4u * n - back) >= 0) {
        stop = back;
        found = true;
      }
    }
    if (!found) stop = a;
    if (static_cast<int32_t>(stop - f) <= 0) return;
    uint32_t cur = 0;
    if (g.is_leader()) cur = claim_front(q, f, stop);
    cur = bcast(g, cur);
    // every queue chunk whose last entry lies in [cur, stop) is now behind the front
    for (uint32_t end = cur - cur % kQcSpots + kQcSpots; static_cast<int32_t>(stop - end) >= 0; end += kQcSpots) {
      uint32_t c = kEmpty;
      if (g.is_leader()) c = atomicExch(q->ring + vid(end - 1u), kEmpty);
      c = bcast(g, c);
      if (c >= kInstalling) continue;
      uint32_t* slots = queue_slots(h, c);
      const uint4 empty = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
      for (uint32_t i = 4u * static_cast<uint32_t>(g.rank); i < kQcSpots; i += 4u * n) st_v4(slots + i, empty);
      __syncwarp(g.mask);
      __threadfence();
      if (g.is_leader()) reuse_put(h, &h->reuse[0], c);
    }
  }
};

// ===================================================== virtualized linked
struct VlStore {
  static constexpr int kKind = 2;
  static constexpr uint32_t kBehind = 0xFFFFFFFDu;

  // Direct-mapped index of recently linked queue chunks (virtual chunk id mod
  // kSkipSlots).  An entry is only a hint, valid when the chunk's vstart
  // matches; it turns the pointer chase of a burst into one lookup.
  __device__ static void remember(HeapCore* h, ClassState* q, uint32_t c, uint32_t vstart) {
    st_relaxed(q->skip + ((vstart / kQcSpots) & (kSkipSlots - 1u)), c);
  }
  __device__ static uint32_t recall(HeapCore* h, ClassState* q, uint32_t pos) {
    const uint32_t c = ld_relaxed(q->skip + ((pos / kQcSpots) & (kSkipSlots - 1u)));
    if (c < h->max_chunks && ld_relaxed(&h->meta[c].vstart) / kQcSpots == pos / kQcSpots) return c;
    return kEmpty;
  }

  // Walk from `from` to the queue chunk holding pos (QueueChunk_impl.cuh:403-426).
  // Returns kBehind when pos precedes `from`, kEmpty on timeout.
  __device__ static uint32_t locate(HeapCore* h, uint32_t from, uint32_t pos) {
    uint32_t cur = from, it = 0;
    for (uint32_t hops = 0; hops < (1u << 20); ++hops) {
      uint32_t vs = ld_relaxed(&h->meta[cur].vstart) / kQcSpots;
      uint32_t want = pos / kQcSpots;
      if (vs == want) return cur;
      if (static_cast<int32_t>(want - vs) < 0) return kBehind;
      uint32_t nx = next_of(h, cur, it);
      if (nx == kEmpty) return kEmpty;
      cur = nx;
    }
    note_timeout(h);
    return kEmpty;
  }

  // locate() for a position the caller holds (its queue chunk cannot drain
  // meanwhile), trying the index first.
  __device__ static uint32_t locate_live(HeapCore* h, ClassState* q, uint32_t from, uint32_t pos) {
    const uint32_t c = recall(h, q, pos);
    return c != kEmpty ? c : locate(h, from, pos);
  }

  // The queue chunk after c, waiting for its link (and installing one when
  // the pre-allocation does not show up).  Only called for positions that a
  // producer has already reserved, so the link must come.
  __device__ static uint32_t next_of(HeapCore* h, uint32_t c, uint32_t& it) {
    uint32_t* link = &h->meta[c].next;
    uint32_t nx;
    while ((nx = ld_acquire(link)) == kEmpty || nx == kInstalling) {
      if (it >= kSpinLimit) { note_timeout(h); return kEmpty; }
      if (nx == kEmpty && it >= kInstallAfter && (it & 63u) == 0u) {
        uint32_t vs = ld_relaxed(&h->meta[c].vstart);
        install_queue_chunk(h, link, 0u, vs - vs % kQcSpots + kQcSpots);   // queue chunks always come from the base pool
      }
      backoff(it);
    }
    return nx;
  }
  __device__ static uint32_t next_of(HeapCore* h, uint32_t c) {
    uint32_t it = 0;
    return next_of(h, c, it);
  }

  // QueueChunk_impl.cuh:440-463 setBackPointer.  Called when cur is full, so
  // its link exists or is about to (its first producer pre-allocates it).
  __device__ static void set_back(HeapCore* h, ClassState* q, uint32_t cur) {
    for (uint32_t i = 0; i < (1u << 16); ++i) {
      uint32_t nx = next_of(h, cur);
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
      uint32_t nx = next_of(h, cur);
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
      if (nx >= kInstalling) break;
      uint32_t seen = atomicCAS(&q->old_ptr, old, nx);
      if (seen == old) {
        --freed;
        if (q->clean_on_recycle) clean_queue_chunk(h, old);
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

  // A producer at the start of a queue chunk links the next one
  // (QueueChunk_impl.cuh:144-158).  A link needs its predecessor, so linking
  // is a chain; when producers already hold positions several queue chunks
  // ahead (a burst), the chain is built up to 8 chunks at a time and offered
  // in one CAS.  A lone producer is never further than one chunk ahead, so it
  // links exactly one chunk, as the reference does.
  __device__ static void preallocate(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos) {
    uint32_t* link = &h->meta[c].next;
    if (ld_relaxed(link) != kEmpty) return;
    const uint32_t back = ld_relaxed(&q->back.v);
    uint32_t ahead = static_cast<int32_t>(back - pos) > static_cast<int32_t>(2u * kQcSpots)
                         ? (back - pos) / kQcSpots - 1u : 1u;
    if (ahead > 8u) ahead = 8u;
    const uint32_t first = new_queue_chunk(h, q->inst, pos + kQcSpots);
    if (first == kEmpty) return;
    uint32_t last = first;
    for (uint32_t i = 1; i < ahead; ++i) {
      uint32_t nq = new_queue_chunk(h, q->inst, pos + (i + 1u) * kQcSpots);
      if (nq == kEmpty) break;
      st_relaxed(&h->meta[last].next, nq);
      last = nq;
    }
    __threadfence();
    if (atomicCAS(link, kEmpty, first) == kEmpty) {
      for (uint32_t cc = first, i = 0; i < 8u; ++i) {
        remember(h, q, cc, pos + (i + 1u) * kQcSpots);
        if (cc == last) break;
        cc = ld_relaxed(&h->meta[cc].next);
      }
    } else {
      for (uint32_t cc = first, i = 0; i < 8u; ++i) {
        uint32_t nx = ld_relaxed(&h->meta[cc].next);
        reuse_put(h, &h->reuse[0], cc);
        if (cc == last) break;
        cc = nx;
      }
    }
  }

  __device__ static Group half_of(const Group& g, uint32_t pos, uint32_t first) {
    const bool second = pos / kQcSpots != first / kQcSpots;
    const uint32_t m2 = __ballot_sync(g.mask, second);
    return make_group(second ? m2 : (g.mask & ~m2));
  }

  template <bool PageQueue, typename Value>
  __device__ static void publish_range(HeapCore* h, ClassState* q, const Group& g, uint32_t b, uint32_t E,
                                       uint32_t chunk, uint32_t entries_per_chunk, Value&& value) {
    const uint32_t n = static_cast<uint32_t>(g.size);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate_live(h, q, ld_acquire(&q->back_ptr), b);
    c1 = bcast(g, c1);
    if (c1 == kEmpty || c1 == kBehind) {
      if (g.is_leader()) set_status(h, kErrCorrupt);
      return;
    }
    if (b % kQcSpots == 0u && g.is_leader()) preallocate(h, q, c1, b);
    // A range may cover several queue chunks (a group that grew many chunks
    // of a small class): walk the chain one segment per queue chunk.
    uint32_t qc = c1;
    for (uint32_t j0 = 0, j1; j0 < E; j0 = j1) {
      const uint32_t room = kQcSpots - ((b + j0) % kQcSpots);
      j1 = E - j0 < room ? E : j0 + room;
      if (j0) {
        if (g.is_leader()) {
          qc = next_of(h, qc);
          if (qc != kEmpty) preallocate(h, q, qc, b + j0);   // b + j0 starts a queue chunk
        }
        qc = bcast(g, qc);
        if (qc == kEmpty) break;
      }
      const uint32_t r2 = (j1 - j0 + n - 1u) / n;
      for (uint32_t i = 0; i < r2; ++i) {
        uint32_t j = j0 + static_cast<uint32_t>(g.rank) + i * n;
        int src = j < j1 ? lane_of_rank(g.mask, static_cast<int>(j / entries_per_chunk)) : g.leader;
        uint32_t cj = __shfl_sync(g.mask, chunk, src);
        if (j < j1) st_relaxed(queue_slots(h, qc) + ((b + j) % kQcSpots), value(j, cj));   // enqueueLinked
      }
      __syncwarp(g.mask);
      __threadfence();
      if (g.is_leader()) count_enqueued(h, q, qc, j1 - j0);
    }
  }

  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    const uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate_live(h, q, ld_acquire(&q->back_ptr), first);
    c1 = bcast(g, c1);
    const Group sg = half_of(g, pos, first);
    if (c1 == kEmpty || c1 == kBehind) {
      if (g.is_leader()) set_status(h, kErrCorrupt);
      return;
    }
    uint32_t qc = c1;
    if (pos / kQcSpots != first / kQcSpots) {
      if (sg.is_leader()) qc = next_of(h, c1);
      qc = bcast(sg, qc);
    }
    if (qc != kEmpty) {
      if (pos % kQcSpots == 0u) preallocate(h, q, qc, pos);
      st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), v);
    }
    __syncwarp(sg.mask);
    __threadfence();
    if (sg.is_leader() && qc != kEmpty) count_enqueued(h, q, qc, static_cast<uint32_t>(sg.size));
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    const uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate_live(h, q, ld_acquire(&q->front_ptr), first);
    c1 = bcast(g, c1);
    const Group sg = half_of(g, pos, first);
    if (c1 == kEmpty || c1 == kBehind) {
      if (g.is_leader()) set_status(h, kErrCorrupt);
      return kEmpty;
    }
    uint32_t qc = c1;
    if (pos / kQcSpots != first / kQcSpots) {
      if (sg.is_leader()) qc = next_of(h, c1);
      qc = bcast(sg, qc);
    }
    uint32_t v = kEmpty;
    if (qc != kEmpty) v = take_slot(h, queue_slots(h, qc) + (pos % kQcSpots));
    __syncwarp(sg.mask);
    if (sg.is_leader() && qc != kEmpty) count_removed(h, q, qc, static_cast<uint32_t>(sg.size));
    return v;
  }

  // ---- chunk-queue side
  __device__ static bool enqueue_one(HeapCore* h, ClassState* q, uint32_t c, uint32_t* qpos) {
    uint32_t b = atomicAdd(&q->back.v, 1u);
    uint32_t qc = locate_live(h, q, ld_acquire(&q->back_ptr), b);
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
    uint32_t qc = recall(h, q, pos);
    if (qc == kEmpty) qc = locate(h, cur.chunk, pos);
    if (qc == kBehind) {
      cur.chunk = ld_acquire(&q->front_ptr);
      return kTomb;
    }
    if (qc == kEmpty) return kEmpty;
    cur.chunk = qc;
    return ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
  }
  __device__ static void remove(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t qc = locate_live(h, q, ld_acquire(&q->front_ptr), pos);
    if (qc == kEmpty || qc == kBehind) return;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    __threadfence();
    count_removed(h, q, qc, 1u);
  }
  // Front moves over removed entries.  The leader walks the chain: per round
  // the group's positions span at most two queue chunks (4 x 32 < 2048), the
  // current one and its successor.  Drained queue chunks leave the chain
  // through count_removed / set_front, not here.
  __device__ static void advance_front(HeapCore* h, ClassState* q, const Group& g) {
    uint32_t f = 0, back = 0, qc = kEmpty, from = 0;
    if (g.is_leader()) {
      f = ld_relaxed(&q->front.v);
      back = ld_relaxed(&q->back.v);
      from = f;
      if (static_cast<int32_t>(back - f) > 0) {
        const uint32_t first = ld_acquire(&q->front_ptr);
        qc = locate(h, first, f);
        if (qc == kBehind) {
          // front lags the first live queue chunk: everything before it is gone
          const uint32_t vs = ld_relaxed(&h->meta[first].vstart);
          from = vs - vs % kQcSpots;
          qc = first;
        }
      }
    }
    f = bcast(g, f);
    back = bcast(g, back);
    from = bcast(g, from);
    qc = bcast(g, qc);
    if (static_cast<int32_t>(back - f) <= 0 || qc == kEmpty) return;
    const uint32_t n = static_cast<uint32_t>(g.size);
    uint32_t a = from & ~3u, stop = 0, range = from / kQcSpots;   // range: the virtual queue chunk qc holds
    bool found = false;
    for (uint32_t r = 0, rounds = front_rounds(n); r < rounds && !found; ++r, a += 4u * n) {
      if (a / kQcSpots != range) {   // the round starts in the next queue chunk
        uint32_t nx = kEmpty;
        if (g.is_leader()) nx = ld_acquire(&h->meta[qc].next);
        nx = bcast(g, nx);
        if (nx >= kInstalling) {
          stop = a;
          found = true;
          break;
        }
        qc = nx;
        range = a / kQcSpots;
      }
      uint32_t nx = kEmpty;   // successor, for lanes past the end of qc
      if ((a + 4u * n - 1u) / kQcSpots != range) {
        if (g.is_leader()) nx = ld_acquire(&h->meta[qc].next);
        nx = bcast(g, nx);
      }
      const uint32_t p = a + 4u * static_cast<uint32_t>(g.rank);
      const uint32_t mine = p / kQcSpots == range ? qc : nx;
      uint4 e = make_uint4(0, 0, 0, 0);
      if (static_cast<int32_t>(p - back) < 0 && mine < kInstalling)
        e = ld_relaxed_v4(queue_slots(h, mine) + (p % kQcSpots));
      found = first_live4(g, p, e, from, back, &stop);
      if (!found && static_cast<int32_t>(a + 4u * n - back) >= 0) {
        stop = back;
        found = true;
      }
    }
    if (!found) stop = a;
    if (static_cast<int32_t>(stop - f) <= 0) return;
    if (g.is_leader()) claim_front(q, f, stop);
  }
};

}  // namespace ouro
