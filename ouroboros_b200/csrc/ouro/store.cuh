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
    if (it >= kSpinLimit) { note_timeout(h, kWaitSlotEmpty); return false; }
    backoff(it);
  }
  return true;
}

// Take the value of a slot once it is there and clear the slot -- bounded.
__device__ __forceinline__ uint32_t take_slot(HeapCore* h, uint32_t* s) {
  uint32_t v, it = 0;
  while ((v = ld_acquire(s)) == kEmpty) {
    if (it >= kSpinLimit) { note_timeout(h, kWaitSlotFull); return kEmpty; }
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

  template <bool PageQueue = true, uint32_t Seg = 0u>
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
  // The removal is counted per 2048-entry segment of the ring after the
  // tombstone is written, so a count never runs ahead of the tombstones.
  __device__ static uint32_t* seg_count(ClassState* q, uint32_t pos) {
    return q->seg + ((pos / 2048u) & q->seg_mask);
  }
  __device__ static bool remove(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* = nullptr) {
    st_relaxed(slot(q, pos), kTomb);
    __threadfence();
    atomicAdd(seg_count(q, pos), 1u);
    return false;
  }
  // remove() in two steps, so that a group counts its removals once per
  // counter: remove_mark writes the tombstone and returns the key of the
  // counter (the segment), remove_count (after a fence of every lane that
  // marked) adds m removals to it.
  __device__ static uint32_t remove_mark(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* = nullptr) {
    st_relaxed(slot(q, pos), kTomb);
    return pos / 2048u;
  }
  __device__ static bool remove_count(HeapCore* h, ClassState* q, uint32_t key, uint32_t m) {
    atomicAdd(q->seg + (key & q->seg_mask), m);
    return false;
  }
  __device__ static void after_drain(HeapCore*, ClassState*, const Group&) {}

  // Move the front past removed entries, freeing their slots for the next lap.
  // A segment whose 2048 entries all lie before the back and were all removed
  // (its count says 2048) is passed without reading its entries.  Passed
  // slots go back to kEmpty; a segment whose end the front passes has its
  // count lowered by 2048 for the next lap (lowered, not reset, so that a
  // count still in flight is kept).
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
      uint32_t skip = a;
      if (g.is_leader() && q->seg) {
        for (uint32_t k = 0; k < 64u; ++k) {
          const uint32_t end = (skip / 2048u + 1u) * 2048u;
          if (static_cast<int32_t>(end - back) > 0) break;
          if (ld_acquire(seg_count(q, skip)) != 2048u) break;
          skip = end;
        }
      }
      a = bcast(g, skip);
      if (static_cast<int32_t>(a - back) >= 0) {
        stop = back;
        found = true;
        break;
      }
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
    if (!q->seg) {
      for (uint32_t p = cur + static_cast<uint32_t>(g.rank); p != stop && static_cast<int32_t>(p - stop) < 0; p += n)
        st_relaxed(slot(q, p), kEmpty);
      return;
    }
    // [cur, stop): the partial segments at either end slot by slot, whole
    // segments one per lane with 16-byte stores
    const uint32_t s0 = (cur + 2047u) / 2048u * 2048u, s1 = stop / 2048u * 2048u;
    if (static_cast<int32_t>(s1 - s0) <= 0) {
      for (uint32_t p = cur + static_cast<uint32_t>(g.rank); static_cast<int32_t>(p - stop) < 0; p += n)
        st_relaxed(slot(q, p), kEmpty);
    } else {
      for (uint32_t p = cur + static_cast<uint32_t>(g.rank); static_cast<int32_t>(p - s0) < 0; p += n)
        st_relaxed(slot(q, p), kEmpty);
      for (uint32_t p = s1 + static_cast<uint32_t>(g.rank); static_cast<int32_t>(p - stop) < 0; p += n)
        st_relaxed(slot(q, p), kEmpty);
      const uint4 empty = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
      for (uint32_t b0 = s0 + static_cast<uint32_t>(g.rank) * 2048u; static_cast<int32_t>(s1 - b0) > 0; b0 += n * 2048u)
        for (uint32_t i = 0; i < 2048u; i += 4u) st_v4(slot(q, b0 + i), empty);
    }
    // segments whose end the front passed: their count starts the next lap
    for (uint32_t end = (cur / 2048u + 1u) * 2048u + static_cast<uint32_t>(g.rank) * 2048u;
         static_cast<int32_t>(stop - end) >= 0; end += n * 2048u)
      atomicSub(seg_count(q, end - 1u), 2048u);
  }
};

// ==================================================== virtualized array
struct VaStore {
  static constexpr int kKind = 1;

  __device__ static uint32_t vid(const ClassState* q, uint32_t pos) { return (pos / kQcSpots) & q->ring_mask; }

  // The index entry of pos's range (spins while its pre-allocation is in
  // flight), not yet checked against the queue chunk's range.
  __device__ static uint32_t qchunk_entry(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t* e = q->ring + vid(q, pos);
    uint32_t c, it = 0;
    while ((c = ld_acquire(e)) == kEmpty || c == kInstalling) {
      if (it >= kSpinLimit) { note_timeout(h, kWaitIndexEntry); return kEmpty; }
      if (c == kEmpty && it >= kInstallAfter && (it & 63u) == 0u)
        install_queue_chunk(h, e, q->inst, pos - pos % kQcSpots, queue_tag(q));
      backoff(it);
    }
    return c;
  }
  // The queue chunk holding pos, checked.
  __device__ static uint32_t qchunk(HeapCore* h, ClassState* q, uint32_t pos) {
    const uint32_t c = qchunk_entry(h, q, pos);
    if (c == kEmpty) return kEmpty;
    if (ld_relaxed(&h->meta[c].vstart) / kQcSpots != pos / kQcSpots) {
      set_status(h, kErrCorrupt);
      return kEmpty;
    }
    return c;
  }
  // The half group sg holds positions of one range; its leader found the
  // entry qc.  The check of qc's range and every lane's first look at its
  // slot go out together; false (and the corruption flag) on a mismatch.
  __device__ static bool range_ok(HeapCore* h, const Group& sg, uint32_t qc, uint32_t pos, uint32_t* s,
                                  uint32_t* first, bool acquire) {
    uint32_t vs = 0;
    if (sg.is_leader()) vs = ld_relaxed(&h->meta[qc].vstart);
    *first = acquire ? ld_acquire(s) : ld_relaxed(s);
    const bool ok = bcast(sg, vs / kQcSpots == pos / kQcSpots ? 1u : 0u) != 0u;
    if (!ok && sg.is_leader()) set_status(h, kErrCorrupt);
    return ok;
  }

  // The producer of a position at the start of a queue chunk allocates the
  // next queue chunk (PageQueueVA_impl.cuh:45-56, :202-212).
  __device__ static void preallocate(HeapCore* h, ClassState* q, uint32_t pos) {
    offer_queue_chunk(h, q->ring + vid(q, pos + kQcSpots), new_queue_chunk(h, q->inst, pos + kQcSpots, queue_tag(q)));
  }

  // Drained queue chunk back to the chunk pool (PageQueueVA_impl.cuh:159-166).
  __device__ static void recycle(HeapCore* h, ClassState* q, uint32_t pos) {
    uint32_t c = atomicExch(q->ring + vid(q, pos), kEmpty);
    if (c < kInstalling) reuse_put(h, &h->reuse[0], c);
  }

  // Count update of a range: m entries enqueued into the chunk of pos (chunk
  // queues: present << 16 | enqueued, which advance_front reads).  A page
  // queue chunk is counted by its consumers alone -- every one of its 2048
  // entries is taken exactly once, and only after it was written -- so its
  // producers add nothing: the queue chunk's count line is not one more line
  // that every group of a free burst passes through.
  template <bool PageQueue>
  __device__ static void count_enqueued(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos, uint32_t m) {
    if constexpr (!PageQueue) atomicAdd(&h->meta[c].qcount, (m << 16) + m);
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
      if constexpr (!PageQueue) {
        __syncwarp(g.mask);
        __threadfence();
        if (g.is_leader()) count_enqueued<PageQueue>(h, q, qc, b + j0, j1 - j0);
      }
    }
  }

  // PageQueue false: a chunk queue, whose queue chunks return to the pool
  // from the front (advance_front), not when their entries are consumed.
  template <bool PageQueue = true, uint32_t Seg = 0u>
  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    const Group sg = half_of(g, pos, bcast(g, pos));
    if (pos % kQcSpots == 0u) preallocate(h, q, pos);
    uint32_t qc = kEmpty;
    if (sg.is_leader()) qc = qchunk_entry(h, q, pos);
    qc = bcast(sg, qc);
    if (qc != kEmpty) {
      uint32_t* s = queue_slots(h, qc) + (pos % kQcSpots);
      uint32_t first = 0;
      if (!range_ok(h, sg, qc, pos, s, &first, false)) qc = kEmpty;
      else if (first == kEmpty || wait_slot_empty(h, s)) st_relaxed(s, v);
    }
    if constexpr (!PageQueue) {
      __syncwarp(sg.mask);
      __threadfence();
      if (sg.is_leader() && qc != kEmpty) count_enqueued<PageQueue>(h, q, qc, pos, static_cast<uint32_t>(sg.size));
    }
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    const Group sg = half_of(g, pos, bcast(g, pos));
    uint32_t qc = kEmpty;
    if (sg.is_leader()) qc = qchunk_entry(h, q, pos);
    qc = bcast(sg, qc);
    uint32_t v = kEmpty;
    if (qc != kEmpty) {
      uint32_t* s = queue_slots(h, qc) + (pos % kQcSpots);
      uint32_t first = kEmpty;
      if (!range_ok(h, sg, qc, pos, s, &first, true)) {
        qc = kEmpty;
      } else if (first != kEmpty) {
        st_relaxed(s, kEmpty);   // take_slot's first poll found it
        v = first;
      } else {
        v = take_slot(h, s);
      }
    }
    __syncwarp(sg.mask);
    if (sg.is_leader() && qc != kEmpty) {
      // entries taken, in the upper half; the taker of the last one recycles
      const uint32_t add = static_cast<uint32_t>(sg.size) << 16;
      const uint32_t old = atomicAdd(&h->meta[qc].qcount, add);
      if ((old + add) >> 16 == kQcSpots) recycle(h, q, pos);
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
  // the queue chunk of the last position peeked at
  struct Cursor { uint32_t chunk; };
  __device__ static Cursor cursor(ClassState*) { return Cursor{kEmpty}; }
  __device__ static uint32_t peek(HeapCore* h, ClassState* q, uint32_t pos, Cursor& cur) {
    uint32_t qc = ld_acquire(q->ring + vid(q, pos));
    cur.chunk = kEmpty;
    if (qc >= kInstalling) return kEmpty;
    // the queue chunk's range and the entry are read together; an entry of a
    // queue chunk that holds another range is discarded
    const uint32_t vs = ld_relaxed(&h->meta[qc].vstart);
    const uint32_t v = ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
    if (vs / kQcSpots != pos / kQcSpots) return kTomb;
    cur.chunk = qc;
    return v;
  }
  // at: the cursor of the peek that found pos's entry, which the caller is
  // removing; its queue chunk cannot drain or be reused before this removal.
  __device__ static bool remove(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* at = nullptr) {
    uint32_t qc = at ? at->chunk : kEmpty;
    if (qc == kEmpty) qc = ld_acquire(q->ring + vid(q, pos));
    if (qc >= kInstalling) return false;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    atomicSub(&h->meta[qc].qcount, 1u << 16);
    return false;   // queue chunks return to the pool from the front
  }
  // remove() in two steps (see FlatStore): the key is the queue chunk.
  __device__ static uint32_t remove_mark(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* at = nullptr) {
    uint32_t qc = at ? at->chunk : kEmpty;
    if (qc == kEmpty) qc = ld_acquire(q->ring + vid(q, pos));
    if (qc >= kInstalling) return kEmpty;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    return qc;
  }
  __device__ static bool remove_count(HeapCore* h, ClassState* q, uint32_t key, uint32_t m) {
    atomicSub(&h->meta[key].qcount, m << 16);
    return false;
  }
  __device__ static void after_drain(HeapCore*, ClassState*, const Group&) {}
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
      // A queue chunk whose 2048 entries were all written and all removed
      // (qcount: 0 present, 2048 enqueued) is passed whole, without reading
      // its entries: after a burst the front may trail the live entries by
      // hundreds of such chunks.
      uint32_t skip = a;
      if (g.is_leader()) {
        for (uint32_t k = 0; k < 64u; ++k) {
          const uint32_t rg = skip / kQcSpots, end = (rg + 1u) * kQcSpots;
          if (static_cast<int32_t>(end - back) > 0) break;
          const uint32_t c = ld_acquire(q->ring + vid(q, skip));
          if (c >= kInstalling || ld_relaxed(&h->meta[c].vstart) / kQcSpots != rg) break;
          if (ld_acquire(&h->meta[c].qcount) != kQcSpots) break;
          skip = end;
        }
      }
      a = bcast(g, skip);
      if (static_cast<int32_t>(a - back) >= 0) {
        stop = back;
        found = true;
        break;
      }
      const uint32_t p = a + 4u * static_cast<uint32_t>(g.rank);
      uint4 e = make_uint4(0, 0, 0, 0);
      if (static_cast<int32_t>(p - back) < 0) {
        if (p / kQcSpots != range) {
          range = p / kQcSpots;
          qc = ld_acquire(q->ring + vid(q, p));
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
    // every queue chunk whose last entry lies in [cur, stop) is now behind the
    // front: one per lane takes it out of the index, cleans its entries and
    // returns it to the pool
    const uint4 empty = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
    for (uint32_t end0 = cur - cur % kQcSpots + kQcSpots; static_cast<int32_t>(stop - end0) >= 0;
         end0 += n * kQcSpots) {
      const uint32_t end = end0 + static_cast<uint32_t>(g.rank) * kQcSpots;
      if (static_cast<int32_t>(stop - end) < 0) continue;
      const uint32_t c = atomicExch(q->ring + vid(q, end - 1u), kEmpty);
      if (c >= kInstalling) continue;
      uint32_t* slots = queue_slots(h, c);
      for (uint32_t i = 0; i < kQcSpots; i += 4u) st_v4(slots + i, empty);
      __threadfence();
      reuse_put(h, &h->reuse[0], c);
    }
  }
};

// ===================================================== virtualized linked
struct VlStore {
  static constexpr int kKind = 2;
  static constexpr uint32_t kBehind = 0xFFFFFFFDu;
  static constexpr uint32_t kStale = 0xFFFFFFFBu;   // a walk met a recycled chunk
  static constexpr uint32_t kRecallPolls = 48u;            // index polls before walking the chain

  // Direct-mapped index of recently linked queue chunks (virtual chunk id mod
  // kSkipSlots).  An entry is only a hint, valid while the chunk carries the
  // class's queue tag and the range; it turns the pointer chase of a burst
  // into one lookup.
  __device__ static void remember(HeapCore* h, ClassState* q, uint32_t c, uint32_t vstart) {
    st_relaxed(q->skip + ((vstart / kQcSpots) & (kSkipSlots - 1u)), c);
  }
  __device__ static uint32_t recall_range(HeapCore* h, ClassState* q, uint32_t range) {
    const uint32_t c = ld_relaxed(q->skip + (range & (kSkipSlots - 1u)));
    if (c >= h->max_chunks) return kEmpty;
    // tag and range are read together (two loads in flight, not one after the other)
    const uint32_t tag = ld_relaxed(&h->meta[c].size);
    const uint32_t vs = ld_relaxed(&h->meta[c].vstart);
    return (tag == queue_tag(q) && vs / kQcSpots == range) ? c : kEmpty;
  }
  __device__ static uint32_t recall(HeapCore* h, ClassState* q, uint32_t pos) {
    return recall_range(h, q, pos / kQcSpots);
  }

  // Walk from `from` to the queue chunk holding pos (QueueChunk_impl.cuh:403-426).
  // `from` is a front_ptr / back_ptr value read a moment ago; the chunk may
  // have been recycled since (front_ptr can pass many drained chunks at once),
  // so every hop is checked: the chunk must carry the class's tag and the next
  // range.  A failed check returns kStale (read the pointer again).  Returns
  // kBehind when pos precedes `from`, kEmpty on timeout.
  __device__ static uint32_t locate(HeapCore* h, ClassState* q, uint32_t from, uint32_t pos) {
    const uint32_t tag = queue_tag(q);
    const uint32_t want = pos / kQcSpots;
    if (from >= h->max_chunks || ld_relaxed(&h->meta[from].size) != tag) return kStale;
    uint32_t cur = from, it = 0;
    uint32_t vs = ld_relaxed(&h->meta[cur].vstart) / kQcSpots;
    for (uint32_t hops = 0; hops < (1u << 20); ++hops) {
      if (vs == want) return cur;
      if (static_cast<int32_t>(want - vs) < 0) return kBehind;
      const uint32_t nx = next_of(h, cur, it);
      if (nx == kEmpty) return kEmpty;
      if (nx >= h->max_chunks || ld_relaxed(&h->meta[nx].size) != tag ||
          ld_relaxed(&h->meta[nx].vstart) / kQcSpots != vs + 1u)
        return kStale;
      cur = nx;
      ++vs;
    }
    note_timeout(h, kWaitLocateHops);
    return kEmpty;
  }

  // locate() for a position the caller holds (its queue chunk cannot drain
  // meanwhile), starting from *start (front_ptr or back_ptr).  The index is
  // tried first and polled for a while: in a burst the chunk is usually being
  // linked at that moment, and its linker enters it in the index as soon as it
  // is attached, which beats walking the chain hop by hop behind it.
  __device__ static uint32_t locate_live(HeapCore* h, ClassState* q, const uint32_t* start, uint32_t pos) {
    for (uint32_t it = 0; it < kRecallPolls;) {
      const uint32_t c = recall(h, q, pos);
      if (c != kEmpty) return c;
      backoff(it);
    }
    for (uint32_t attempt = 0; attempt < 64u; ++attempt) {
      const uint32_t c = locate(h, q, ld_acquire(start), pos);
      if (c != kStale) return c;
      const uint32_t r = recall(h, q, pos);
      if (r != kEmpty) return r;
    }
    note_timeout(h, kWaitLocateStale);
    return kEmpty;
  }

  // The queue chunk after c, waiting for its link (and installing one when
  // the pre-allocation does not show up).  Only called for positions that a
  // producer has already reserved, so the link must come.
  __device__ static uint32_t next_of(HeapCore* h, uint32_t c, uint32_t& it) {
    uint32_t* link = &h->meta[c].next;
    uint32_t nx;
    while ((nx = ld_acquire(link)) == kEmpty || nx == kInstalling) {
      if (it >= kSpinLimit) { note_timeout(h, kWaitLink); return kEmpty; }
      if (nx == kEmpty && it >= kInstallAfter && (it & 63u) == 0u) {
        uint32_t vs = ld_relaxed(&h->meta[c].vstart);
        install_queue_chunk(h, link, 0u, vs - vs % kQcSpots + kQcSpots,   // queue chunks always come from the base pool
                            ld_relaxed(&h->meta[c].size));
      }
      backoff(it);
    }
    return nx;
  }
  __device__ static uint32_t next_of(HeapCore* h, uint32_t c) {
    uint32_t it = 0;
    return next_of(h, c, it);
  }

  // QueueChunk_impl.cuh:440-463 setBackPointer.  back_ptr, where locate()
  // starts for producers, moves over full queue chunks whose successor is
  // linked.  Every walk starts from the current back_ptr and publishes with
  // one CAS, so a chunk that fills while another group walks is passed by one
  // of the two.  Chunks fill out of order in a burst, so the filler of the
  // oldest one may have hundreds to pass: the group looks at one queue chunk
  // per lane and round, lane i at the range i after the walk's position,
  // found through the index and checked against its predecessor's link (a
  // chunk the index does not hold ends the round; the next round starts from
  // the real link, so a round passes at least one chunk).  Collective over g.
  __device__ static void set_back(HeapCore* h, ClassState* q, const Group& g) {
    const uint32_t n = static_cast<uint32_t>(g.size), r = static_cast<uint32_t>(g.rank);
    const uint32_t tag = queue_tag(q);
    uint32_t bp = 0;
    if (g.is_leader()) bp = ld_acquire(&q->back_ptr);
    bp = bcast(g, bp);
    for (uint32_t round = 0; round < 64u; ++round) {
      uint32_t cur = bp;
      for (uint32_t step = 0; step < (1u << 16); ++step) {
        uint32_t r0 = 0;
        if (g.is_leader()) r0 = ld_relaxed(&h->meta[cur].vstart) / kQcSpots;
        r0 = bcast(g, r0);
        // lane r: the queue chunk of range r0 + r (lane 0: cur itself)
        uint32_t c = r == 0u ? cur : recall_range(h, q, r0 + r);
        bool pass = false;
        uint32_t nx = kEmpty;
        if (c < h->max_chunks && ld_relaxed(&h->meta[c].size) == tag) {
          pass = (ld_acquire(&h->meta[c].qcount) & 0xFFFFu) == kQcSpots;
          nx = ld_acquire(&h->meta[c].next);
          pass = pass && nx < kInstalling;
        }
        // lane r continues lane r - 1's chain only if that chunk links to it
        const uint32_t prev_next = __shfl_sync(g.mask, nx, lane_of_rank(g.mask, r > 0u ? static_cast<int>(r) - 1 : 0));
        const bool ok = pass && (r == 0u || prev_next == c);
        const uint32_t stop = __ballot_sync(g.mask, !ok);
        const uint32_t k = stop ? first_rank(g, stop) : n;   // lanes 0 .. k-1 are passed
        if (k == 0u) break;
        cur = __shfl_sync(g.mask, nx, lane_of_rank(g.mask, static_cast<int>(k) - 1));
      }
      if (cur == bp) return;
      uint32_t seen = 0;
      if (g.is_leader()) seen = atomicCAS(&q->back_ptr, bp, cur);
      seen = bcast(g, seen);
      if (seen == bp) return;
      bp = seen;   // moved by someone else: walk on from there
    }
  }

  // Rank of the lowest lane of m within the group.
  __device__ static uint32_t first_rank(const Group& g, uint32_t m) {
    return static_cast<uint32_t>(__popc(g.mask & ((1u << (__ffs(m) - 1)) - 1u)));
  }

  // From chunk fp on, the queue chunks that are drained (all 2048 entries
  // taken) and linked to a successor.  Index i = u x n + r (u = 0, 1: two
  // chunks per lane and round) looks up the chunk of range (fp's range + i)
  // in the index and checks that it is the successor of index i-1's chunk, so
  // a round covers up to two chunks per lane; an index miss ends the round
  // early.  Returns how many chunks can be passed and moves *fp to the first
  // one that cannot.  Collective over g.
  __device__ static uint32_t walk_drained(HeapCore* h, ClassState* q, const Group& g, uint32_t* fp_io) {
    const uint32_t n = static_cast<uint32_t>(g.size), r = static_cast<uint32_t>(g.rank);
    const int prev_lane = lane_of_rank(g.mask, r == 0u ? static_cast<int>(n) - 1 : static_cast<int>(r) - 1);
    uint32_t fp = *fp_io, passed = 0;
    uint32_t range = ld_relaxed(&h->meta[fp].vstart) / kQcSpots;
    for (uint32_t round = 0; round < (1u << 16); ++round) {
      uint32_t c[2], cnt[2] = {0u, 0u}, nx[2] = {kEmpty, kEmpty};
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        c[u] = i == 0u ? fp : recall_range(h, q, range + i);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        if (c[u] != kEmpty) {
          cnt[u] = ld_acquire(&h->meta[c[u]].qcount);
          nx[u] = ld_acquire(&h->meta[c[u]].next);
        }
      }
      bool linked[2], pass[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        const uint32_t same = __shfl_sync(g.mask, nx[u], prev_lane);          // index i-1 when r > 0
        const uint32_t wrap = __shfl_sync(g.mask, nx[u > 0 ? u - 1 : 0], prev_lane);   // index i-1 when r == 0
        const uint32_t prev = r > 0u ? same : wrap;
        linked[u] = i == 0u || (c[u] != kEmpty && c[u] == prev);
        pass[u] = linked[u] && cnt[u] == kQcSpots && nx[u] < kInstalling;
      }
      const uint32_t s0 = __ballot_sync(g.mask, !pass[0]), s1 = __ballot_sync(g.mask, !pass[1]);
      const uint32_t k = s0 ? first_rank(g, s0) : (s1 ? n + first_rank(g, s1) : 2u * n);
      if (k == 0u) break;
      const int last = lane_of_rank(g.mask, static_cast<int>((k - 1u) % n));
      const uint32_t a0 = __shfl_sync(g.mask, nx[0], last), a1 = __shfl_sync(g.mask, nx[1], last);
      fp = (k - 1u) / n == 0u ? a0 : a1;
      passed += k;
      range += k;
      if (k < 2u * n) {
        // stopped at a chunk that is linked but not passable: the walk ends;
        // stopped at an index miss: the next round starts from the real link
        const int at = lane_of_rank(g.mask, static_cast<int>(k % n));
        const uint32_t l0 = __shfl_sync(g.mask, linked[0] ? 1u : 0u, at), l1 = __shfl_sync(g.mask, linked[1] ? 1u : 0u, at);
        if (k / n == 0u ? l0 : l1) break;
      }
    }
    *fp_io = fp;
    return passed;
  }

  // Return k chained queue chunks starting at c to the base pool: index
  // i = u x n + r (two per lane and round) finds its chunk as in walk_drained,
  // clears its tag and page size (and its entries for chunk queues), and all
  // of a round are published with one reservation on the reuse ring.
  // Returns the chunk after the last one.  Collective over g.
  __device__ static uint32_t recycle_run(HeapCore* h, ClassState* q, const Group& g, uint32_t c, uint32_t k) {
    const uint32_t n = static_cast<uint32_t>(g.size), r = static_cast<uint32_t>(g.rank);
    const int prev_lane = lane_of_rank(g.mask, r == 0u ? static_cast<int>(n) - 1 : static_cast<int>(r) - 1);
    ReuseQueue* rq = &h->reuse[0];
    uint32_t range = ld_relaxed(&h->meta[c].vstart) / kQcSpots;
    for (uint32_t guard = 0; k > 0u && guard < (1u << 16); ++guard) {
      const uint32_t want = k < 2u * n ? k : 2u * n;
      uint32_t mine[2] = {kEmpty, kEmpty}, nx[2] = {kEmpty, kEmpty};
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        if (i < want) mine[u] = i == 0u ? c : recall_range(h, q, range + i);
      }
#pragma unroll
      for (int u = 0; u < 2; ++u)
        if (mine[u] != kEmpty) nx[u] = ld_acquire(&h->meta[mine[u]].next);
      bool ok[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        const uint32_t same = __shfl_sync(g.mask, nx[u], prev_lane);
        const uint32_t wrap = __shfl_sync(g.mask, nx[u > 0 ? u - 1 : 0], prev_lane);
        const uint32_t prev = r > 0u ? same : wrap;
        ok[u] = i < want && (i == 0u || (mine[u] != kEmpty && mine[u] == prev)) && nx[u] < kInstalling;
      }
      const uint32_t b0 = __ballot_sync(g.mask, !ok[0]), b1 = __ballot_sync(g.mask, !ok[1]);
      const uint32_t L = b0 ? first_rank(g, b0) : (b1 ? n + first_rank(g, b1) : 2u * n);
      if (L == 0u) {   // a chunk behind front_ptr without a successor: the chain is broken
        if (g.is_leader()) set_status(h, kErrCorrupt);
        break;
      }
      const int last = lane_of_rank(g.mask, static_cast<int>((L - 1u) % n));
      const uint32_t a0 = __shfl_sync(g.mask, nx[0], last), a1 = __shfl_sync(g.mask, nx[1], last);
      const uint32_t after = (L - 1u) / n == 0u ? a0 : a1;
      bool any = false;
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        if (i < L) {
          if (q->clean_on_recycle) clean_queue_chunk(h, mine[u]);
          st_relaxed(&h->meta[mine[u]].size, 0u);
          st_relaxed(&h->meta[mine[u]].page_size, 0u);
          any = true;
        }
      }
      if (any) __threadfence();
      __syncwarp(g.mask);
      uint32_t pos = 0, take = L;
      if (g.is_leader()) {
        const int32_t fill = atomicAdd(&rq->count.v, static_cast<int32_t>(L));
        if (fill + static_cast<int32_t>(L) > static_cast<int32_t>(kReuseSize)) {
          take = fill >= static_cast<int32_t>(kReuseSize) ? 0u : kReuseSize - static_cast<uint32_t>(fill);
          atomicSub(&rq->count.v, static_cast<int32_t>(L - take));
          set_status(h, kErrQueueFull);   // those chunks stay out of circulation
        }
        if (take) pos = atomicAdd(&rq->back.v, take);
      }
      pos = bcast(g, pos);
      take = bcast(g, take);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t i = static_cast<uint32_t>(u) * n + r;
        if (i < take) {
          uint32_t* sl = rq->ring + ((pos + i) & (kReuseSize - 1u));
          if (wait_slot_empty(h, sl)) st_release(sl, mine[u]);
        }
      }
      c = after;
      range += L;
      k -= L;
    }
    return c;
  }

  // QueueChunk_impl.cuh:467-551 setFrontPointer + setOldPointer.  One group
  // at a time (try-lock on the class's ptr_lock line) moves front_ptr over
  // every drained queue chunk whose successor is linked and returns the
  // drained chunks more than kOldHold behind it to the pool -- held back so
  // that a lane that read front_ptr a little while ago can still walk forward
  // from it.  A group that finds the lock taken returns: the holder re-checks
  // the chunk at front_ptr after unlocking, so no drain is lost.  Collective
  // over g.
  __device__ static void on_empty(HeapCore* h, ClassState* q, const Group& g) {
    for (uint32_t round = 0; round < 64u; ++round) {
      uint32_t mine = 0;
      if (g.is_leader()) mine = atomicCAS(&q->ptr_lock.v, 0u, 1u) == 0u ? 1u : 0u;
      if (!bcast(g, mine)) return;
      __threadfence();
      uint32_t fp = 0, held = 0, old = 0;
      if (g.is_leader()) {
        fp = ld_relaxed(&q->front_ptr);
        held = ld_relaxed(&q->old_count);
        old = ld_relaxed(&q->old_ptr);
      }
      fp = bcast(g, fp);
      held = bcast(g, held);
      old = bcast(g, old);
      const uint32_t passed = walk_drained(h, q, g, &fp);
      if (passed) {
        if (g.is_leader()) st_release(&q->front_ptr, fp);
        held += passed;
        if (held > kOldHold) {
          old = recycle_run(h, q, g, old, held - kOldHold);
          held = kOldHold;
        }
        if (g.is_leader()) {
          st_relaxed(&q->old_ptr, old);
          st_relaxed(&q->old_count, held);
        }
      }
      __syncwarp(g.mask);
      uint32_t again = 0;
      if (g.is_leader()) {
        __threadfence();
        atomicExch(&q->ptr_lock.v, 0u);
        const uint32_t f2 = ld_acquire(&q->front_ptr);
        again = ld_acquire(&h->meta[f2].qcount) == kQcSpots && ld_acquire(&h->meta[f2].next) < kInstalling ? 1u : 0u;
      }
      if (!bcast(g, again)) return;
    }
  }

  // Count update of m enqueued entries into chunk c (QueueChunk_impl.cuh:160-182).
  // Returns kFilled when this update fills the chunk (the caller's group then
  // runs set_back) and kDrained when it completes the chunk's drain (then
  // on_empty), in that order.
  static constexpr uint32_t kDrained = 1u, kFilled = 2u;
  __device__ static uint32_t count_enqueued(HeapCore* h, ClassState* q, uint32_t c, uint32_t m) {
    uint32_t add = (m << 16) + m;
    uint32_t old = atomicAdd(&h->meta[c].qcount, add);
    return ((old & 0xFFFFu) + m == kQcSpots ? kFilled : 0u) | (old + add == kQcSpots ? kDrained : 0u);
  }
  __device__ static void after_enqueue(HeapCore* h, ClassState* q, const Group& g, uint32_t flags) {
    if (flags & kFilled) set_back(h, q, g);
    if (flags & kDrained) on_empty(h, q, g);
  }

  __device__ static bool count_removed(HeapCore* h, ClassState* q, uint32_t c, uint32_t m) {
    uint32_t sub = m << 16;
    uint32_t old = atomicSub(&h->meta[c].qcount, sub);
    return old - sub == kQcSpots;
  }

  // A producer at the start of a queue chunk links the next one
  // (QueueChunk_impl.cuh:144-158).  A link needs its predecessor, so linking
  // is a chain.  When producers already hold positions several queue chunks
  // ahead (a burst), the group links pieces of up to kPieceRounds chunks per
  // lane: one reservation of chunks, headers and links written in parallel,
  // one CAS to attach the piece, and index entries written right after, so
  // that waiting producers find their chunk in the index instead of walking.
  // Up to kPieceSegments pieces follow one another in one call, each attached
  // to the last chunk of the one before, so a burst of up to
  // kPieceSegments x kPieceRounds x 32 queue chunks (2^20 entries) is linked by
  // one group without waiting for the producers further on.  The first piece
  // is only ever attached to c, whose range the caller holds a position of: c
  // cannot drain meanwhile.  (A chunk the caller does not hold may be
  // drained, recycled and reused with an empty link, and a piece attached
  // there would duplicate ranges of the live chain.)  Each further piece goes
  // after the group's own newest chunk, whose link is still empty: front_ptr
  // cannot pass a chunk without a successor, so that chunk is not recycled
  // either.  A lone producer is never more than one chunk ahead, so it links
  // exactly one chunk, as the reference does.  c holds the range starting at
  // pos.  Collective over g.
  // Segments: pieces one call may link (the page queues' producers use
  // kPieceSegments; the chunk queues, whose bursts bring at most one entry per
  // chunk, one: it keeps the allocation kernels' code small).
  static constexpr int kPieceRounds = 4;
  static constexpr uint32_t kPieceSegments = 4u;
  template <uint32_t Segments = 1u>
  __device__ static void preallocate(HeapCore* h, ClassState* q, const Group& g, uint32_t c, uint32_t pos) {
    const uint32_t n = static_cast<uint32_t>(g.size);
    uint32_t ahead = 0;
    if (g.is_leader() && ld_relaxed(&h->meta[c].next) == kEmpty) {
      const uint32_t back = ld_relaxed(&q->back.v);
      ahead = static_cast<int32_t>(back - pos) > static_cast<int32_t>(2u * kQcSpots)
                  ? (back - pos) / kQcSpots - 1u : 1u;
      if (ahead > Segments * kPieceRounds * n) ahead = Segments * kPieceRounds * n;
    }
    ahead = bcast(g, ahead);
    if constexpr (Segments == 1u) {
      if (ahead) link_piece<false>(h, q, g, c, pos, ahead);
    } else {
      while (ahead) {
        const uint32_t part = ahead < kPieceRounds * n ? ahead : kPieceRounds * n;
        const uint32_t last = link_piece<true>(h, q, g, c, pos, part);
        if (last == kEmpty) return;   // a shorter piece, none, or someone else linked c
        ahead -= part;
        c = last;
        pos += part * kQcSpots;
      }
    }
  }

  // One piece of `part` queue chunks after c (range starting at pos).  Tail:
  // return the piece's last chunk when the whole piece was attached (kEmpty
  // otherwise); without Tail, kEmpty.
  template <bool Tail>
  __device__ static uint32_t link_piece(HeapCore* h, ClassState* q, const Group& g, uint32_t c, uint32_t pos,
                                        uint32_t part) {
    uint32_t* link = &h->meta[c].next;
    const uint32_t n = static_cast<uint32_t>(g.size), r = static_cast<uint32_t>(g.rank);
    uint32_t mine[kPieceRounds];
    const uint32_t got = alloc_chunk_rounds<kPieceRounds>(h, g, part, q->inst, true, mine);
    // the piece is the prefix of chunks up to the first one missing
    uint32_t hole = part;
#pragma unroll
    for (int j = 0; j < kPieceRounds; ++j) {
      const uint32_t i = static_cast<uint32_t>(j) * n + r;
      if (i < part && (i >= got || mine[j] == kEmpty) && i < hole) hole = i;
    }
    const uint32_t L = __reduce_min_sync(g.mask, hole);
    const int next_lane = lane_of_rank(g.mask, r + 1u < n ? static_cast<int>(r) + 1 : static_cast<int>(r));
    uint32_t tail = kEmpty;   // the piece's last chunk, on the lane that holds it
#pragma unroll
    for (int j = 0; j < kPieceRounds; ++j) {
      const uint32_t i = static_cast<uint32_t>(j) * n + r;
      const uint32_t succ_same = __shfl_sync(g.mask, mine[j], next_lane);
      const uint32_t succ_next = __shfl_sync(g.mask, mine[j + 1 < kPieceRounds ? j + 1 : j], g.leader);
      if (i < L) {
        init_queue_chunk(h, mine[j], pos + (i + 1u) * kQcSpots, queue_tag(q));
        if (i + 1u < L) st_relaxed(&h->meta[mine[j]].next, r + 1u < n ? succ_same : succ_next);
        else if constexpr (Tail) tail = mine[j];
      } else if (i < got && mine[j] != kEmpty) {
        reuse_put(h, &h->reuse[0], mine[j]);   // behind a hole: not part of the piece
      }
    }
    __threadfence();
    __syncwarp(g.mask);
    if (L == 0u) return kEmpty;
    const uint32_t piece = __shfl_sync(g.mask, mine[0], g.leader);
    uint32_t ok = 0;
    if (g.is_leader()) ok = atomicCAS(link, kEmpty, piece) == kEmpty ? 1u : 0u;
    ok = bcast(g, ok);
#pragma unroll
    for (int j = 0; j < kPieceRounds; ++j) {
      const uint32_t i = static_cast<uint32_t>(j) * n + r;
      if (i >= L) continue;
      if (ok) {
        remember(h, q, mine[j], pos + (i + 1u) * kQcSpots);
      } else {   // someone else linked it: the piece goes back, untagged
        st_relaxed(&h->meta[mine[j]].size, 0u);
        __threadfence();
        reuse_put(h, &h->reuse[0], mine[j]);
      }
    }
    if (!Tail || !ok || L < part) return kEmpty;
    return __shfl_sync(g.mask, tail, lane_of_rank(g.mask, static_cast<int>((L - 1u) % n)));
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
    if (g.is_leader()) c1 = locate_live(h, q, &q->back_ptr, b);
    c1 = bcast(g, c1);
    if (c1 == kEmpty || c1 == kBehind) {
      if (g.is_leader()) set_status(h, kErrCorrupt);
      return;
    }
    if (b % kQcSpots == 0u) preallocate<PageQueue ? kPieceSegments : 1u>(h, q, g, c1, b);
    // A range may cover several queue chunks (a group that grew many chunks
    // of a small class): walk the chain one segment per queue chunk.
    uint32_t qc = c1;
    for (uint32_t j0 = 0, j1; j0 < E; j0 = j1) {
      const uint32_t room = kQcSpots - ((b + j0) % kQcSpots);
      j1 = E - j0 < room ? E : j0 + room;
      if (j0) {
        if (g.is_leader()) qc = next_of(h, qc);
        qc = bcast(g, qc);
        if (qc == kEmpty) break;
        preallocate<PageQueue ? kPieceSegments : 1u>(h, q, g, qc, b + j0);   // b + j0 starts a queue chunk
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
      uint32_t flags = 0;
      if (g.is_leader()) flags = count_enqueued(h, q, qc, j1 - j0);
      after_enqueue(h, q, g, bcast(g, flags));
    }
  }

  // Seg: pieces one preallocate call may link (0: the queue kind's default).
  template <bool PageQueue = true, uint32_t Seg = 0u>
  __device__ static void publish_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos, uint32_t v) {
    const uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate_live(h, q, &q->back_ptr, first);
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
    if (qc == kEmpty) return;
    const uint32_t starts = __ballot_sync(sg.mask, pos % kQcSpots == 0u);
    if (starts)
      preallocate<Seg ? Seg : (PageQueue ? kPieceSegments : 1u)>(h, q, sg, qc, __shfl_sync(sg.mask, pos, __ffs(starts) - 1));
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), v);
    __syncwarp(sg.mask);
    __threadfence();
    uint32_t flags = 0;
    if (sg.is_leader()) flags = count_enqueued(h, q, qc, static_cast<uint32_t>(sg.size));
    after_enqueue(h, q, sg, bcast(sg, flags));
  }

  __device__ static uint32_t consume_lane(HeapCore* h, ClassState* q, const Group& g, uint32_t pos) {
    const uint32_t first = bcast(g, pos);
    uint32_t c1 = kEmpty;
    if (g.is_leader()) c1 = locate_live(h, q, &q->front_ptr, first);
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
    if (qc == kEmpty) return kEmpty;
    const uint32_t v = take_slot(h, queue_slots(h, qc) + (pos % kQcSpots));
    __syncwarp(sg.mask);
    uint32_t drained = 0;
    if (sg.is_leader()) drained = count_removed(h, q, qc, static_cast<uint32_t>(sg.size)) ? 1u : 0u;
    if (bcast(sg, drained)) on_empty(h, q, sg);
    return v;
  }

  // ---- chunk-queue side
  __device__ static bool enqueue_one(HeapCore* h, ClassState* q, uint32_t c, uint32_t* qpos) {
    uint32_t b = atomicAdd(&q->back.v, 1u);
    uint32_t qc = locate_live(h, q, &q->back_ptr, b);
    if (qc == kEmpty || qc == kBehind) { set_status(h, kErrCorrupt); return false; }
    const Group self = make_group(1u << lane_id());
    if (b % kQcSpots == 0u) preallocate(h, q, self, qc, b);
    st_relaxed(qpos, b);
    __threadfence();
    st_release(queue_slots(h, qc) + (b % kQcSpots), c);
    __threadfence();
    after_enqueue(h, q, self, count_enqueued(h, q, qc, 1u));
    return true;
  }
  struct Cursor { uint32_t chunk; };
  __device__ static Cursor cursor(ClassState* q) { return Cursor{ld_acquire(&q->front_ptr)}; }
  __device__ static uint32_t peek(HeapCore* h, ClassState* q, uint32_t pos, Cursor& cur) {
    uint32_t qc = recall(h, q, pos);
    if (qc == kEmpty) {
      // walk from the cursor's chunk, or from front_ptr once the cursor's chunk fell behind it
      const uint32_t fp = ld_acquire(&q->front_ptr);
      const uint32_t fr = ld_relaxed(&h->meta[fp].vstart) / kQcSpots;
      const uint32_t cr = ld_relaxed(&h->meta[cur.chunk].vstart) / kQcSpots;
      qc = locate(h, q, static_cast<int32_t>(cr - fr) < 0 ? fp : cur.chunk, pos);
      if (qc == kStale) {
        cur.chunk = fp;
        return kEmpty;
      }
    }
    if (qc == kBehind) {
      cur.chunk = ld_acquire(&q->front_ptr);
      return kTomb;
    }
    if (qc == kEmpty) return kEmpty;
    cur.chunk = qc;
    return ld_acquire(queue_slots(h, qc) + (pos % kQcSpots));
  }
  // Returns true when this removal drained the queue chunk: the caller's
  // group then runs after_drain (on_empty), so that front_ptr moves with a
  // whole group's walk rather than one lane's.
  // at: the cursor of the peek that found pos's entry (see VaStore::remove).
  __device__ static bool remove(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* at = nullptr) {
    uint32_t qc = at ? at->chunk : kEmpty;
    if (qc == kEmpty || ld_relaxed(&h->meta[qc].vstart) / kQcSpots != pos / kQcSpots)
      qc = locate_live(h, q, &q->front_ptr, pos);
    if (qc == kEmpty || qc == kBehind) return false;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    __threadfence();
    return count_removed(h, q, qc, 1u);
  }
  // remove() in two steps (see FlatStore): the key is the queue chunk;
  // remove_count returns true when the m removals drained it.
  __device__ static uint32_t remove_mark(HeapCore* h, ClassState* q, uint32_t pos, const Cursor* at = nullptr) {
    uint32_t qc = at ? at->chunk : kEmpty;
    if (qc == kEmpty || ld_relaxed(&h->meta[qc].vstart) / kQcSpots != pos / kQcSpots)
      qc = locate_live(h, q, &q->front_ptr, pos);
    if (qc == kEmpty || qc == kBehind) return kEmpty;
    st_relaxed(queue_slots(h, qc) + (pos % kQcSpots), kTomb);
    return qc;
  }
  __device__ static bool remove_count(HeapCore* h, ClassState* q, uint32_t key, uint32_t m) {
    return count_removed(h, q, key, m);
  }
  __device__ static void after_drain(HeapCore* h, ClassState* q, const Group& g) { on_empty(h, q, g); }
  // Front moves over removed entries.  The leader walks the chain: per round
  // the group's positions span at most two queue chunks (4 x 32 < 2048), the
  // current one and its successor.  Drained queue chunks leave the chain
  // through count_removed / on_empty, not here.
  __device__ static void advance_front(HeapCore* h, ClassState* q, const Group& g) {
    uint32_t f = 0, back = 0, qc = kEmpty, from = 0;
    if (g.is_leader()) {
      f = ld_relaxed(&q->front.v);
      back = ld_relaxed(&q->back.v);
      from = f;
      if (static_cast<int32_t>(back - f) > 0) {
        const uint32_t first = ld_acquire(&q->front_ptr);
        qc = locate(h, q, first, f);
        if (qc == kStale) qc = kEmpty;
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
