// queues.cuh -- page-based and chunk-based size-class queues over a storage.
//
// Page-based (PageQueue*_impl.cuh): the queue holds one entry per free page;
//   a group takes g.size consecutive positions with one atomic on `front`.
// Chunk-based (ChunkQueue*_impl.cuh): the queue holds chunks with free pages;
//   a group scans from `front`, reserves pages on a chunk with one atomic on its
//   count and claims bits of its occupancy mask cooperatively.
#pragma once

#include "semaphore.cuh"
#include "store.cuh"

namespace ouro {

__device__ __forceinline__ void* page_address(HeapCore* h, uint32_t chunk, uint32_t page, uint32_t page_shift) {
  return h->data + (static_cast<size_t>(chunk) << kChunkShift) + (static_cast<size_t>(page) << page_shift);
}

// Metadata of freshly allocated data chunks.  The count/mask of a chunk-index
// chunk are written before its page size, which is what lanes validate.
__device__ __forceinline__ void init_data_chunk(HeapCore* h, ClassState* q, uint32_t c, bool chunk_based) {
  ChunkMeta* m = h->meta + c;
  st_relaxed(&m->size, q->ppc);
  st_relaxed(&m->head, 0u);
  if (chunk_based) {
    st_relaxed(&m->count, static_cast<int32_t>(q->ppc));
    st_relaxed(&m->queue_pos, kEmpty);
    // ChunkAccess.cuh:69-89: all ppc pages free
    uint32_t n = q->ppc;
#pragma unroll
    for (uint32_t w = 0; w < 16u; ++w) {
      st_relaxed(m->mask(w), n >= 32u ? 0xFFFFFFFFu : ((1u << n) - 1u));
      n = n > 32u ? n - 32u : 0u;
    }
    __threadfence();
  }
  st_relaxed(&m->page_size, q->page_size);
  if (q->inst == 1u) {
    // the three continuation chunks of a 32 KiB chunk point at their head
    for (uint32_t k = 1; k < 4u; ++k) {
      st_relaxed(&h->meta[c + k].head, k);
      st_relaxed(&h->meta[c + k].page_size, q->page_size);
    }
  }
}

// Queue capacity guard: a class may not own more pages than its queue holds
// (the reference traps in that case, PageQueue_impl.cuh:34).  Returns the
// class's page count before the reservation, kEmpty when refused.
__device__ __forceinline__ uint32_t reserve_class_pages(HeapCore* h, ClassState* q, uint32_t pages) {
  uint32_t old = atomicAdd(&q->class_pages, pages);
  if (old + pages > q->page_cap || old + pages < old) {
    atomicSub(&q->class_pages, pages);
    set_status(h, kErrQueueFull);
    return kEmpty;
  }
  return old;
}

// Virtualized queues take their queue chunks from the same pool as data
// chunks.  A class only grows while the queue chunks it will need at its new
// size still fit: `budget` counts data chunks plus, per class, the queue
// chunks for its entries and a margin, against the usable chunks.  Without
// it the last data chunks would leave no queue chunk for the entries they
// bring, and producers would wait for a link that cannot come.  The queue of
// the class grows from e0 entries by `per` entries per chunk; returns how
// many of the k chunks (factor base chunks each) the class may add.  A claim
// that overshoots the limit is undone at once, so near the limit another
// group can see the budget spent while that claim is only passing through:
// a group that meets it spent looks again a few times (about 3 us in all)
// before it gives up.
__device__ __forceinline__ uint32_t queue_chunks_for(uint32_t entries) { return (entries + kQcSpots - 1u) / kQcSpots; }

__device__ inline uint32_t commit_budget(HeapCore* h, uint32_t k, uint32_t factor, uint32_t e0, uint32_t per) {
  for (uint32_t look = 0, it = 0; look < 8u; ++look) {
    if (look) backoff(it);
    if (ld_relaxed(&h->budget.v) + factor > h->budget_limit) continue;   // spent for now: no atomics
    for (uint32_t kk = k; kk; kk >>= 1) {
      const unsigned long long d = static_cast<unsigned long long>(kk) * factor + queue_chunks_for(e0 + kk * per) -
                                   queue_chunks_for(e0);
      const unsigned long long old = atomicAdd(&h->budget.v, d);
      if (old + d <= h->budget_limit) return kk;
      atomicAdd(&h->budget.v, 0ull - d);
    }
  }
  return 0u;
}

// ============================================================ page queues

// The group adds k chunks to its class (the wait lambda of
// PageQueue_impl.cuh:114-125): allocate, describe, publish all their pages at
// the back with one position reservation, and credit the semaphore.  `owed`:
// the chunks cover a deficit (semaphore demand), so getting fewer marks the
// class short; pre-population owes nothing.
template <class Store>
__device__ uint32_t page_grow(HeapCore* h, ClassState* q, const Group& g, uint32_t k, bool owed) {
  const uint32_t factor = instance_factor(q->inst);
  uint32_t kk = 0;   // chunks this group may add
  if (g.is_leader()) {
    const uint32_t old = reserve_class_pages(h, q, k * q->ppc);
    if (old != kEmpty) {
      kk = k;
      if constexpr (Store::kKind != 0) kk = commit_budget(h, k, factor, old, q->ppc);
      if (kk < k) atomicSub(&q->class_pages, (k - kk) * q->ppc);
    }
  }
  kk = bcast(g, kk);
  uint32_t got = 0, c = kEmpty;
  if (kk) {
    got = alloc_chunks(h, g, kk, q->inst, false, &c);
    if (static_cast<uint32_t>(g.rank) < got && c != kEmpty) init_data_chunk(h, q, c, false);
    if (g.is_leader() && got < kk) {
      atomicSub(&q->class_pages, (kk - got) * q->ppc);
      if constexpr (Store::kKind != 0) atomicAdd(&h->budget.v, 0ull - static_cast<unsigned long long>(kk - got) * factor);
    }
  }
  const uint32_t E = got * q->ppc;
  if (E) {
    __threadfence();
    uint32_t b = 0;
    if (g.is_leader()) b = atomicAdd(&q->back.v, E);
    b = bcast(g, b);
    const uint32_t ppc = q->ppc;
    Store::template publish_range<true>(h, q, g, b, E, c, ppc,
                                        [ppc](uint32_t j, uint32_t cj) { return mem_index(cj, j % ppc); });
    __syncwarp(g.mask);
    __threadfence();
  }
  if (g.is_leader()) {
    // the pages first, then the holes: a group that resolves on seeing the
    // holes already counts the pages that did arrive
    sem_signal(q, E);
    if (owed && got < k) sem_mark_short(q, (k - got) * q->ppc);
  }
  return got;
}

template <class Store>
__device__ void* page_alloc(HeapCore* h, ClassState* q, const Group& g) {
#ifdef OURO_SCAN_STATS
  const long long t0 = clock64();
#endif
  uint32_t granted = sem_acquire(h, q, g, [&](uint32_t k) { page_grow<Store>(h, q, g, k, true); });
#ifdef OURO_SCAN_STATS
  const long long t1 = clock64();
#endif
  const bool served = static_cast<uint32_t>(g.rank) < granted;
  if (granted < static_cast<uint32_t>(g.size) && g.is_leader()) {
    atomicAdd(&h->oom.v, static_cast<unsigned long long>(g.size - granted));
    set_status(h, kErrOom);
  }
  const uint32_t smask = __ballot_sync(g.mask, served);
  if (!served) return nullptr;
  Group s = make_group(smask);
  uint32_t t = 0;
  if (s.is_leader()) t = atomicAdd(&q->front.v, granted);
  t = bcast(s, t);
  uint32_t v = Store::consume_lane(h, q, s, t + static_cast<uint32_t>(s.rank));
#ifdef OURO_SCAN_STATS
  if (s.is_leader()) {
    const long long t2 = clock64();
    atomicAdd(&h->scan[0].v, 1ull);
    atomicAdd(&h->scan[1].v, static_cast<unsigned long long>(t1 - t0));
    atomicAdd(&h->scan[2].v, static_cast<unsigned long long>(t2 - t1));
    if (t2 - t0 > (1ll << 20)) atomicAdd(&h->scan[8].v, 1ull);
    atomicMax(&h->scan[9].v, static_cast<unsigned long long>(t2 - t0));
  }
#endif
  if (v == kEmpty) return nullptr;
  return page_address(h, v >> kPageBits, v & ((1u << kPageBits) - 1u), q->page_shift);
}

// PageQueue_impl.cuh:137-142 / PageQueueVA_impl.cuh:175-224 / PageQueueVL_impl.cuh:102-122
template <class Store>
__device__ void page_free(HeapCore* h, ClassState* q, const Group& g, uint32_t index) {
  __threadfence();   // the caller's writes to the page are visible before it is handed out again
#ifdef OURO_SCAN_STATS
  const long long t0 = clock64();
#endif
  uint32_t b = 0;
  if (g.is_leader()) b = atomicAdd(&q->back.v, static_cast<uint32_t>(g.size));
  b = bcast(g, b);
  Store::publish_lane(h, q, g, b + static_cast<uint32_t>(g.rank), index);
  __syncwarp(g.mask);
  __threadfence();
  if (g.is_leader()) sem_signal(q, static_cast<uint32_t>(g.size));
#ifdef OURO_SCAN_STATS
  if (g.is_leader()) {
    const long long t1 = clock64();
    atomicAdd(&h->scan[4].v, 1ull);
    atomicAdd(&h->scan[5].v, static_cast<unsigned long long>(t1 - t0));
    atomicMax(&h->scan[6].v, static_cast<unsigned long long>(t1 - t0));
  }
#endif
}

// =========================================================== chunk queues

__device__ __forceinline__ uint32_t rotr32(uint32_t m, uint32_t off) { return off ? __funnelshift_r(m, m, off) : m; }
__device__ __forceinline__ uint32_t rotl32(uint32_t m, uint32_t off) { return off ? __funnelshift_l(m, m, off) : m; }

// Entries of the chunk queue: how many, against the queue capacity.
__device__ __forceinline__ uint32_t chunk_queue_cap(const ClassState* q, int kind) {
  return kind == 2 ? 0xFFFFFFF0u : q->page_cap;
}

template <class Store>
__device__ void chunk_enqueue(HeapCore* h, ClassState* q, uint32_t c) {
  int32_t fill = atomicAdd(&q->entries.v, 1);
  if (static_cast<uint32_t>(fill) >= chunk_queue_cap(q, Store::kKind)) {
    atomicSub(&q->entries.v, 1);
    st_relaxed(&h->meta[c].queue_pos, kEmpty);
    set_status(h, kErrQueueFull);
    return;
  }
  if (!Store::enqueue_one(h, q, c, &h->meta[c].queue_pos)) {
    atomicSub(&q->entries.v, 1);
    st_relaxed(&h->meta[c].queue_pos, kEmpty);
  }
}

// chunk_enqueue for the lanes of g, one chunk each, whose queue_pos the
// lanes have already moved from kEmpty to kPending: one reservation of g.size
// entries and back positions for the whole group instead of one per chunk.
// Seg: pieces of queue chunks one link call of a linked queue may attach
// (0: the default, one).  The frees of a burst re-enqueue up to one chunk per
// lane, so a free launch may need many queue chunks in a row; the allocation
// paths keep one, which keeps their kernels' code small.
constexpr uint32_t kFreeEnqueueSegments = 4u;
template <class Store, uint32_t Seg = 0u>
__device__ void chunk_enqueue_group(HeapCore* h, ClassState* q, const Group& g, uint32_t c) {
  const uint32_t n = static_cast<uint32_t>(g.size);
  uint32_t b = 0, full = 0;
  if (g.is_leader()) {
    const int32_t fill = atomicAdd(&q->entries.v, static_cast<int32_t>(n));
    if (static_cast<uint32_t>(fill) + n > chunk_queue_cap(q, Store::kKind)) {
      atomicSub(&q->entries.v, static_cast<int32_t>(n));
      set_status(h, kErrQueueFull);
      full = 1u;
    } else {
      b = atomicAdd(&q->back.v, n);
    }
  }
  if (bcast(g, full)) {
    st_relaxed(&h->meta[c].queue_pos, kEmpty);
    return;
  }
  const uint32_t pos = bcast(g, b) + static_cast<uint32_t>(g.rank);
  st_relaxed(&h->meta[c].queue_pos, pos);
  __threadfence();   // queue_pos before the entry: a consumer that finds the entry can remove it
  Store::template publish_lane<false, Seg>(h, q, g, pos, c);
}

// A chunk whose count rose above zero must be findable: enqueue it unless it
// still has (or is getting) an entry.  The reference does this on the first
// free of a full chunk (ChunkQueue_impl.cuh:157-161).
template <class Store>
__device__ void ensure_enqueued(HeapCore* h, ClassState* q, uint32_t c) {
  if (atomicCAS(&h->meta[c].queue_pos, kEmpty, kPending) == kEmpty) chunk_enqueue<Store>(h, q, c);
}

// The front moves over removed entries; one group at a time does it (a
// try-lock nobody waits on), so removals all over the queue do not turn into
// thousands of groups scanning the same run.  Collective over g.
template <class Store>
__device__ void help_front(HeapCore* h, ClassState* q, const Group& g) {
  uint32_t mine = 0;
  // test before the CAS: while one group moves the front, the others only read the line
  if (g.is_leader() && ld_relaxed(&q->advancing.v) == 0u) mine = atomicCAS(&q->advancing.v, 0u, 1u) == 0u ? 1u : 0u;
  if (!bcast(g, mine)) return;
  Store::advance_front(h, q, g);
  __syncwarp(g.mask);
  if (g.is_leader()) {
    __threadfence();
    atomicExch(&q->advancing.v, 0u);
  }
}

// Remove the entry of an exhausted chunk (the DEQUEUE_CHUNK mode of
// ChunkQueue_impl.cuh:128-137).  Called by one lane; returns kRemoved when it
// removed the entry, after which its group should help the front, plus
// kDrainedQc when the removal drained a queue chunk, after which its group
// runs Store::after_drain.  count = false leaves the class's entry count to
// the caller, which lowers it once for all removals of its group (the count
// line is shared by every group of the class).
// `at` is the cursor of the peek that found the entry: the queue chunk holding
// pos, which cannot drain before this removal, so the store need not find it
// again.
constexpr uint32_t kRemoved = 1u, kDrainedQc = 2u;
template <class Store>
__device__ uint32_t chunk_dequeue(HeapCore* h, ClassState* q, uint32_t c, uint32_t pos, bool count = true,
                                  const typename Store::Cursor* at = nullptr) {
  uint32_t* qp = &h->meta[c].queue_pos;
  // the CAS first: only an enqueue in flight (kPending) is waited for
  uint32_t seen = atomicCAS(qp, pos, kEmpty);
  for (uint32_t it = 0; seen == kPending;) {
    if (it >= 4096u) return 0u;
    backoff(it);
    seen = atomicCAS(qp, pos, kEmpty);
  }
  if (seen != pos) return 0u;   // someone else removed or moved it
  const bool drained = Store::remove(h, q, pos, at);
  if (count) atomicSub(&q->entries.v, 1);
  __threadfence();
  if (ld_relaxed(&h->meta[c].count) > 0) ensure_enqueued<Store>(h, q, c);
  return kRemoved | (drained ? kDrainedQc : 0u);
}

// Cooperative claim of `got` free pages of chunk c for the unserved lanes of
// s (in rank order).  The leader visits the mask words in the order the
// reference searches them for the leader's thread (ChunkAccess_impl.cuh:
// 75-125: first word (tid + 1) mod words, bits rotated by (tid + bid) mod 32),
// one word at a time and stopping as soon as enough bits are won: it picks
// the lowest set bits in rotated order, clears them with one atomicAnd, and
// the group hands the won bits to its unserved lanes by rank.
// `words`: the mask words the search visits.  A lone lane visits all W, in
// the reference's order (sequential parity); a group of two or more visits
// only the words the class's pages occupy (ceil(pages per chunk / 32)), since
// the rest are always empty: starting at (tid + 1) mod 16, a 256 B group
// otherwise loaded up to 15 empty words one after another before its own.
template <uint32_t W>
__device__ void claim_pages(HeapCore* h, const Group& s, uint32_t c, uint32_t got, bool& served, uint32_t& page,
                            uint32_t words = W) {
  ChunkMeta* m = h->meta + c;
  const uint32_t start = bcast(s, (threadIdx.x + 1u) % words);
  const uint32_t offset = bcast(s, (threadIdx.x + blockIdx.x) % 32u);
  uint32_t remaining = got;
  for (uint32_t attempt = 0; attempt < 64u && remaining; ++attempt) {
    for (uint32_t j = 0; j < words && remaining; ++j) {
      const uint32_t w = (start + j) % words;
      uint32_t won = 0;
      if (s.is_leader()) {
        const uint32_t rot = rotr32(ld_relaxed(m->mask(w)), offset);
        const uint32_t avail = static_cast<uint32_t>(__popc(rot));
        const uint32_t take = avail < remaining ? avail : remaining;
        if (take) {
          const uint32_t p = __fns(rot, 0u, static_cast<int>(take));
          const uint32_t picked = rotl32(rot & ((2u << p) - 1u), offset);
          won = picked & atomicAnd(m->mask(w), ~picked);
        }
      }
      won = bcast(s, won);
      if (!won) continue;
      // the u-th unserved lane takes the u-th won bit (in rotated order)
      const uint32_t unserved = __ballot_sync(s.mask, !served);
      const uint32_t u = static_cast<uint32_t>(__popc(unserved & ((1u << lane_id()) - 1u)));
      const uint32_t cnt = static_cast<uint32_t>(__popc(won));
      if (!served && u < cnt) {
        const uint32_t p = __fns(rotr32(won, offset), 0u, static_cast<int>(u + 1u));
        page = w * 32u + (p + offset) % 32u;
        served = true;
      }
      remaining -= cnt;
    }
  }
  if (remaining && s.is_leader()) set_status(h, kErrCorrupt);   // count promised pages the mask did not show
}

// The wait lambda of ChunkQueue_impl.cuh:86-100: k empty chunks, each with one
// queue entry, then credit the semaphore (`owed` as for page_grow).
template <class Store>
__device__ uint32_t chunk_grow(HeapCore* h, ClassState* q, const Group& g, uint32_t k, bool owed) {
  const uint32_t factor = instance_factor(q->inst);
  uint32_t kk = k;
  if constexpr (Store::kKind != 0) {
    // a chunk has at most one live entry; removed entries wait for the front
    // and re-enqueued chunks take new positions: the budget counts three queue
    // entries per chunk
    if (g.is_leader()) {
      const uint32_t old = atomicAdd(&q->class_chunks, k);
      kk = commit_budget(h, k, factor, 3u * old, 3u);
      if (kk < k) atomicSub(&q->class_chunks, k - kk);
    }
    kk = bcast(g, kk);
  }
  uint32_t c = kEmpty;
  uint32_t got = kk ? alloc_chunks(h, g, kk, q->inst, false, &c) : 0u;
  if constexpr (Store::kKind != 0) {
    if (g.is_leader() && got < kk) {
      atomicSub(&q->class_chunks, kk - got);
      atomicAdd(&h->budget.v, 0ull - static_cast<unsigned long long>(kk - got) * factor);
    }
  }
  const bool mine = static_cast<uint32_t>(g.rank) < got && c != kEmpty;
  if (mine) {
    init_data_chunk(h, q, c, true);
    st_relaxed(&h->meta[c].queue_pos, kPending);
  }
  __syncwarp(g.mask);
  __threadfence();
  // one entry per chunk, in rank order (k <= group size), reserved together
  const uint32_t em = __ballot_sync(g.mask, mine);
  if (mine) chunk_enqueue_group<Store>(h, q, make_group(em), c);
  __syncwarp(g.mask);
  __threadfence();
  if (g.is_leader()) {
    sem_signal(q, got * q->ppc);   // pages first, then holes (as in page_grow)
    if (owed && got < k) sem_mark_short(q, (k - got) * q->ppc);
  }
  return got;
}

// Next-fit run for a contended group: `run` consecutive queue positions from
// the class's scan cursor, mapped into the current window [front, back).
template <class Store>
__device__ uint32_t claim_run(HeapCore* h, ClassState* q, uint32_t run) {
  const uint32_t c = atomicAdd(&q->cursor.v, run);
  const uint32_t f = ld_relaxed(&q->front.v);
  const uint32_t w = ld_relaxed(&q->back.v) - f;
  if (static_cast<int32_t>(w) <= 0) return f;
  return f + (c - f) % w;
}

// Exclusive prefix sum of v over the ranks of group g.
__device__ __forceinline__ uint32_t group_exclusive_sum(const Group& g, uint32_t v) {
  uint32_t incl = v;
  const int r = g.rank;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t other = __shfl_sync(g.mask, incl, lane_of_rank(g.mask, r >= d ? r - d : r));
    if (d < g.size && r >= d) incl += other;
  }
  return incl - v;
}

// A group takes one run of ceil(lanes / pages-per-chunk) positions from the
// scan cursor and works it in parallel: lane r examines position r of the run
// (entry, page size, free count) and reserves on its chunk what the group
// still needs after the lanes below it; the pages are claimed (each lane on
// its own chunk when the run covers several, the group together when it is
// one chunk) and the takers of a chunk's last pages remove its entry.
// Whatever the run could not serve is left to the probe loop.
template <class Store>
__device__ void chunk_alloc_run(HeapCore* h, ClassState* q, const Group& s, typename Store::Cursor& cur,
                                uint32_t run, bool& served, uint32_t& page, uint32_t& chunk) {
  const uint32_t r = static_cast<uint32_t>(s.rank);
  const uint32_t need = static_cast<uint32_t>(s.size);
  uint32_t base = 0, back = 0;
  if (s.is_leader()) {
    base = claim_run<Store>(h, q, run);
    back = ld_relaxed(&q->back.v);
  }
  base = bcast(s, base);
  back = bcast(s, back);
  const uint32_t pos = base + r;
  uint32_t v = kEmpty, cnt = 0;
  if (r < run && static_cast<int32_t>(back - pos) > 0) {
    v = Store::peek(h, q, pos, cur);
    if (v < h->max_chunks) {
      const uint4 hd = ld_relaxed_v4(&h->meta[v].page_size);   // page_size, head, size, count
      if (hd.x == q->page_size && hd.y == 0u && static_cast<int32_t>(hd.w) > 0) cnt = hd.w;
    }
  }
  const uint32_t before = group_exclusive_sum(s, cnt);
  uint32_t want = need > before ? need - before : 0u;
  if (want > cnt) want = cnt;
  uint32_t got = 0;
  bool last = false;
  if (want) {
    const int32_t old = atomicSub(&h->meta[v].count, static_cast<int32_t>(want));
    got = old <= 0 ? 0u : (static_cast<uint32_t>(old) < want ? static_cast<uint32_t>(old) : want);
    if (got < want) {
      const int32_t give = static_cast<int32_t>(want - got);
      const int32_t prev = atomicAdd(&h->meta[v].count, give);
      if (prev <= 0 && prev + give > 0) ensure_enqueued<Store>(h, q, v);
    }
    last = got > 0u && old <= static_cast<int32_t>(want);
  }
  if (run > 1u) {
    // More than one chunk: a chunk then has at most 16 pages, all in mask
    // word 0, so every lane that reserved pages claims its own chunk's bits
    // (lowest first) at the same time, and the won pages go to the lanes in
    // rank order by a prefix sum over them.
    uint32_t won = 0;
    if (got) {
      uint32_t* mw = h->meta[v].mask(0);
      uint32_t remaining = got;
      for (uint32_t attempt = 0; attempt < 64u && remaining; ++attempt) {
        const uint32_t w = ld_relaxed(mw);
        const uint32_t avail = static_cast<uint32_t>(__popc(w));
        const uint32_t take = avail < remaining ? avail : remaining;
        if (!take) continue;
        const uint32_t p = __fns(w, 0u, static_cast<int>(take));   // the take-th lowest set bit
        const uint32_t picked = w & (p == 31u ? ~0u : ((2u << p) - 1u));
        const uint32_t wonnow = picked & atomicAnd(mw, ~picked);
        won |= wonnow;
        remaining -= static_cast<uint32_t>(__popc(wonnow));
      }
      if (remaining) set_status(h, kErrCorrupt);   // count promised pages the mask did not show
    }
    const uint32_t wcnt = static_cast<uint32_t>(__popc(won));
    const uint32_t first = group_exclusive_sum(s, wcnt);
    for (uint32_t m = __ballot_sync(s.mask, won != 0u); m; m &= m - 1u) {
      const int src = __ffs(m) - 1;
      const uint32_t c = __shfl_sync(s.mask, v, src);
      const uint32_t wb = __shfl_sync(s.mask, won, src);
      const uint32_t f0 = __shfl_sync(s.mask, first, src);
      if (r >= f0 && r < f0 + static_cast<uint32_t>(__popc(wb))) {
        page = __fns(wb, 0u, static_cast<int>(r - f0 + 1u));
        chunk = c;
        served = true;
      }
    }
  } else {
    for (uint32_t m = __ballot_sync(s.mask, got > 0u); m; m &= m - 1u) {
      const int src = __ffs(m) - 1;
      const uint32_t c = __shfl_sync(s.mask, v, src);
      const uint32_t k = __shfl_sync(s.mask, got, src);
      const bool was = served;
      if (q->inst == 0u) claim_pages<16u>(h, s, c, k, served, page, (q->ppc + 31u) / 32u);
      else claim_pages<1u>(h, s, c, k, served, page);
      if (served && !was) chunk = c;
    }
  }
  // The takers of the chunks' last pages remove their entries together: each
  // claims its entry (queue_pos) and writes the tombstone, then the removals
  // are counted once per counter (segment or queue chunk) and once on the
  // class's entry count.  A run's positions are consecutive, so its removals
  // nearly always share one counter, which every group of the burst would
  // otherwise hit once per removal.
  uint32_t key = kEmpty;
  bool mine = false;
  if (last) {
    uint32_t* qp = &h->meta[v].queue_pos;
    uint32_t seen = atomicCAS(qp, pos, kEmpty);   // only an enqueue in flight (kPending) is waited for
    for (uint32_t it = 0; seen == kPending && it < 4096u;) {
      backoff(it);
      seen = atomicCAS(qp, pos, kEmpty);
    }
    if (seen == pos) {
      mine = true;
      key = Store::remove_mark(h, q, pos, &cur);
    }
  }
  const uint32_t removed = __ballot_sync(s.mask, mine);
  uint32_t drained = 0;
  if (removed) {
    __syncwarp(s.mask);
    __threadfence();   // tombstones before counts; queue_pos before the count re-check below
    const uint32_t keyed = __ballot_sync(s.mask, mine && key != kEmpty);
    if (mine && key != kEmpty) {
      const Group kg = group_by(keyed, key);
      if (kg.is_leader() && Store::remove_count(h, q, key, static_cast<uint32_t>(kg.size))) drained = 1u;
    }
    if (s.is_leader()) atomicSub(&q->entries.v, __popc(removed));
    // a free that raced with the removal may have found the entry still there
    if (mine && ld_relaxed(&h->meta[v].count) > 0) ensure_enqueued<Store>(h, q, v);
  }
  if (__ballot_sync(s.mask, drained != 0u)) Store::after_drain(h, q, s);
  if (removed) help_front<Store>(h, q, s);
}

// ChunkQueue_impl.cuh:82-148 allocPage, for a group.  The first probe is the
// front entry, which is where the reference starts and where a lone lane
// always finds pages (exhausted chunks leave the queue at once).  A group that
// misses there is contending with others and continues with next-fit runs of
// ceil(need / pages-per-chunk) entries taken from the scan cursor, so
// concurrent groups work on disjoint chunks instead of all scanning from the
// front.
template <class Store>
__device__ void* chunk_alloc(HeapCore* h, ClassState* q, const Group& g) {
#ifdef OURO_SCAN_STATS
  long long t_begin = clock64(), t_claim = 0, t_deq = 0;
#endif
  uint32_t granted = sem_acquire(h, q, g, [&](uint32_t k) { chunk_grow<Store>(h, q, g, k, true); });
#ifdef OURO_SCAN_STATS
  const long long t_sem = clock64() - t_begin;
#endif
  const bool in = static_cast<uint32_t>(g.rank) < granted;
  if (granted < static_cast<uint32_t>(g.size) && g.is_leader()) {
    atomicAdd(&h->oom.v, static_cast<unsigned long long>(g.size - granted));
    set_status(h, kErrOom);
  }
  const uint32_t smask = __ballot_sync(g.mask, in);
  if (!in) return nullptr;
  Group s = make_group(smask);
  bool served = false;
  uint32_t page = 0, chunk = kEmpty;
  uint32_t pos = 0, run_end = 0, streak = 0;
  typename Store::Cursor cur = Store::cursor(q);
  uint32_t need = static_cast<uint32_t>(s.size);
  {
    // A group starts with a run from the cursor, which spreads concurrent
    // groups over the chunks; a lone lane starts at the front as the
    // reference does.
    const uint32_t run = (need + q->ppc - 1u) / q->ppc;
    if (s.size > 1) {
      chunk_alloc_run<Store>(h, q, s, cur, run, served, page, chunk);
      // the whole group stays in the probe loop, served lanes included: its
      // sweeps cover one position per lane of the group, not of the rest
      need = static_cast<uint32_t>(__popc(__ballot_sync(s.mask, !served)));
      if (need == 0u) {
#ifdef OURO_SCAN_STATS
        if (s.is_leader()) {   // served by the run: slow ones are counted with the slow probe-loop groups
          const unsigned long long total = static_cast<unsigned long long>(clock64() - t_begin);
          if (total > (1ull << 19)) {
            atomicAdd(&h->scan[4].v, static_cast<unsigned long long>(t_sem));
            atomicAdd(&h->scan[5].v, total - static_cast<unsigned long long>(t_sem));
            atomicAdd(&h->scan[8].v, 1ull);
          }
          atomicMax(&h->scan[9].v, total);
        }
#endif
        return page_address(h, chunk, page, q->page_shift);
      }
    }
  }
  if (s.is_leader()) {
    pos = ld_relaxed(&q->front.v);
    run_end = pos + 1u;
  }
#ifdef OURO_SCAN_STATS
  unsigned long long st_probe = 0, st_miss = 0, st_run = 0;
#define OURO_STAT(x) ++(x)
#else
#define OURO_STAT(x) ((void)0)
#endif
  for (uint32_t iter = 0;; ++iter) {
    uint32_t c = kEmpty, got = 0, last = 0, help = 0;
    if (s.is_leader()) {
      if (iter > 4u * kSpinLimit) {
        note_timeout(h, kWaitChunkScan);
        c = kTomb;
      } else {
        if (pos == run_end) {
          const uint32_t run = (need + q->ppc - 1u) / q->ppc;
          pos = claim_run<Store>(h, q, run);
          run_end = pos + run;
          OURO_STAT(st_run);
        }
        const uint32_t v = Store::peek(h, q, pos, cur);
        OURO_STAT(st_probe);
        if (v == kTomb && iter == 0u) help = 1u;   // the front entry is gone
        const bool live = v < kTomb && v < h->max_chunks && ld_relaxed(&h->meta[v].page_size) == q->page_size;
        if (live && ld_relaxed(&h->meta[v].count) > 0) {
          int32_t old = atomicSub(&h->meta[v].count, static_cast<int32_t>(need));
          got = old <= 0 ? 0u : (static_cast<uint32_t>(old) < need ? static_cast<uint32_t>(old) : need);
          if (got < need) {
            int32_t give = static_cast<int32_t>(need - got);
            int32_t prev = atomicAdd(&h->meta[v].count, give);
            if (prev <= 0 && prev + give > 0) ensure_enqueued<Store>(h, q, v);
          }
          last = (got > 0 && old <= static_cast<int32_t>(need)) ? 1u : 0u;
          c = got ? v : kEmpty;
        }
        if (!got) {
          OURO_STAT(st_miss);
          ++pos;
          ++streak;
          if (static_cast<int32_t>(ld_relaxed(&q->back.v) - pos) <= 0) run_end = pos;   // next: a fresh run
        } else {
          streak = 0;
        }
      }
    }
    c = bcast(s, c);
    if (c == kTomb) return nullptr;   // gave up
    if (bcast(s, help)) help_front<Store>(h, q, s);
    got = bcast(s, got);
    if (got) {
      last = bcast(s, last);
      bool before = served;
#ifdef OURO_SCAN_STATS
      long long t0 = clock64();
#endif
      if (q->inst == 0u) claim_pages<16u>(h, s, c, got, served, page, s.size > 1 ? (q->ppc + 31u) / 32u : 16u);
      else claim_pages<1u>(h, s, c, got, served, page);
#ifdef OURO_SCAN_STATS
      t_claim += clock64() - t0;
      t0 = clock64();
#endif
      if (served && !before) chunk = c;
      uint32_t removed = 0;
      if (s.is_leader()) {
        if (last) removed = chunk_dequeue<Store>(h, q, c, pos, true, &cur);
        ++pos;
      }
      removed = bcast(s, removed);
      if (removed & kDrainedQc) Store::after_drain(h, q, s);
      if (removed) help_front<Store>(h, q, s);
#ifdef OURO_SCAN_STATS
      t_deq += clock64() - t0;
#endif
      need = static_cast<uint32_t>(__popc(__ballot_sync(s.mask, !served)));
      if (need == 0u) break;
    } else {
      if (s.is_leader() && iter == 0u) run_end = pos;   // missed at the front: contended, switch to next-fit runs
      // Two misses in a row: the chunks with free pages have become sparse.
      // Late in a burst they sit near the front (the front moves over removed
      // entries), so the group sweeps from the front, one position per lane
      // and round -- entry, page size, free count -- and the leader moves to
      // the first chunk with free pages; after four empty rounds a fresh run.
      if (bcast(s, streak >= 2u ? 1u : 0u)) {
        uint32_t p0 = 0, back = 0;
        if (s.is_leader()) {
          p0 = ld_relaxed(&q->front.v);
          back = ld_relaxed(&q->back.v);
        }
        p0 = bcast(s, p0);
        back = bcast(s, back);
        uint32_t m = 0, sweeps = 0;
        for (; sweeps < 4u && !m && static_cast<int32_t>(back - p0) > 0; ++sweeps, p0 += static_cast<uint32_t>(s.size)) {
          const uint32_t p = p0 + static_cast<uint32_t>(s.rank);
          bool cand = false;
          if (static_cast<int32_t>(back - p) > 0) {
            const uint32_t v = Store::peek(h, q, p, cur);
            if (v < h->max_chunks) {
              const uint4 hd = ld_relaxed_v4(&h->meta[v].page_size);   // page_size, head, size, count
              cand = hd.x == q->page_size && hd.y == 0u && static_cast<int32_t>(hd.w) > 0;
            }
          }
          m = __ballot_sync(s.mask, cand);
          if (m) break;
        }
        // nothing with free pages near the front: removed entries may hide
        // them there, so the group moves the front before its next run
        if (!m) help_front<Store>(h, q, s);
        if (s.is_leader()) {
          streak = 0;
          if (m) {
            // groups that sweep at the same time see the same candidates: each
            // takes one picked by a hash of its warp, so that they spread over
            // the chunks instead of queueing for the first one (with one or two
            // pages per chunk that convoy cost O(groups^2) probes)
            const uint32_t k = (blockIdx.x * 0x9E3779B1u + (threadIdx.x >> 5) * 0x85EBCA77u + iter * 0xC2B2AE3Du) %
                               static_cast<uint32_t>(__popc(m));
            const uint32_t lane = __fns(m, 0u, static_cast<int>(k + 1u));
            pos = p0 + static_cast<uint32_t>(__popc(s.mask & ((1u << lane) - 1u)));
            run_end = pos + 1u;
          } else {
            pos = run_end;   // nothing near the front: a fresh run next
          }
        }
#ifdef OURO_SCAN_STATS
        st_probe += static_cast<unsigned long long>(sweeps) * s.size;
#endif
      }
    }
  }
#ifdef OURO_SCAN_STATS
  if (s.is_leader()) {
    atomicAdd(&h->scan[0].v, 1ull);
    atomicAdd(&h->scan[1].v, st_probe);
    atomicAdd(&h->scan[2].v, st_miss);
    atomicAdd(&h->scan[3].v, st_run);
    const unsigned long long total = static_cast<unsigned long long>(clock64() - t_begin);
    if (total > (1ull << 19)) {   // slow groups: where their time went
      atomicAdd(&h->scan[4].v, static_cast<unsigned long long>(t_sem));
      atomicAdd(&h->scan[5].v, static_cast<unsigned long long>(clock64() - t_begin - t_sem - t_claim - t_deq));
      atomicAdd(&h->scan[6].v, static_cast<unsigned long long>(t_deq));
      atomicAdd(&h->scan[7].v, static_cast<unsigned long long>(t_claim));
      atomicAdd(&h->scan[8].v, 1ull);
      atomicAdd(&h->scan[10].v, st_probe);
      atomicAdd(&h->scan[11].v, st_miss);
    }
    atomicMax(&h->scan[9].v, total);
  }
#endif
#undef OURO_STAT
  return page_address(h, chunk, page, q->page_shift);
}

// ChunkQueue*_impl.cuh freePage: set the bits, raise the counts, re-enqueue
// chunks that were full, then signal the semaphore once for the class group.
template <class Store, bool Standard>
__device__ void chunk_free(HeapCore* h, ClassState* q, const Group& g, uint32_t c, uint32_t page) {
  __threadfence();
  Group cg = group_by(g.mask, c);
  Group wg = group_by(cg.mask, page >> 5);
  uint32_t bits = __reduce_or_sync(wg.mask, 1u << (page & 31u));
  ChunkMeta* m = h->meta + c;
  if (wg.is_leader()) atomicOr(m->mask(page >> 5), bits);
  __syncwarp(cg.mask);
  __threadfence();
  uint32_t flashed = 0, help = 0, enq = 0, drained = 0;
  if (cg.is_leader()) {
    const int32_t n = cg.size;
    int32_t old = atomicAdd(&m->count, n);
    const int32_t size = static_cast<int32_t>(ld_relaxed(&m->size));
    if (old <= 0 && old + n > 0) {
      // the chunk needs an entry unless it still has (or is getting) one
      enq = atomicCAS(&m->queue_pos, kEmpty, kPending) == kEmpty ? 1u : 0u;
      // frees only add entries at the back: when removed entries pile up
      // ahead of the front (nothing has been allocating), move the front, so
      // that the queue chunks behind it return to the pool
      if (ld_relaxed(&q->back.v) - ld_relaxed(&q->front.v) >
          static_cast<uint32_t>(ld_relaxed(&q->entries.v)) + kFrontSlack)
        help = 1u;
    } else if (Standard && old + n == size && ld_relaxed(&q->entries.v) > kLowerFillC) {
      // ChunkQueue_impl.cuh:162-199: hand a fully free chunk back to the pool
      if (sem_try_reduce(q, static_cast<uint32_t>(size - n))) {
        if (atomicCAS(&m->count, size, 0) == size) {
          uint32_t qp, it = 0;
          while ((qp = ld_relaxed(&m->queue_pos)) == kPending && it < 4096u) backoff(it);
          if (qp != kPending && qp != kEmpty && atomicCAS(&m->queue_pos, qp, kEmpty) == qp) {
            drained = Store::remove(h, q, qp) ? 1u : 0u;
            atomicSub(&q->entries.v, 1);
            flashed = 2u;
          } else {
            flashed = 1u;
          }
          reuse_put(h, &h->reuse[q->inst], c);
        } else {
          sem_signal(q, static_cast<uint32_t>(size - n));
        }
      }
    }
  }
  // the chunks of the warp that need an entry are enqueued together
  const uint32_t em = __ballot_sync(g.mask, enq != 0u);
  if (enq) chunk_enqueue_group<Store, kFreeEnqueueSegments>(h, q, make_group(em), c);
  flashed = __shfl_sync(cg.mask, flashed, cg.leader);
  help = __shfl_sync(cg.mask, help, cg.leader);
  if (__shfl_sync(cg.mask, drained, cg.leader)) Store::after_drain(h, q, cg);
  if (flashed == 2u || help) help_front<Store>(h, q, cg);
  __syncwarp(g.mask);
  __threadfence();
  uint32_t total = __reduce_add_sync(g.mask, flashed ? 0u : 1u);
  if (g.is_leader()) sem_signal(q, total);
}

// ========================================================= initial chunks
// Ouroboros.cuh:291-295 enqueueInitialChunk, together with the chunk
// initializer its callers run first (PageIndexChunk.cuh:82-86,
// ChunkIndexChunk.cuh:73-78 with ChunkAccess.cuh:31-64): chunk c, taken from
// the pool by the caller, joins class q with its first ppc - avail pages in the
// caller's use and the other avail pages free.  Page-based, those pages are
// queued in page order (PageQueue_impl.cuh:40-53, PageQueueVA_impl.cuh:94-125,
// PageQueueVL_impl.cuh:54-63); chunk-based, the chunk gets one queue entry
// (ChunkQueue_impl.cuh:69-77, ChunkQueueVA_impl.cuh:54-72,
// ChunkQueueVL_impl.cuh:49-56).  Then the semaphore gains avail pages.  One
// lane; false when the queue or the chunk budget has no room.
template <class Store, bool PageBased>
__device__ bool enqueue_initial(HeapCore* h, ClassState* q, uint32_t c, uint32_t avail) {
  const Group self = make_group(1u << lane_id());
  const uint32_t ppc = q->ppc, start = ppc - avail;
  ChunkMeta* m = h->meta + c;
  if constexpr (PageBased) {
    const uint32_t old = reserve_class_pages(h, q, ppc);
    if (old == kEmpty) return false;
    if constexpr (Store::kKind != 0) {
      if (!commit_budget(h, 1u, 1u, old, ppc)) {
        atomicSub(&q->class_pages, ppc);
        return false;
      }
    }
    init_data_chunk(h, q, c, false);
    __threadfence();
    const uint32_t b = atomicAdd(&q->back.v, avail);
    Store::template publish_range<true>(h, q, self, b, avail, c, avail,
                                        [start](uint32_t j, uint32_t cj) { return mem_index(cj, start + j); });
    __threadfence();
  } else {
    if constexpr (Store::kKind != 0) {
      const uint32_t old = atomicAdd(&q->class_chunks, 1u);
      if (!commit_budget(h, 1u, 1u, 3u * old, 3u)) {
        atomicSub(&q->class_chunks, 1u);
        return false;
      }
    }
    st_relaxed(&m->size, ppc);
    st_relaxed(&m->head, 0u);
    st_relaxed(&m->count, static_cast<int32_t>(avail));
    st_relaxed(&m->queue_pos, kPending);
    // ChunkAccess.cuh:31-64: pages [0, ppc - avail) taken, the rest free
    uint32_t n = ppc, taken = start;
#pragma unroll
    for (uint32_t w = 0; w < 16u; ++w) {
      const uint32_t full = n >= 32u ? 0xFFFFFFFFu : ((1u << n) - 1u);
      const uint32_t used = taken >= 32u ? 0xFFFFFFFFu : ((1u << taken) - 1u);
      st_relaxed(m->mask(w), full & ~used);
      n = n > 32u ? n - 32u : 0u;
      taken = taken > 32u ? taken - 32u : 0u;
    }
    __threadfence();
    st_relaxed(&m->page_size, q->page_size);
    __threadfence();
    chunk_enqueue<Store>(h, q, c);
  }
  sem_signal(q, avail);
  return true;
}

}  // namespace ouro
