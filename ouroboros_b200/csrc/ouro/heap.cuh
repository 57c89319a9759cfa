// heap.cuh -- heap layout, chunk metadata, chunk allocation and the chunk
// reuse queue.
#pragma once

#include "common.cuh"

namespace ouro {

// Out-of-band metadata of one base chunk (one 128 B line).  A chunk plays one
// role at a time: page chunk (page-based variants), chunk-index chunk
// (chunk-based variants: free-page count + occupancy bitmask) or queue chunk
// (2048 queue entries of the virtualized variants, stored in its data).
// The first 32 B sector holds what an allocation of a chunk-based class with
// at most 128 pages per chunk touches: the header, the free count and the
// first four mask words; the queue fields follow in the same 64 B half, so a
// request of 64 B or more reads the record from DRAM once, in one piece.
struct alignas(128) ChunkMeta {
  uint32_t page_size;   // data chunks: page size of their class; 0 otherwise
  uint32_t head;        // >0: continuation of a 4-chunk chunk starting `head` chunks lower
  uint32_t size;        // pages in the chunk
  int32_t count;        // chunk-based: free pages (may dip below 0 transiently)
  uint32_t mask_lo[4];  // chunk-based: mask words 0..3 (one bit per page, 1 = free)
  uint32_t queue_pos;   // chunk-based: virtual position of its queue entry, kEmpty or kPending
  uint32_t qcount;      // queue chunk: present << 16 | enqueued
  uint32_t vstart;      // queue chunk: first virtual position stored here
  uint32_t next;        // linked queue chunk: next queue chunk, kEmpty if none yet
  uint32_t reserved_[4];
  uint32_t mask_hi[12]; // chunk-based: mask words 4..15 (pages 128..511 of the 16 B class)
  uint32_t reserved2_[4];
  // mask word w (0..15)
  __host__ __device__ uint32_t* mask(uint32_t w) { return w < 4u ? mask_lo + w : mask_hi + (w - 4u); }
  __host__ __device__ const uint32_t* mask(uint32_t w) const { return w < 4u ? mask_lo + w : mask_hi + (w - 4u); }
};
static_assert(sizeof(ChunkMeta) == 128, "metadata record must be one 128 B line");

// A counter of its own 256 B block.
template <typename T>
struct alignas(256) Line {
  T v;
};

// A counter that many warps hit.  One hot 32-bit address takes about 1.5 G
// RMW/s from one L2 slice.  Two hot addresses 128 B apart (one 256 B block)
// together still take 1.3 G/s: they share the slice.  At 4 KiB apart they
// take 2.8 G/s, and 8 of them 8.9 G/s; nearer strides can still land in one
// slice.  So the counters that one request path hits together (semaphore,
// front or back, entry count, cursor) are each given 4 KiB of their own.
template <typename T>
struct alignas(4096) Hot {
  T v;
};

// Per size class queue state.  Every counter that many warps hit is a Hot
// block, so that the L2 slices serve them independently.
struct alignas(4096) ClassState {
  Hot<unsigned long long> sem;   // page semaphore (count / supply)
  Hot<uint32_t> front;           // consumer position (virtual)
  Hot<uint32_t> back;            // producer position (virtual)
  Hot<int32_t> entries;          // chunk-based: entries in the queue (count_)
  Hot<uint32_t> cursor;          // chunk-based: next-fit scan cursor for contended groups
  Hot<uint32_t> advancing;       // chunk-based: try-lock of the group moving the front
  Hot<uint32_t> ptr_lock;        // linked: try-lock of the group moving front_ptr / old_ptr
  // cold line
  uint32_t* ring;                 // standard: the ring; virtualized array: the index array
  uint32_t ring_mask;
  uint32_t cls, inst, page_size, page_shift, ppc, words;
  uint32_t front_ptr, back_ptr, old_ptr, old_count;  // linked: chunk indices
  uint32_t class_pages;           // pages ever created for the class (queue capacity guard)
  uint32_t class_chunks;          // chunk-based: chunks ever created for the class (budget)
  uint32_t page_cap;
  uint32_t clean_on_recycle;      // chunk queues: queue chunks hold kTomb entries when drained
  int32_t holes;                  // semaphore: pages of failed chunk additions not yet handed back
  uint32_t* skip;                 // linked: index of recently linked queue chunks
  uint32_t* seg;                  // standard chunk queues: removed entries per 2048-entry ring segment
  uint32_t seg_mask;              // standard chunk queues: ring segments - 1
};

struct alignas(4096) ReuseQueue {
  Hot<int32_t> count;
  Hot<uint32_t> front;
  Hot<uint32_t> back;
  uint32_t* ring;
};

constexpr uint32_t kScanCounters = 12u;

// Device-resident control block, the object device code calls malloc/free on.
struct alignas(4096) HeapCore {
  // cold configuration line
  int32_t variant;
  uint32_t max_chunks;
  ChunkMeta* meta;
  char* data;
  char* data_end;
  char* base;
  unsigned long long alloc_bytes;
  unsigned long long heap_bytes;
  unsigned long long budget_limit;     // virtualized: chunks the budget may commit (0: no budget)
  uint32_t agg_width;                  // lanes per aggregation segment of a warp (1..32, a power of two)
  // hot / warm counters
  Hot<unsigned long long> next_free_chunk;
  Hot<uint32_t> status;
  Hot<unsigned long long> oom;        // null results handed out
  Line<unsigned long long> timeouts;   // bounded waits that gave up
  Line<uint32_t> timeout_sites;        // WaitSite bits of the waits that gave up
  Line<unsigned long long> chunk_allocs;
  Hot<unsigned long long> budget;     // virtualized: data chunks + queue chunks the classes need
  ReuseQueue reuse[2];
  ClassState cls[kNumClasses];
  // diagnostic counters, only written when built with OURO_SCAN_STATS (their
  // meaning per heap kind is listed at ouro_scan_stats in the C header)
  Line<unsigned long long> scan[kScanCounters];
  // work counter and result of the host's bulk pre-population call, kept in
  // the heap so that the call allocates nothing
  Line<uint32_t> prefill_next;
  Line<unsigned long long> prefill_done;
};

constexpr size_t kCoreBytes = 1u << 20;
static_assert(sizeof(HeapCore) <= kCoreBytes, "control block grew past its region");

__device__ __forceinline__ void set_status(HeapCore* h, uint32_t bits) { atomicOr(&h->status.v, bits); }
// Bounded waits, one bit each in HeapCore::timeout_sites when they give up.
enum WaitSite : uint32_t {
  kWaitSemRounds = 1u << 0,    // (unused: the semaphore has no acquisition rounds)
  kWaitSemCas = 1u << 1,       // (unused: the semaphore has no CAS loop on its hot path)
  kWaitSemReserve = 1u << 2,   // semaphore: pages of a group in deficit that do not arrive
  kWaitSlotEmpty = 1u << 3,    // queue slot still holding the previous lap's entry
  kWaitSlotFull = 1u << 4,     // queue slot whose producer does not write it
  kWaitIndexEntry = 1u << 5,   // virtualized array: queue chunk of a range
  kWaitLink = 1u << 6,         // linked: successor of a queue chunk
  kWaitLocateHops = 1u << 7,   // linked: walk longer than 2^20 hops
  kWaitLocateStale = 1u << 8,  // linked: walks kept meeting recycled chunks
  kWaitReuseRead = 1u << 9,    // chunk reuse ring: reserved entry not written
  kWaitReusePut = 1u << 10,    // chunk reuse ring: slot not yet read
  kWaitChunkScan = 1u << 11,   // chunk queue: scan for a chunk with free pages
};

__device__ __forceinline__ void note_timeout(HeapCore* h, uint32_t site) {
  set_status(h, kErrTimeout);
  atomicOr(&h->timeout_sites.v, site);
  atomicAdd(&h->timeouts.v, 1ull);
}

// -------------------------------------------------------------- layout
// Capacity: the reference's MemoryInitialization.cuh:156-166 arithmetic on its
// own object and queue sizes, so that max_chunks (and with it every success /
// failure count) is identical.  Physical placement is this build's own.
struct Layout {
  unsigned long long ring_entries;   // standard queues: ring entries per class
  unsigned long long vq_entries;     // virtualized-array queues: index entries per class
  unsigned long long ref_queue_bytes;
  unsigned long long ref_total_required;
  unsigned long long max_chunks;
  unsigned long long meta_off, data_off, ring_off, vq_off, skip_off, reuse_off, seg_off;
  unsigned long long alloc_bytes;
};

__host__ __device__ inline unsigned long long align_up(unsigned long long v, unsigned long long a) {
  return (v + a - 1u) / a * a;
}

// kind: 0 standard, 1 virtualized array, 2 virtualized linked list.  The queue
// sizes default to the reference's (page_queue_size, virtual_queue_size).
__host__ inline bool compute_layout(int kind, unsigned long long heap_bytes, Layout* L,
                                    unsigned long long ring_entries = kRingSize,
                                    unsigned long long vq_entries = kVqSize) {
  L->ring_entries = ring_entries;
  L->vq_entries = vq_entries;
  const unsigned long long per_queue = kind == 0 ? ring_entries * 4u : kind == 1 ? vq_entries * 4u : 0u;
  const unsigned long long reuse = align_up((unsigned long long)kReuseSize * 4u, kChunkBytes);
  const unsigned long long pq = align_up(per_queue, kChunkBytes);
  L->ref_queue_bytes = reuse + pq * 10u + reuse + pq * 2u;
  L->ref_total_required = align_up(8192u + L->ref_queue_bytes, kRefStride);
  const unsigned long long aligned = align_up(heap_bytes, kRefStride);
  if (aligned <= L->ref_total_required) return false;
  L->max_chunks = (aligned - L->ref_total_required) / kRefStride;
  if (L->max_chunks >= (1ull << (32 - kPageBits))) return false;   // MemoryIndex chunk bits
  L->meta_off = kCoreBytes;
  L->data_off = align_up(L->meta_off + L->max_chunks * kMetaBytes, kChunkBytes);
  unsigned long long off = L->data_off + L->max_chunks * kChunkBytes;
  L->ring_off = off;
  if (kind == 0) off += (unsigned long long)kNumClasses * ring_entries * 4u;
  L->vq_off = off;
  if (kind == 1) off += (unsigned long long)kNumClasses * vq_entries * 4u;
  L->skip_off = off;
  if (kind == 2) off += (unsigned long long)kNumClasses * kSkipSlots * 4u;
  L->reuse_off = off;
  off += 2ull * kReuseSize * 4u;
  L->seg_off = off;
  if (kind == 0) off += (unsigned long long)kNumClasses * (ring_entries / kQcSpots) * 4u;
  L->alloc_bytes = align_up(off, kChunkBytes) + kChunkBytes;   // + slack to 8 KiB-align the base
  return true;
}

// ------------------------------------------------------- reuse queue
// The chunk reuse ring (queues/Queue_impl.cuh:20-66): FIFO of whole chunks
// that left a queue.  take() serves up to k chunks for one group.
__device__ inline uint32_t reuse_take(HeapCore* h, ReuseQueue* r, uint32_t k, uint32_t* first_pos) {
  if (ld_relaxed(&r->count.v) <= 0) return 0u;   // empty: no atomics (a cold heap grows by the bump pointer)
  int32_t old = atomicSub(&r->count.v, static_cast<int32_t>(k));
  uint32_t got = old <= 0 ? 0u : (static_cast<uint32_t>(old) < k ? static_cast<uint32_t>(old) : k);
  if (got < k) atomicAdd(&r->count.v, static_cast<int32_t>(k - got));
  if (got) *first_pos = atomicAdd(&r->front.v, got);
  return got;
}

__device__ inline uint32_t reuse_read(HeapCore* h, ReuseQueue* r, uint32_t pos) {
  uint32_t* s = r->ring + (pos & (kReuseSize - 1u));
  uint32_t v, it = 0;
  while ((v = ld_acquire(s)) == kEmpty) {
    if (it >= kSpinLimit) { note_timeout(h, kWaitReuseRead); return kEmpty; }
    backoff(it);
  }
  st_relaxed(s, kEmpty);
  return v;
}

__device__ inline void reuse_put(HeapCore* h, ReuseQueue* r, uint32_t chunk) {
  // a pooled chunk is nobody's data chunk: lanes that still hold a stale
  // queue entry for it see the page size change and skip it
  st_relaxed(&h->meta[chunk].page_size, 0u);
  __threadfence();
  int32_t fill = atomicAdd(&r->count.v, 1);
  if (fill >= static_cast<int32_t>(kReuseSize)) {
    atomicSub(&r->count.v, 1);
    set_status(h, kErrQueueFull);   // the chunk stays out of circulation
    return;
  }
  uint32_t pos = atomicAdd(&r->back.v, 1u);
  uint32_t* s = r->ring + (pos & (kReuseSize - 1u));
  uint32_t it = 0;
  while (ld_relaxed(s) != kEmpty) {
    if (it >= kSpinLimit) { note_timeout(h, kWaitReusePut); return; }
    backoff(it);
  }
  st_release(s, chunk);
}

// ---------------------------------------------------- chunk allocation
// Ouroboros.cuh:108-136 / 200-229 allocateChunk, for a whole group: up to k
// chunks (k <= R x group size) with one reservation, reuse queue first, then
// the bump pointer.  Chunk i of the k goes to the lane of rank i mod n, in
// mine[i / n]; chunks i < result are valid (a reuse slot that timed out
// leaves kEmpty).  A chunk is valid when index + factor < max_chunks (the
// reference's bound).
template <int R>
__device__ inline uint32_t alloc_chunk_rounds(HeapCore* h, const Group& g, uint32_t k, uint32_t inst, bool queue_chunk,
                                              uint32_t (&mine)[R]) {
  const uint32_t factor = queue_chunk ? 1u : instance_factor(inst);
  ReuseQueue* r = (inst != 0u && queue_chunk) ? &h->reuse[0] : &h->reuse[inst];
  uint32_t from_reuse = 0, rpos = 0;
  unsigned long long first = 0;
  if (g.is_leader()) {
    from_reuse = reuse_take(h, r, k, &rpos);
    bool bumped = false;
    if (from_reuse < k) {
      // past the end the bump pointer is not moved again: an exhausted heap
      // answers with loads only
      first = ld_relaxed(&h->next_free_chunk.v);
      if (first + factor < h->max_chunks) {
        first = atomicAdd(&h->next_free_chunk.v, (unsigned long long)(k - from_reuse) * factor);
        bumped = true;
      }
    }
    if (from_reuse || bumped) atomicAdd(&h->chunk_allocs.v, (unsigned long long)k);
  }
  from_reuse = bcast(g, from_reuse);
  rpos = bcast(g, rpos);
  first = bcast64(g, first);
  const uint32_t n = static_cast<uint32_t>(g.size);
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const uint32_t i = static_cast<uint32_t>(j) * n + static_cast<uint32_t>(g.rank);
    uint32_t c = kEmpty;
    if (i < from_reuse) {
      c = reuse_read(h, r, rpos + i);
    } else if (i < k) {
      unsigned long long idx = first + (unsigned long long)(i - from_reuse) * factor;
      if (idx + factor < h->max_chunks) c = static_cast<uint32_t>(idx);
    }
    mine[j] = c;
  }
  // bumped chunks are valid as a prefix of their range
  unsigned long long avail = h->max_chunks > first + factor ? (h->max_chunks - first - 1u) / factor : 0u;
  uint32_t bumped = k - from_reuse;
  return from_reuse + (avail < bumped ? static_cast<uint32_t>(avail) : bumped);
}

// One chunk per lane (k <= group size): lane of rank i < result holds its
// chunk in *mine.
__device__ inline uint32_t alloc_chunks(HeapCore* h, const Group& g, uint32_t k, uint32_t inst, bool queue_chunk,
                                        uint32_t* mine) {
  uint32_t m[1];
  const uint32_t got = alloc_chunk_rounds<1>(h, g, k, inst, queue_chunk, m);
  *mine = m[0];
  return got;
}

// Fresh queue chunk (QueueChunk.cuh:217-221): header reset and all 2048
// entries set to kEmpty by the calling lane with 16 B stores.
// Header only: the entries of a queue chunk are already kEmpty when it is
// handed out -- the heap's data starts flooded with kEmpty (the reference's
// d_cleanChunks, MemoryInitialization.cuh:21-38), page queues leave every
// entry kEmpty as they drain, and chunk queues clean a queue chunk when they
// return it to the pool (clean_queue_chunk).  This keeps the 8 KiB rewrite
// off the path where producers wait for the next queue chunk.
__device__ inline void init_queue_chunk(HeapCore* h, uint32_t c, uint32_t vstart, uint32_t tag) {
  ChunkMeta* m = h->meta + c;
  st_relaxed(&m->page_size, 0u);
  st_relaxed(&m->size, tag);
  st_relaxed(&m->head, 0u);
  st_relaxed(&m->qcount, 0u);
  st_relaxed(&m->vstart, vstart);
  st_relaxed(&m->next, kEmpty);
}

// All 2048 entries of a queue chunk back to kEmpty (chunk queues leave
// removed entries as kTomb).
__device__ inline void clean_queue_chunk(HeapCore* h, uint32_t c) {
  uint32_t* slots = reinterpret_cast<uint32_t*>(h->data + (static_cast<size_t>(c) << kChunkShift));
  const uint4 e = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
#pragma unroll 8
  for (uint32_t i = 0; i < kQcSpots; i += 4u) st_v4(slots + i, e);
  __threadfence();
}

__device__ __forceinline__ uint32_t* queue_slots(HeapCore* h, uint32_t c) {
  return reinterpret_cast<uint32_t*>(h->data + (static_cast<size_t>(c) << kChunkShift));
}

// One lane allocates one queue chunk (allocateChunk<true>) and initializes it.
__device__ inline uint32_t new_queue_chunk(HeapCore* h, uint32_t inst, uint32_t vstart, uint32_t tag);

// Owner tag of a class's queue chunks, kept in ChunkMeta::size (data chunks
// hold their page count there, at most 512; recycled queue chunks 0): an index
// entry is trusted only for a chunk that still carries its class's tag.
constexpr uint32_t kQueueTag = 0x40000000u;
__device__ __forceinline__ uint32_t queue_tag(const ClassState* q) { return kQueueTag | q->cls; }

// Link slot of a queue chunk (a virtual-array index entry or a `next` field):
// the pre-allocating lane offers its chunk with a CAS; if a waiting lane got
// there first the offered chunk goes back to the pool.
__device__ inline void offer_queue_chunk(HeapCore* h, uint32_t* link, uint32_t nq) {
  if (nq == kEmpty) return;
  if (atomicCAS(link, kEmpty, nq) != kEmpty) reuse_put(h, &h->reuse[0], nq);
}

// A lane that has waited long for a link installs a queue chunk itself.
// Returns true when the link is now set (by anyone).
__device__ inline void install_queue_chunk(HeapCore* h, uint32_t* link, uint32_t inst, uint32_t vstart,
                                           uint32_t tag) {
  if (atomicCAS(link, kEmpty, kInstalling) != kEmpty) return;
  uint32_t nq = new_queue_chunk(h, inst, vstart, tag);
  st_release(link, nq);   // kEmpty again when no chunk was free: someone retries later
}

__device__ inline uint32_t new_queue_chunk(HeapCore* h, uint32_t inst, uint32_t vstart, uint32_t tag) {
  Group self = make_group(1u << lane_id());
  uint32_t c;
  uint32_t got = alloc_chunks(h, self, 1u, inst, true, &c);
  if (!got || c == kEmpty) return kEmpty;
  init_queue_chunk(h, c, vstart, tag);
  __threadfence();
  return c;
}

}  // namespace ouro
