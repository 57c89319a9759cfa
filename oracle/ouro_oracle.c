/*
 * ouro_oracle.c -- TEST INFRASTRUCTURE ONLY (see ouro_oracle.h).
 *
 * Sequential restatement of the reference allocator.  Every function names the
 * reference lines it follows (paths relative to the reference project root).
 * With a single thread every atomic of the reference collapses to a plain
 * read-modify-write, every spin either ends at once or never (reported as
 * ORC_ERR_HANG), and every warp-collective reduces to the calling lane.
 */
#include "ouro_oracle.h"

#include <stdlib.h>
#include <string.h>

#define EMPTY32 0xFFFFFFFFu
#define NONE_CHUNK 0xFFFFFFFFu
#define CHUNK_DATA 8192u            /* Parameters.h:18 CHUNK_SIZE           */
#define CHUNK_META 128u             /* Parameters.h:19 CHUNK_METADATA_SIZE  */
#define CHUNK_STRIDE 8320u          /* Chunk.cuh:23-26 meta + data           */
#define OBJECT_BYTES 8192u          /* Ouroboros.cuh:260 size_() aligns to ChunkBase::size_ */
#define QC_SPOTS 2048u              /* QueueChunk.cuh:26 num_spots_          */
#define VQ_SIZE 16384u              /* Parameters.h:12 virtual_queue_size    */
#define RING_SIZE (1u << 23)        /* Parameters.h:11 page_queue_size       */
#define REUSE_SIZE 65536u           /* Parameters.h:10 chunk_queue_size      */
#define OLD_HOLD 10u                /* Parameters.h:13 LARGEST_OLD_COUNT_VALUE */
#define C_LOWER_FILL 838860         /* ChunkQueue.cuh:32 (int)(2^23 * 0.1f)  */
#define QC_EMPTY_COUNT 2048u        /* counterA == 2048, counterB == 0       */

enum { KIND_S = 0, KIND_VA = 1, KIND_VL = 2 };

/* The two instances of every Multi* type (InstanceDefinitions.cuh:16-34,
 * Ouroboros.cuh:53-66): smallest page, queue count, chunk size, base chunks
 * per chunk, bitmask words (ChunkAccess.cuh:15), log2(smallest page). */
typedef struct { uint32_t smallest; int nq; uint32_t chunk_size; uint32_t factor; int words; int spf; } inst_t;
static const inst_t INST[2] = {{16u, 10, 8192u, 1u, 16, 4}, {16384u, 2, 32768u, 4u, 1, 14}};

typedef struct {
  uint32_t page_size;           /* CommonChunk::page_size (Chunk.cuh:9-13)       */
  uint32_t number_pages;        /* PageChunk (PageIndexChunk.cuh:13)             */
  int32_t acc_count;            /* ChunkAccess::count (ChunkAccess.cuh:28)       */
  uint32_t acc_size;            /* ChunkAccess::size                             */
  uint32_t mask[16];            /* ChunkAccess::availability_mask                */
  uint32_t queue_pos;           /* ChunkIndexChunk::queue_pos                    */
  uint32_t next;                /* QueueChunk::next_ as a chunk index            */
  uint32_t qcount;              /* QueueChunk::count_ (counterB << 16 | counterA) */
  uint32_t vstart;              /* QueueChunk::virtual_start_                    */
  uint32_t* slots;              /* QueueChunk storage, 2048 entries              */
} chunk_t;

typedef struct { uint32_t* q; int32_t count; uint32_t front, back; } reuse_t;

typedef struct {
  int64_t count, expected, reserved;   /* BulkSemaphore fields                 */
  uint32_t front, back;                /* virtual front/back                    */
  int32_t count_;                      /* chunk-based: chunk entries            */
  uint32_t** ring_blocks;              /* standard ring, 2^23 entries, lazily   */
  uint32_t* vq;                        /* VA: virtual index array (16384)      */
  uint32_t front_ptr, back_ptr, old_ptr, old_count;  /* VL                     */
  uint32_t page_size, ppc;
  int inst, q;
} cq_t;

struct orc_heap {
  int variant, page_based, kind;
  uint32_t tid, bid;
  orc_layout lay;
  uint64_t next_free_chunk;
  uint32_t* locator;
  uint64_t locator_words;
  chunk_t* ch;
  uint64_t ch_cap;
  reuse_t reuse[2];
  cq_t cq[2][10];
};

static uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

/* MemoryInitialization.cuh:156-166 and Ouroboros.cuh:80-82,168-170 */
int orc_layout_of(int variant, uint64_t heap_bytes, orc_layout* out) {
  if (variant < 0 || variant > 5 || !out) return ORC_ERR_ARG;
  int kind = variant / 2;
  uint64_t per_queue = kind == KIND_S ? (uint64_t)RING_SIZE * 4u : kind == KIND_VA ? (uint64_t)VQ_SIZE * 4u : 0u;
  uint64_t chunk_q = align_up((uint64_t)REUSE_SIZE * 4u, CHUNK_DATA);
  uint64_t pq = align_up(per_queue, CHUNK_DATA);
  uint64_t mm = chunk_q + pq * 10u + chunk_q + pq * 2u;
  out->object_bytes = OBJECT_BYTES;
  out->queue_bytes = mm;
  out->total_required = align_up(OBJECT_BYTES + mm, CHUNK_STRIDE);
  uint64_t aligned = align_up(heap_bytes, CHUNK_STRIDE);
  if (aligned <= out->total_required) return ORC_ERR_ARG;
  out->max_chunks = (aligned - out->total_required) / CHUNK_STRIDE;
  uint64_t adjacency = align_up(out->max_chunks * CHUNK_STRIDE, 128u);
  out->locator_bytes = align_up((out->max_chunks + 31u) / 32u * 4u, CHUNK_STRIDE);
  out->allocation_bytes = align_up(out->total_required + adjacency + out->locator_bytes, CHUNK_STRIDE);
  return ORC_OK;
}

/* ---------------------------------------------------------------- helpers */

static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

/* Helper.cuh:11-18 getNextPow2Pow (the size is truncated to int by __clz) */
static int next_pow2_pow(uint64_t n) {
  uint32_t v = (uint32_t)n;
  if ((n & (n - 1u)) == 0u) return 32 - clz32(v) - 1;
  return 32 - clz32(v);
}

/* Helper.cuh:42-45 QueueIndex::getQueueIndex */
static int queue_index(int inst, uint64_t size) {
  int q = next_pow2_pow(size) - INST[inst].spf;
  return q < 0 ? 0 : q;
}

static uint32_t rotr32(uint32_t m, uint32_t off) {
  /* ChunkAccess_impl.cuh:103-104: (m >> off) | (m << (32 - off)); a shift by
   * 32 yields 0 on the GPU, so off == 0 leaves m unchanged. */
  return off ? ((m >> off) | (m << (32u - off))) : m;
}

static chunk_t* chunk_at(orc_heap* h, uint64_t c) {
  if (c >= h->ch_cap) return NULL;
  return &h->ch[c];
}

/* ------------------------------------------------------------ reuse queue */

/* queues/Queue_impl.cuh:20-38 IndexQueue::enqueue */
static int reuse_enqueue(reuse_t* r, uint32_t c) {
  int fill = r->count++;
  if (fill < (int)REUSE_SIZE) {
    uint32_t pos = r->back++ % REUSE_SIZE;
    if (r->q[pos] != EMPTY32) return ORC_ERR_HANG;
    r->q[pos] = c;
    return ORC_OK;
  }
  return ORC_OK; /* full: the chunk is silently lost (count_ stays raised) */
}

/* queues/Queue_impl.cuh:54-66 IndexQueue::dequeue */
static int reuse_dequeue(reuse_t* r, uint32_t* c, int* got) {
  int readable = r->count--;
  if (readable <= 0) { r->count++; *got = 0; return ORC_OK; }
  uint32_t pos = r->front++ % REUSE_SIZE;
  if (r->q[pos] == EMPTY32) return ORC_ERR_HANG;
  *c = r->q[pos];
  r->q[pos] = EMPTY32;
  *got = 1;
  return ORC_OK;
}

/* ChunkLocator.cuh:21-24 */
static void locator_set(orc_heap* h, uint64_t c) {
  if ((c >> 5) < h->locator_words) h->locator[c >> 5] |= 1u << (c & 31u);
}

/* ChunkLocator.cuh:29-51 */
static int locator_find(const orc_heap* h, uint64_t c, uint64_t* out) {
  uint64_t index = c >> 5;
  uint32_t bit = (uint32_t)(c & 31u);
  uint32_t mask = bit == 31u ? 0xFFFFFFFFu : ((1u << (bit + 1u)) - 1u);
  if (index >= h->locator_words) return ORC_ERR_UB;
  for (;;) {
    uint32_t w = h->locator[index] & mask;
    int local = 32 - clz32(w);
    if (local) { *out = (index << 5) + (uint64_t)(local - 1); return ORC_OK; }
    if (index == 0) return ORC_ERR_TRAP;
    --index;
    mask = 0xFFFFFFFFu;
  }
}

/* Ouroboros.cuh:108-136 (chunks) and :200-229 (pages): allocateChunk<QUEUECHUNK>.
 * A false return is ignored by every caller in the reference (undefined
 * behaviour); the restatement reports it as ORC_ERR_UB. */
static int allocate_chunk(orc_heap* h, int inst, int queuechunk, uint32_t* c) {
  reuse_t* r = (inst != 0 && queuechunk) ? &h->reuse[0] : &h->reuse[inst];
  int got = 0, rc = reuse_dequeue(r, c, &got);
  if (rc) return rc;
  if (got) return ORC_OK;
  uint64_t add = queuechunk ? 1u : INST[inst].factor;
  uint64_t idx = h->next_free_chunk;
  h->next_free_chunk += add;
  locator_set(h, idx);
  *c = (uint32_t)idx;
  if (!(idx + add < h->lay.max_chunks)) return ORC_ERR_UB;
  return ORC_OK;
}

/* QueueChunk.cuh:217-221 initializeChunk: header reset, storage left as is
 * (fresh chunks were flooded with 0xFFFFFFFF by d_cleanChunks,
 * MemoryInitialization.cuh:21-38; recycled queue chunks drained to the marker). */
static int qc_init(orc_heap* h, uint32_t c, uint32_t vstart) {
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  k->page_size = 0u;
  k->next = NONE_CHUNK;
  k->qcount = 0u;
  k->vstart = vstart;
  if (!k->slots) {
    k->slots = (uint32_t*)malloc(QC_SPOTS * sizeof(uint32_t));
    if (!k->slots) return ORC_ERR_ARG;
    memset(k->slots, 0xFF, QC_SPOTS * sizeof(uint32_t));
  }
  return ORC_OK;
}

/* QueueChunk.cuh:123-127 checkVirtualStart */
static int qc_matches(const chunk_t* k, uint32_t vpos) { return k->vstart / QC_SPOTS == vpos / QC_SPOTS; }

/* ------------------------------------------------------- ChunkAccess */

/* ChunkAccess.cuh:31-89: both constructors give a full mask over number_pages */
static void access_init(chunk_t* k, uint32_t number_pages) {
  k->acc_count = (int32_t)number_pages;
  k->acc_size = number_pages;
  uint32_t n = number_pages;
  for (int i = 0; i < 16; ++i) {
    k->mask[i] = n >= 32u ? 0xFFFFFFFFu : ((1u << n) - 1u);
    n = n > 32u ? n - 32u : 0u;
  }
}

enum { MODE_SUCCESS = 0, MODE_DEQUEUE = 1, MODE_REENQUEUE = 2, MODE_CONTINUE = 3 };
enum { FREE_SUCCESS = 0, FREE_FIRST = 1, FREE_DEQUEUE = 2 };

/* ChunkAccess_impl.cuh:38-135 allocPage, for thread (tid, bid) */
static int access_alloc(const orc_heap* h, chunk_t* k, int words, uint32_t* page, int* mode) {
  int32_t cc = k->acc_count--;
  if (cc <= 0) { k->acc_count++; *mode = MODE_CONTINUE; return ORC_OK; }
  *mode = cc == 1 ? MODE_DEQUEUE : MODE_SUCCESS;
  uint32_t offset = (h->tid + h->bid) % 32u;
  int bitmask_index = (int)h->tid;
  for (int iter = 0; iter < words * 2 + 2; ++iter) {
    ++bitmask_index;
    uint32_t w = (uint32_t)bitmask_index % (uint32_t)words;
    uint32_t m = k->mask[w];
    uint32_t fm = rotr32(m, offset);
    if (fm) {
      uint32_t bit = ((uint32_t)__builtin_ctz(fm) + offset) % 32u;
      *page = 32u * w + bit;
      k->mask[w] = m & ~(1u << bit);
      return ORC_OK;
    }
  }
  return ORC_ERR_HANG;
}

/* ChunkAccess_impl.cuh:7-25 freePage */
static int access_free(chunk_t* k, uint32_t page) {
  k->mask[page / 32u] |= 1u << (page % 32u);
  int32_t cur = ++k->acc_count;
  if (cur == 1) return FREE_FIRST;
  if ((uint32_t)cur == k->acc_size) return FREE_DEQUEUE;
  return FREE_SUCCESS;
}

/* ---------------------------------------------------------- semaphore */

/* BulkSemaphore_impl.cuh:116-217 wait() for a single lane (N = 1). */
typedef int (*chunk_fn)(orc_heap* h, cq_t* q);
static int sem_wait(orc_heap* h, cq_t* q, chunk_fn fn) {
  for (int guard = 0; guard < 64; ++guard) {
    if (q->count - 1 >= 0) { q->count -= 1; return ORC_OK; }
    if (q->count + q->expected - q->reserved < 1) {
      q->expected += q->ppc;
      int rc = fn(h, q);
      if (rc) return rc;
      continue;
    }
    return ORC_ERR_HANG;
  }
  return ORC_ERR_HANG;
}

/* BulkSemaphore_impl.cuh:222-225 signalExpected; returns the old count */
static int64_t sem_signal_expected(cq_t* q, uint32_t n) {
  int64_t old = q->count;
  q->count += n;
  q->expected -= n;
  return old;
}

/* BulkSemaphore_impl.cuh:229-232 signal; returns the old count */
static int64_t sem_signal(cq_t* q, uint32_t n) {
  int64_t old = q->count;
  q->count += n;
  return old;
}

/* BulkSemaphore_impl.cuh:7-17 tryReduce */
static int sem_try_reduce(cq_t* q, int64_t n) {
  if (q->count - n < 0) return 0;
  q->count -= n;
  return 1;
}

/* ------------------------------------------------------- standard ring */

static uint32_t* ring_slot(cq_t* q, uint32_t pos) {
  uint32_t p = pos % RING_SIZE;
  uint32_t b = p >> 16;
  if (!q->ring_blocks[b]) {
    q->ring_blocks[b] = (uint32_t*)malloc(65536u * sizeof(uint32_t));
    if (!q->ring_blocks[b]) return NULL;
    memset(q->ring_blocks[b], 0xFF, 65536u * sizeof(uint32_t));
  }
  return &q->ring_blocks[b][p & 65535u];
}

static uint32_t mem_index(uint32_t chunk, uint32_t page) { return (chunk << 9) + page; }

/* ================================================== page queue: standard */

/* page/PageQueue_impl.cuh:57-79 enqueueChunk */
static int pq_enqueue_chunk(cq_t* q, uint32_t c, uint32_t ppc) {
  if (!(sem_signal_expected(q, ppc) < (int64_t)RING_SIZE)) return ORC_ERR_TRAP;
  uint32_t pos = q->back;
  q->back += ppc;
  for (uint32_t i = 0; i < ppc; ++i) {
    uint32_t* s = ring_slot(q, pos + i);
    if (!s) return ORC_ERR_ARG;
    if (*s != EMPTY32) return ORC_ERR_HANG;
    *s = mem_index(c, i);
  }
  return ORC_OK;
}

/* page/PageQueue_impl.cuh:112-124 (the wait lambda) + PageIndexChunk.cuh:74-78 */
static int pq_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  k->page_size = INST[q->inst].chunk_size / q->ppc;
  k->number_pages = q->ppc;
  return pq_enqueue_chunk(q, c, q->ppc);
}

/* page/PageQueue_impl.cuh:108-133 allocPage */
static int pq_alloc(orc_heap* h, cq_t* q, uint32_t* idx) {
  int rc = sem_wait(h, q, pq_new_chunk);
  if (rc) return rc;
  uint32_t* s = ring_slot(q, q->front++);
  if (!s) return ORC_ERR_ARG;
  if (*s == EMPTY32) return ORC_ERR_HANG;
  *idx = *s;
  *s = EMPTY32;
  return ORC_OK;
}

/* page/PageQueue_impl.cuh:21-36 enqueue, :137-142 freePage */
static int pq_free(orc_heap* h, cq_t* q, uint32_t idx) {
  (void)h;
  if (!(sem_signal(q, 1u) < (int64_t)RING_SIZE)) return ORC_ERR_TRAP;
  uint32_t* s = ring_slot(q, q->back++);
  if (!s) return ORC_ERR_ARG;
  if (*s != EMPTY32) return ORC_ERR_HANG;
  *s = idx;
  return ORC_OK;
}

/* ====================================== virtualized-array queue storage */

/* PageQueueVA_impl.cuh:228-248 / ChunkQueueVA_impl.cuh:310-331 accessQueueElement */
static int va_access(orc_heap* h, cq_t* q, uint32_t chunk_id, uint32_t vpos, chunk_t** out) {
  uint32_t qc = q->vq[chunk_id];
  if (qc == EMPTY32) return ORC_ERR_HANG;
  chunk_t* k = chunk_at(h, qc);
  if (!k) return ORC_ERR_UB;
  if (!qc_matches(k, vpos)) return ORC_ERR_TRAP;
  *out = k;
  return ORC_OK;
}

static uint32_t va_chunk_id(uint32_t vpos) { return (vpos / QC_SPOTS) % VQ_SIZE; }

/* QueueChunk_impl.cuh:87-107 enqueue (array mode); returns the old count_ */
static int qc_enqueue(chunk_t* k, uint32_t position, uint32_t element, uint32_t* old) {
  if (k->slots[position] != EMPTY32) return ORC_ERR_HANG;
  k->slots[position] = element;
  *old = k->qcount;
  k->qcount += (1u << 16) + 1u;
  return ORC_OK;
}

/* QueueChunk.cuh:185-190 checkChunkEmptyEnqueue<N> */
static int qc_empty_after_enqueue(uint32_t old, uint32_t n) { return old + (n << 16) + n == QC_EMPTY_COUNT; }
/* QueueChunk.cuh:194-198 checkChunkEmptyDequeue */
static int qc_empty_after_dequeue(uint32_t old) { return old - (1u << 16) == QC_EMPTY_COUNT; }

/* QueueChunk_impl.cuh:323-345 dequeue (array mode) */
static int qc_dequeue(chunk_t* k, uint32_t position, uint32_t* element, int* empty) {
  if (k->slots[position] == EMPTY32) return ORC_ERR_HANG;
  *element = k->slots[position];
  k->slots[position] = EMPTY32;
  uint32_t old = k->qcount;
  k->qcount -= 1u << 16;
  *empty = qc_empty_after_dequeue(old);
  return ORC_OK;
}

/* QueueChunk_impl.cuh:349-359 deleteElement */
static int qc_delete(chunk_t* k, uint32_t position) {
  k->slots[position] = EMPTY32;
  uint32_t old = k->qcount;
  k->qcount -= 1u << 16;
  return qc_empty_after_dequeue(old);
}

/* Recycle the queue chunk of a drained virtual range (PageQueueVA_impl.cuh:76-83). */
static int va_recycle(orc_heap* h, cq_t* q, uint32_t chunk_id, int base_queue) {
  uint32_t r = q->vq[chunk_id];
  q->vq[chunk_id] = EMPTY32;
  reuse_t* rq = (q->inst != 0 && base_queue) ? &h->reuse[0] : &h->reuse[q->inst];
  return reuse_enqueue(rq, r);
}

/* PageQueueVA_impl.cuh:11-28 / ChunkQueueVA_impl.cuh:12-29 init */
static int va_init(orc_heap* h, cq_t* q) {
  q->vq = (uint32_t*)malloc(VQ_SIZE * sizeof(uint32_t));
  if (!q->vq) return ORC_ERR_ARG;
  memset(q->vq, 0xFF, VQ_SIZE * sizeof(uint32_t));
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 1, &c);
  if (rc) return rc;
  rc = qc_init(h, c, 0u);
  if (rc) return rc;
  q->vq[0] = c;
  return ORC_OK;
}

/* ========================================= page queue: virtualized array */

/* PageQueueVA_impl.cuh:32-90 enqueueChunk */
static int vap_enqueue_chunk(orc_heap* h, cq_t* q, uint32_t c, uint32_t ppc) {
  if (!(sem_signal_expected(q, ppc) < (int64_t)VQ_SIZE * QC_SPOTS)) return ORC_ERR_TRAP;
  uint32_t vpos = q->back;
  q->back += ppc;
  uint32_t chunk_id = va_chunk_id(vpos);
  uint32_t position = vpos % QC_SPOTS;
  int rc;
  if (position + ppc > QC_SPOTS || position == 0u) {
    uint32_t nq;
    rc = allocate_chunk(h, q->inst, 1, &nq);
    if (rc) return rc;
    rc = qc_init(h, nq, vpos + QC_SPOTS + (position != 0u ? QC_SPOTS - position : 0u));
    if (rc) return rc;
    q->vq[(position != 0u ? chunk_id + 2u : chunk_id + 1u) % VQ_SIZE] = nq;
  }
  chunk_t* k;
  rc = va_access(h, q, chunk_id, vpos, &k);
  if (rc) return rc;
  for (uint32_t i = 0; i < ppc; ++i) {
    if (position == 0u) {
      chunk_id = va_chunk_id(vpos);
      rc = va_access(h, q, chunk_id, vpos, &k);
      if (rc) return rc;
    }
    uint32_t old;
    rc = qc_enqueue(k, position, mem_index(c, i), &old);
    if (rc) return rc;
    if (qc_empty_after_enqueue(old, 1u)) {
      rc = va_recycle(h, q, chunk_id, 1);
      if (rc) return rc;
    }
    ++vpos;
    position = vpos % QC_SPOTS;
  }
  return ORC_OK;
}

static int vap_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  k->page_size = INST[q->inst].chunk_size / q->ppc;
  k->number_pages = q->ppc;
  return vap_enqueue_chunk(h, q, c, q->ppc);
}

/* PageQueueVA_impl.cuh:129-171 allocPage */
static int vap_alloc(orc_heap* h, cq_t* q, uint32_t* idx) {
  int rc = sem_wait(h, q, vap_new_chunk);
  if (rc) return rc;
  uint32_t vpos = q->front++;
  uint32_t chunk_id = va_chunk_id(vpos);
  chunk_t* k;
  rc = va_access(h, q, chunk_id, vpos, &k);
  if (rc) return rc;
  int empty;
  rc = qc_dequeue(k, vpos % QC_SPOTS, idx, &empty);
  if (rc) return rc;
  if (empty) return va_recycle(h, q, chunk_id, 1);
  return ORC_OK;
}

/* PageQueueVA_impl.cuh:193-224 enqueue */
static int vap_enqueue(orc_heap* h, cq_t* q, uint32_t idx) {
  uint32_t vpos = q->back++;
  uint32_t chunk_id = va_chunk_id(vpos);
  uint32_t position = vpos % QC_SPOTS;
  int rc;
  if (position == 0u) {
    uint32_t nq;
    rc = allocate_chunk(h, q->inst, 1, &nq);
    if (rc) return rc;
    rc = qc_init(h, nq, vpos + QC_SPOTS);
    if (rc) return rc;
    q->vq[(chunk_id + 1u) % VQ_SIZE] = nq;
  }
  chunk_t* k;
  rc = va_access(h, q, chunk_id, vpos, &k);
  if (rc) return rc;
  uint32_t old;
  rc = qc_enqueue(k, position, idx, &old);
  if (rc) return rc;
  if (qc_empty_after_enqueue(old, 1u)) return va_recycle(h, q, chunk_id, 1);
  return ORC_OK;
}

/* PageQueueVA_impl.cuh:175-189 freePage */
static int vap_free(orc_heap* h, cq_t* q, uint32_t idx) {
  if (!(sem_signal(q, 1u) < (int64_t)VQ_SIZE * QC_SPOTS)) return ORC_ERR_TRAP;
  return vap_enqueue(h, q, idx);
}

/* ============================================ virtualized-linked storage */

/* QueueChunk_impl.cuh:403-426 locateQueueChunkForPosition / the traversal of
 * guaranteeWarpSyncPerChunk (:7-72) for one lane. */
static int vl_locate(orc_heap* h, uint32_t from, uint32_t vpos, chunk_t** out, uint32_t* out_idx) {
  uint32_t cur = from;
  for (uint64_t guard = 0; guard < (1ull << 24); ++guard) {
    chunk_t* k = chunk_at(h, cur);
    if (!k) return ORC_ERR_UB;
    if (qc_matches(k, vpos)) { *out = k; if (out_idx) *out_idx = cur; return ORC_OK; }
    if (k->next == NONE_CHUNK) return ORC_ERR_HANG;
    cur = k->next;
  }
  return ORC_ERR_HANG;
}

/* QueueChunk_impl.cuh:440-463 setBackPointer */
static void vl_set_back(orc_heap* h, cq_t* q, uint32_t cur) {
  while (q->back_ptr == cur) {
    chunk_t* k = chunk_at(h, cur);
    q->back_ptr = k->next;
    chunk_t* nk = chunk_at(h, k->next);
    if (nk && (nk->qcount & 0xFFFFu) == QC_SPOTS) cur = k->next;
    else break;
  }
}

/* QueueChunk_impl.cuh:467-490 setFrontPointer */
static uint32_t vl_set_front(orc_heap* h, cq_t* q, uint32_t cur) {
  uint32_t ret = 0;
  while (q->front_ptr == cur) {
    chunk_t* k = chunk_at(h, cur);
    q->front_ptr = k->next;
    ++ret;
    chunk_t* nk = chunk_at(h, k->next);
    if (nk && nk->qcount == QC_EMPTY_COUNT) cur = k->next;
    else break;
  }
  return ret;
}

/* QueueChunk_impl.cuh:494-551 setOldPointer */
static int vl_set_old(orc_heap* h, cq_t* q, uint32_t free_count) {
  uint32_t cur = q->old_count;
  if (cur < OLD_HOLD) {
    q->old_count += free_count;
    if (cur + free_count > OLD_HOLD) {
      free_count = cur + free_count - OLD_HOLD;
      q->old_count -= free_count;
    } else {
      free_count = 0;
    }
  }
  while (free_count > 0) {
    uint32_t old = q->old_ptr;
    chunk_t* k = chunk_at(h, old);
    if (!k) return ORC_ERR_UB;
    q->old_ptr = k->next;
    --free_count;
    int rc = reuse_enqueue(&h->reuse[0], old);
    if (rc) return rc;
  }
  return ORC_OK;
}

/* The "chunk became empty" tail shared by every linked operation
 * (QueueChunk_impl.cuh:170-182, 252-263, 381-389). */
static int vl_on_empty(orc_heap* h, cq_t* q, uint32_t chunk_idx) {
  uint32_t n = vl_set_front(h, q, chunk_idx);
  return vl_set_old(h, q, n);
}

/* QueueChunk_impl.cuh:137-185 linked enqueue of one element */
static int vl_enqueue(orc_heap* h, cq_t* q, uint32_t vpos, uint32_t element) {
  chunk_t* k;
  uint32_t kidx;
  int rc = vl_locate(h, q->back_ptr, vpos, &k, &kidx);
  if (rc) return rc;
  uint32_t local = vpos % QC_SPOTS;
  if (local == 0u) {
    uint32_t nq;
    rc = allocate_chunk(h, q->inst, 1, &nq);
    if (rc) return rc;
    rc = qc_init(h, nq, vpos + QC_SPOTS);
    if (rc) return rc;
    k = chunk_at(h, kidx);
    k->next = nq;
  }
  k->slots[local] = element;                     /* enqueueLinked: atomicExch */
  uint32_t old = k->qcount;
  k->qcount += (1u << 16) + 1u;
  if ((old & 0xFFFFu) + 1u == QC_SPOTS) vl_set_back(h, q, kidx);
  if (qc_empty_after_enqueue(old, 1u)) return vl_on_empty(h, q, kidx);
  return ORC_OK;
}

/* QueueChunk_impl.cuh:189-319 linked enqueueChunk (SINGLE / V4 modes): ppc
 * entries, pages start .. start + ppc - 1 of chunk c (its start_index) */
static int vl_enqueue_chunk(orc_heap* h, cq_t* q, uint32_t position, uint32_t c, uint32_t ppc, uint32_t start) {
  chunk_t* k;
  uint32_t kidx;
  int rc = vl_locate(h, q->back_ptr, position, &k, &kidx);
  if (rc) return rc;
  uint32_t local = position % QC_SPOTS;
  uint32_t potential_next = NONE_CHUNK;
  if (local == 0u || local + ppc > QC_SPOTS) {
    rc = allocate_chunk(h, q->inst, 1, &potential_next);
    if (rc) return rc;
    uint32_t vs = local == 0u ? position + QC_SPOTS : position + QC_SPOTS + (QC_SPOTS - local);
    rc = qc_init(h, potential_next, vs);
    if (rc) return rc;
    k = chunk_at(h, kidx);
  }
  uint32_t off = 0;
  int v4 = (local % 4u == 0u) && ppc >= 4u;
  while (off < ppc) {
    if (local == 0u) k->next = potential_next;
    uint32_t step = v4 ? 4u : 1u;
    for (uint32_t j = 0; j < step; ++j) k->slots[local + j] = mem_index(c, start + off + j);
    uint32_t old = k->qcount;
    k->qcount += (step << 16) + step;
    if ((old & 0xFFFFu) + step == QC_SPOTS) vl_set_back(h, q, kidx);
    if (qc_empty_after_enqueue(old, step)) {
      rc = vl_on_empty(h, q, kidx);
      if (rc) return rc;
    }
    if (local == (v4 ? QC_SPOTS - 4u : QC_SPOTS - 1u)) {
      if (k->next == NONE_CHUNK) return ORC_ERR_HANG;
      kidx = k->next;
      k = chunk_at(h, kidx);
      if (!k) return ORC_ERR_UB;
      local = 0u;
    } else {
      local += step;
    }
    off += step;
    if (!v4) { if (local % 4u == 0u && ppc - off >= 4u) v4 = 1; }
    else { if (ppc - off < 4u) v4 = 0; }
  }
  return ORC_OK;
}

/* QueueChunk_impl.cuh:365-392 linked dequeue (DEQUEUE or DELETE mode) */
static int vl_dequeue(orc_heap* h, cq_t* q, uint32_t vpos, int delete_mode, uint32_t* element) {
  chunk_t* k;
  uint32_t kidx;
  int rc = vl_locate(h, q->front_ptr, vpos, &k, &kidx);
  if (rc) return rc;
  uint32_t local = vpos % QC_SPOTS;
  int empty;
  if (!delete_mode) {
    rc = qc_dequeue(k, local, element, &empty);
    if (rc) return rc;
  } else {
    empty = qc_delete(k, local);
  }
  if (empty) return vl_on_empty(h, q, kidx);
  return ORC_OK;
}

/* PageQueueVL_impl.cuh:11-30 / ChunkQueueVL_impl.cuh:12-31 init */
static int vl_init(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 1, &c);
  if (rc) return rc;
  rc = qc_init(h, c, 0u);
  if (rc) return rc;
  q->front_ptr = q->back_ptr = q->old_ptr = c;
  return ORC_OK;
}

/* ====================================== page queue: virtualized linked */

/* PageQueueVL_impl.cuh:34-48 enqueueChunk */
static int vlp_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  k->page_size = INST[q->inst].chunk_size / q->ppc;
  k->number_pages = q->ppc;
  uint32_t vpos = q->back;
  q->back += q->ppc;
  rc = vl_enqueue_chunk(h, q, vpos, c, q->ppc, 0u);
  if (rc) return rc;
  sem_signal_expected(q, q->ppc);
  return ORC_OK;
}

/* PageQueueVL_impl.cuh:67-98 allocPage */
static int vlp_alloc(orc_heap* h, cq_t* q, uint32_t* idx) {
  int rc = sem_wait(h, q, vlp_new_chunk);
  if (rc) return rc;
  uint32_t vpos = q->front++;
  return vl_dequeue(h, q, vpos, 0, idx);
}

/* PageQueueVL_impl.cuh:102-122 freePage / enqueue */
static int vlp_free(orc_heap* h, cq_t* q, uint32_t idx) {
  uint32_t vpos = q->back++;
  int rc = vl_enqueue(h, q, vpos, idx);
  if (rc) return rc;
  sem_signal(q, 1u);
  return ORC_OK;
}

/* ================================================ chunk-based queues */

/* ChunkIndexChunk.cuh:70-84 initializeChunk / initializeEmptyChunk */
static int cidx_init(orc_heap* h, cq_t* q, uint32_t c, chunk_t** out) {
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  k->page_size = INST[q->inst].chunk_size / q->ppc;
  access_init(k, q->ppc);
  k->queue_pos = EMPTY32;
  *out = k;
  return ORC_OK;
}

/* chunk/ChunkQueue_impl.cuh:22-54 enqueue */
static int cq_enqueue(cq_t* q, uint32_t c, chunk_t* k) {
  int fill = q->count_++;
  if (!(fill < (int)RING_SIZE)) return ORC_ERR_TRAP;
  uint32_t pos = q->back++ % RING_SIZE;
  uint32_t* s = ring_slot(q, pos);
  if (!s) return ORC_ERR_ARG;
  if (*s != EMPTY32) return ORC_ERR_HANG;
  *s = c;
  if (k) k->queue_pos = pos;
  return ORC_OK;
}

/* chunk/ChunkQueue_impl.cuh:86-100 (the wait lambda) + :58-66 enqueueChunk */
static int cq_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k;
  rc = cidx_init(h, q, c, &k);
  if (rc) return rc;
  rc = cq_enqueue(q, c, k);
  if (rc) return rc;
  sem_signal_expected(q, q->ppc);
  return ORC_OK;
}

/* chunk/ChunkQueue_impl.cuh:82-148 allocPage */
static int cq_alloc(orc_heap* h, cq_t* q, uint32_t* out_c, uint32_t* out_p) {
  int rc = sem_wait(h, q, cq_new_chunk);
  if (rc) return rc;
  uint32_t cur = q->front;
  for (uint64_t guard = 0; guard < (uint64_t)RING_SIZE + 1u; ++guard, ++cur) {
    uint32_t* s = ring_slot(q, cur);
    if (!s) return ORC_ERR_ARG;
    uint32_t c = *s;
    if (c == EMPTY32) continue;
    chunk_t* k = chunk_at(h, c);
    if (!k) return ORC_ERR_UB;
    uint32_t page;
    int mode;
    rc = access_alloc(h, k, INST[q->inst].words, &page, &mode);
    if (rc) return rc;
    if (mode == MODE_CONTINUE) continue;
    if (mode == MODE_DEQUEUE) {
      if (q->front < cur + 1u) q->front = cur + 1u;
      k->queue_pos = EMPTY32;
      *s = EMPTY32;
      q->count_--;
    }
    *out_c = c;
    *out_p = page;
    return ORC_OK;
  }
  return ORC_ERR_HANG;
}

/* chunk/ChunkQueue_impl.cuh:152-205 freePage */
static int cq_free(orc_heap* h, cq_t* q, uint32_t c, uint32_t page) {
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  int mode = access_free(k, page);
  if (mode == FREE_FIRST) {
    int rc = cq_enqueue(q, c, k);
    if (rc) return rc;
  } else if (mode == FREE_DEQUEUE && q->count_ > C_LOWER_FILL) {
    uint32_t n = k->acc_size;
    if (sem_try_reduce(q, (int64_t)n - 1)) {
      if (k->acc_count == (int32_t)k->acc_size) {      /* tryFlashChunk */
        k->acc_count = 0;
        if (k->queue_pos == EMPTY32) return ORC_ERR_HANG;
        uint32_t* s = ring_slot(q, k->queue_pos);
        if (!s) return ORC_ERR_ARG;
        *s = EMPTY32;
        q->count_--;
        return reuse_enqueue(&h->reuse[q->inst], c);
      }
      sem_signal(q, n);
      return ORC_OK;
    }
  }
  sem_signal(q, 1u);
  return ORC_OK;
}

/* chunk/ChunkQueueVA_impl.cuh:274-306 enqueue */
static int vac_enqueue(orc_heap* h, cq_t* q, uint32_t idx, chunk_t* kc) {
  uint32_t vpos = q->back++;
  uint32_t chunk_id = va_chunk_id(vpos);
  uint32_t position = vpos % QC_SPOTS;
  int rc;
  if (position == 0u) {
    uint32_t nq;
    rc = allocate_chunk(h, q->inst, 1, &nq);
    if (rc) return rc;
    rc = qc_init(h, nq, vpos + QC_SPOTS);
    if (rc) return rc;
    q->vq[(chunk_id + 1u) % VQ_SIZE] = nq;
  }
  chunk_t* k;
  rc = va_access(h, q, chunk_id, vpos, &k);
  if (rc) return rc;
  if (kc) kc->queue_pos = vpos;
  uint32_t old;
  rc = qc_enqueue(k, position, idx, &old);
  if (rc) return rc;
  if (qc_empty_after_enqueue(old, 1u)) return va_recycle(h, q, chunk_id, 1);
  return ORC_OK;
}

/* chunk/ChunkQueueVA_impl.cuh:33-50 enqueueChunk + the wait lambda :88-98 */
static int vac_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k;
  rc = cidx_init(h, q, c, &k);
  if (rc) return rc;
  if (!(q->count_++ < (int)(VQ_SIZE * QC_SPOTS))) return ORC_ERR_TRAP;
  rc = vac_enqueue(h, q, c, k);
  if (rc) return rc;
  sem_signal_expected(q, q->ppc);
  return ORC_OK;
}

/* chunk/ChunkQueueVA_impl.cuh:76-192 allocPage */
static int vac_alloc(orc_heap* h, cq_t* q, uint32_t* out_c, uint32_t* out_p) {
  int rc = sem_wait(h, q, vac_new_chunk);
  if (rc) return rc;
  uint32_t vpos = q->front;
  for (uint64_t guard = 0; guard < (1ull << 26); ++guard, ++vpos) {
    uint32_t chunk_id = va_chunk_id(vpos);
    uint32_t qci = q->vq[chunk_id];
    if (qci == EMPTY32) continue;
    chunk_t* qk = chunk_at(h, qci);
    if (!qk) return ORC_ERR_UB;
    if (!qc_matches(qk, vpos)) return ORC_ERR_TRAP;
    uint32_t c = qk->slots[vpos % QC_SPOTS];
    if (c == EMPTY32) continue;
    chunk_t* k = chunk_at(h, c);
    if (!k) return ORC_ERR_UB;
    uint32_t page;
    int mode;
    rc = access_alloc(h, k, INST[q->inst].words, &page, &mode);
    if (rc) return rc;
    if (mode == MODE_CONTINUE) continue;
    if (mode == MODE_DEQUEUE) {
      if (q->front < vpos + 1u) q->front = vpos + 1u;
      if (qc_delete(qk, vpos % QC_SPOTS)) {
        uint32_t r = q->vq[chunk_id];
        q->vq[chunk_id] = EMPTY32;
        memset(qk->slots, 0xFF, QC_SPOTS * sizeof(uint32_t));   /* cleanChunk */
        rc = reuse_enqueue(&h->reuse[q->inst], r);              /* enqueueChunkForReuse<false> */
        if (rc) return rc;
      }
      q->count_--;
    }
    *out_c = c;
    *out_p = page;
    return ORC_OK;
  }
  return ORC_ERR_HANG;
}

/* chunk/ChunkQueueVA_impl.cuh:196-270 freePage */
static int vac_free(orc_heap* h, cq_t* q, uint32_t c, uint32_t page) {
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  int mode = access_free(k, page);
  if (mode == FREE_FIRST) {
    if (!(q->count_++ < (int)(VQ_SIZE * QC_SPOTS))) return ORC_ERR_TRAP;
    int rc = vac_enqueue(h, q, c, k);
    if (rc) return rc;
  } else if (mode == FREE_DEQUEUE) {
    uint32_t n = k->acc_size;
    if (sem_try_reduce(q, (int64_t)n - 1)) {
      sem_signal(q, n);        /* the flash branch is disabled (:229) */
      return ORC_OK;
    }
  }
  sem_signal(q, 1u);
  return ORC_OK;
}

/* chunk/ChunkQueueVL_impl.cuh:202-208 enqueue */
static int vlc_enqueue(orc_heap* h, cq_t* q, uint32_t c) {
  uint32_t vpos = q->back++;
  return vl_enqueue(h, q, vpos, c);
}

/* chunk/ChunkQueueVL_impl.cuh:35-46 enqueueChunk + the wait lambda :71-81 */
static int vlc_new_chunk(orc_heap* h, cq_t* q) {
  uint32_t c;
  int rc = allocate_chunk(h, q->inst, 0, &c);
  if (rc) return rc;
  chunk_t* k;
  rc = cidx_init(h, q, c, &k);
  if (rc) return rc;
  rc = vlc_enqueue(h, q, c);
  if (rc) return rc;
  sem_signal_expected(q, q->ppc);
  return ORC_OK;
}

/* chunk/ChunkQueueVL_impl.cuh:62-142 allocPage */
static int vlc_alloc(orc_heap* h, cq_t* q, uint32_t* out_c, uint32_t* out_p) {
  int rc = sem_wait(h, q, vlc_new_chunk);
  if (rc) return rc;
  uint32_t vpos = q->front;
  uint32_t qidx = q->front_ptr;
  for (uint64_t guard = 0; guard < (1ull << 26); ++guard, ++vpos) {
    chunk_t* qk;
    rc = vl_locate(h, qidx, vpos, &qk, &qidx);
    if (rc) return rc;
    uint32_t c = qk->slots[vpos % QC_SPOTS];
    if (c == EMPTY32) continue;
    chunk_t* k = chunk_at(h, c);
    if (!k) return ORC_ERR_UB;
    uint32_t page;
    int mode;
    rc = access_alloc(h, k, INST[q->inst].words, &page, &mode);
    if (rc) return rc;
    if (mode == MODE_CONTINUE) continue;
    if (mode == MODE_DEQUEUE) {
      if (q->front < vpos + 1u) q->front = vpos + 1u;
      uint32_t dummy;
      rc = vl_dequeue(h, q, vpos, 1, &dummy);
      if (rc) return rc;
    }
    *out_c = c;
    *out_p = page;
    return ORC_OK;
  }
  return ORC_ERR_HANG;
}

/* chunk/ChunkQueueVL_impl.cuh:146-198 freePage */
static int vlc_free(orc_heap* h, cq_t* q, uint32_t c, uint32_t page) {
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  int mode = access_free(k, page);
  if (mode == FREE_FIRST) {
    int rc = vlc_enqueue(h, q, c);
    if (rc) return rc;
  }
  sem_signal(q, 1u);
  return ORC_OK;
}

/* ================================================= public interface */

static void free_heap(orc_heap* h) {
  if (!h) return;
  if (h->ch) {
    for (uint64_t i = 0; i < h->ch_cap; ++i) free(h->ch[i].slots);
    free(h->ch);
  }
  for (int i = 0; i < 2; ++i) {
    free(h->reuse[i].q);
    for (int q = 0; q < 10; ++q) {
      cq_t* c = &h->cq[i][q];
      if (c->ring_blocks) {
        for (uint32_t b = 0; b < RING_SIZE / 65536u; ++b) free(c->ring_blocks[b]);
        free(c->ring_blocks);
      }
      free(c->vq);
    }
  }
  free(h->locator);
  free(h);
}

/* MemoryInitialization.cuh:123-219 initialize + :91-119 queue init */
orc_heap* orc_create(int variant, uint64_t heap_bytes, uint32_t tid, uint32_t bid) {
  orc_heap* h = (orc_heap*)calloc(1, sizeof(orc_heap));
  if (!h) return NULL;
  if (orc_layout_of(variant, heap_bytes, &h->lay)) { free(h); return NULL; }
  h->variant = variant;
  h->kind = variant / 2;
  h->page_based = (variant % 2) == 0;
  h->tid = tid;
  h->bid = bid;
  h->locator_words = (h->lay.max_chunks + 31u) / 32u;
  h->locator = (uint32_t*)calloc(h->locator_words ? h->locator_words : 1u, sizeof(uint32_t));
  h->ch_cap = h->lay.max_chunks + 8u;
  h->ch = (chunk_t*)calloc(h->ch_cap, sizeof(chunk_t));
  if (!h->locator || !h->ch) { free_heap(h); return NULL; }
  for (int i = 0; i < 2; ++i) {
    h->reuse[i].q = (uint32_t*)malloc(REUSE_SIZE * sizeof(uint32_t));
    if (!h->reuse[i].q) { free_heap(h); return NULL; }
    memset(h->reuse[i].q, 0xFF, REUSE_SIZE * sizeof(uint32_t));
  }
  /* Ouroboros<...>::initQueues (MemoryInitialization.cuh:102-119): instance 0
   * queues 0..9, then instance 1 queues 0..1, each init in order. */
  for (int i = 0; i < 2; ++i) {
    for (int q = 0; q < INST[i].nq; ++q) {
      cq_t* c = &h->cq[i][q];
      c->inst = i;
      c->q = q;
      c->page_size = INST[i].smallest << q;
      c->ppc = (INST[i].chunk_size / INST[i].smallest) >> q;
      int rc = ORC_OK;
      if (h->kind == KIND_S) {
        c->ring_blocks = (uint32_t**)calloc(RING_SIZE / 65536u, sizeof(uint32_t*));
        if (!c->ring_blocks) rc = ORC_ERR_ARG;
      } else if (h->kind == KIND_VA) {
        rc = va_init(h, c);
      } else {
        rc = vl_init(h, c);
      }
      if (rc) { free_heap(h); return NULL; }
    }
  }
  return h;
}

void orc_destroy(orc_heap* h) { free_heap(h); }

uint64_t orc_next_free_chunk(const orc_heap* h) { return h ? h->next_free_chunk : 0u; }

static int64_t ref_offset(uint32_t c, uint32_t p, uint32_t page_size) {
  return (int64_t)c * CHUNK_STRIDE + CHUNK_META + (int64_t)p * page_size;
}

/* Ouroboros_impl.cuh:83-91 malloc -> :17-26 / :50-59 allocPage */
int orc_malloc(orc_heap* h, uint64_t size, uint64_t* res, int64_t* ref_off) {
  if (!h || !res || !ref_off) return ORC_ERR_ARG;
  int inst;
  if (size <= INST[0].smallest << (INST[0].nq - 1)) inst = 0;
  else if (size <= INST[1].smallest << (INST[1].nq - 1)) inst = 1;
  else { *res = ORC_RES_DEVHEAP; *ref_off = -2; return ORC_OK; }  /* Ouroboros.cuh:401-408 */
  int qi = queue_index(inst, size);
  cq_t* q = &h->cq[inst][qi];
  uint32_t c = 0, p = 0, idx = 0;
  int rc;
  switch (h->variant) {
    case ORC_P: rc = pq_alloc(h, q, &idx); c = idx >> 9; p = idx & 511u; break;
    case ORC_VAP: rc = vap_alloc(h, q, &idx); c = idx >> 9; p = idx & 511u; break;
    case ORC_VLP: rc = vlp_alloc(h, q, &idx); c = idx >> 9; p = idx & 511u; break;
    case ORC_C: rc = cq_alloc(h, q, &c, &p); break;
    case ORC_VAC: rc = vac_alloc(h, q, &c, &p); break;
    default: rc = vlc_alloc(h, q, &c, &p); break;
  }
  if (rc) return rc;
  *res = ((uint64_t)(inst * 16 + qi) << 32) | (uint64_t)mem_index(c, p);
  *ref_off = ref_offset(c, p, q->page_size);
  return ORC_OK;
}

/* Ouroboros_impl.cuh:95-125 free, restated on the reference layout */
int orc_free(orc_heap* h, uint64_t res) {
  if (!h) return ORC_ERR_ARG;
  if (res & ORC_RES_FAIL) return ORC_OK;
  if (res & ORC_RES_DEVHEAP) return ORC_OK;                      /* ::free */
  uint32_t cls = (uint32_t)(res >> 32) & 0xFFu;
  int inst = (int)(cls / 16u);
  int qi = (int)(cls % 16u);
  if (inst > 1 || qi >= INST[inst].nq) return ORC_ERR_ARG;
  uint32_t idx = (uint32_t)res;
  uint32_t page_size = INST[inst].smallest << qi;
  int64_t off = ref_offset(idx >> 9, idx & 511u, page_size);
  if (!((uint64_t)off + OBJECT_BYTES < h->lay.allocation_bytes)) return ORC_ERR_ARG;
  uint64_t base = (uint64_t)off / CHUNK_STRIDE;                  /* Chunk.cuh:52-56 */
  uint64_t c;
  int rc = locator_find(h, base, &c);
  if (rc) return rc;
  chunk_t* k = chunk_at(h, c);
  if (!k || k->page_size == 0u) return ORC_ERR_UB;
  uint32_t page = (uint32_t)(((uint64_t)off - c * CHUNK_STRIDE - CHUNK_META) / k->page_size);
  /* freePageRecursive: page size picks the instance, the header the queue */
  int finst = k->page_size <= (INST[0].smallest << (INST[0].nq - 1)) ? 0 : 1;
  int fq = queue_index(finst, k->page_size);
  cq_t* q = &h->cq[finst][fq];
  uint32_t mi = mem_index((uint32_t)c, page);
  switch (h->variant) {
    case ORC_P: return pq_free(h, q, mi);
    case ORC_VAP: return vap_free(h, q, mi);
    case ORC_VLP: return vlp_free(h, q, mi);
    case ORC_C: return cq_free(h, q, (uint32_t)c, page);
    case ORC_VAC: return vac_free(h, q, (uint32_t)c, page);
    default: return vlc_free(h, q, (uint32_t)c, page);
  }
}

/* Ouroboros.cuh:108-136 allocateChunk<false> of the first instance: the call a
 * caller of enqueueInitialChunk makes first. */
int orc_allocate_chunk(orc_heap* h, uint32_t* chunk) {
  if (!h || !chunk) return ORC_ERR_ARG;
  return allocate_chunk(h, 0, 0, chunk);
}

/* ChunkAccess.cuh:31-64: count = available pages, mask over number_pages with
 * the first number_pages - available pages taken */
static void access_init_avail(chunk_t* k, uint32_t available, uint32_t number_pages) {
  k->acc_count = (int32_t)available;
  k->acc_size = number_pages;
  uint32_t taken = number_pages - available, n = number_pages;
  for (int i = 0; i < 16; ++i) {
    if (taken >= 32u) {
      k->mask[i] = 0u;
      taken -= 32u;
    } else {
      k->mask[i] = n >= 32u ? ~((1u << taken) - 1u) : (~((1u << taken) - 1u) & ((1u << n) - 1u));
      taken = 0u;
    }
    n = n > 32u ? n - 32u : 0u;
  }
}

/* Ouroboros.cuh:291-295 enqueueInitialChunk, after the chunk initializer its
 * callers run (PageIndexChunk.cuh:82-86 / ChunkIndexChunk.cuh:73-78). */
int orc_enqueue_initial(orc_heap* h, uint32_t queue_index, uint32_t c, uint32_t available) {
  if (!h || queue_index >= (uint32_t)INST[0].nq) return ORC_ERR_ARG;
  cq_t* q = &h->cq[0][queue_index];
  if (available == 0u || available > q->ppc) return ORC_ERR_ARG;
  chunk_t* k = chunk_at(h, c);
  if (!k) return ORC_ERR_UB;
  const uint32_t start = q->ppc - available;
  k->page_size = INST[0].chunk_size / q->ppc;
  int rc = ORC_OK;
  if (h->page_based) {
    k->number_pages = q->ppc;
    if (h->kind == KIND_S) {
      /* PageQueue_impl.cuh:40-53 */
      for (uint32_t i = start; i < q->ppc; ++i) {
        uint32_t* s = ring_slot(q, q->back++);
        if (!s) return ORC_ERR_ARG;
        *s = mem_index(c, i);
      }
    } else if (h->kind == KIND_VA) {
      /* PageQueueVA_impl.cuh:94-125 */
      for (uint32_t i = start; i < q->ppc; ++i) {
        uint32_t vpos = q->back++;
        uint32_t chunk_id = va_chunk_id(vpos);
        if (vpos % QC_SPOTS == 0u) {
          uint32_t nq;
          rc = allocate_chunk(h, q->inst, 1, &nq);
          if (rc) return rc;
          rc = qc_init(h, nq, vpos + QC_SPOTS);
          if (rc) return rc;
          q->vq[(chunk_id + 1u) % VQ_SIZE] = nq;
        }
        chunk_t* qk;
        rc = va_access(h, q, chunk_id, vpos, &qk);
        if (rc) return rc;
        qk->slots[vpos % QC_SPOTS] = mem_index(c, i);   /* QueueChunk_impl.cuh:77-83 enqueueInitial */
        qk->qcount += (1u << 16) + 1u;
      }
    } else {
      /* PageQueueVL_impl.cuh:54-63 */
      uint32_t vpos = q->back;
      q->back += available;
      rc = vl_enqueue_chunk(h, q, vpos, c, available, start);
      if (rc) return rc;
    }
  } else {
    access_init_avail(k, available, q->ppc);
    k->queue_pos = EMPTY32;
    if (h->kind == KIND_S) {
      /* ChunkQueue_impl.cuh:69-77: count_ is set, not raised */
      q->count_ = 1;
      uint32_t* s = ring_slot(q, q->back++);
      if (!s) return ORC_ERR_ARG;
      *s = c;
    } else if (h->kind == KIND_VA) {
      /* ChunkQueueVA_impl.cuh:54-72: the first entry of the first queue chunk,
       * then the second queue chunk; defined only on a fresh queue */
      if (q->back != 0u) return ORC_ERR_UB;
      ++q->count_;
      ++q->back;
      chunk_t* qk;
      rc = va_access(h, q, 0u, 0u, &qk);
      if (rc) return rc;
      qk->slots[0] = c;
      qk->qcount += (1u << 16) + 1u;
      uint32_t nq;
      rc = allocate_chunk(h, q->inst, 1, &nq);
      if (rc) return rc;
      rc = qc_init(h, nq, QC_SPOTS);
      if (rc) return rc;
      q->vq[1] = nq;
    } else {
      /* ChunkQueueVL_impl.cuh:49-56 */
      rc = vlc_enqueue(h, q, c);
      if (rc) return rc;
    }
  }
  sem_signal(q, available);
  return ORC_OK;
}

/* The encoded result of page `page` of chunk c, for a free of a page that a
 * caller held from an initial chunk. */
static int page_result(orc_heap* h, uint32_t c, uint32_t page, uint64_t* res) {
  chunk_t* k = chunk_at(h, c);
  if (!k || k->page_size == 0u) return ORC_ERR_ARG;
  int inst = k->page_size <= (INST[0].smallest << (INST[0].nq - 1)) ? 0 : 1;
  int qi = queue_index(inst, k->page_size);
  *res = ((uint64_t)(inst * 16 + qi) << 32) | (uint64_t)mem_index(c, page);
  return ORC_OK;
}

int orc_run_trace(orc_heap* h, const uint32_t* ops, uint64_t n_ops, uint64_t* res, int64_t* ref_off,
                  uint64_t* failed_at) {
  if (!h || !ops || !res || !ref_off) return ORC_ERR_ARG;
  for (uint64_t i = 0; i < n_ops; ++i) {
    int rc;
    const uint32_t op = ops[2 * i], arg = ops[2 * i + 1];
    res[i] = 0;
    ref_off[i] = 0;
    if (op == 0u) {
      rc = orc_malloc(h, arg, &res[i], &ref_off[i]);
    } else if (op == 1u) {
      if (arg >= i || ops[2 * arg] != 0u) rc = ORC_ERR_ARG;
      else rc = orc_free(h, res[arg]);
    } else if (op == 2u) {
      uint32_t c = 0;
      rc = orc_allocate_chunk(h, &c);
      res[i] = c;
      ref_off[i] = c;
    } else if (op == 3u || op == 4u) {
      uint64_t j = op == 3u ? (arg >> 14) : (arg >> 10);
      if (j >= i || ops[2 * j] != 2u) {
        rc = ORC_ERR_ARG;
      } else if (op == 3u) {
        rc = orc_enqueue_initial(h, arg & 15u, (uint32_t)res[j], (arg >> 4) & 1023u);
      } else {
        uint64_t r = 0;
        rc = page_result(h, (uint32_t)res[j], arg & 1023u, &r);
        if (!rc) rc = orc_free(h, r);
      }
    } else {
      rc = ORC_ERR_ARG;
    }
    if (rc) { if (failed_at) *failed_at = i; return rc; }
  }
  return ORC_OK;
}

int orc_state(const orc_heap* h, uint64_t* out) {
  if (!h || !out) return ORC_ERR_ARG;
  memset(out, 0, ORC_STATE_WORDS * sizeof(uint64_t));
  out[0] = h->next_free_chunk;
  for (int i = 0; i < 2; ++i) {
    out[1 + 3 * i] = (uint64_t)(int64_t)h->reuse[i].count;
    out[2 + 3 * i] = h->reuse[i].front;
    out[3 + 3 * i] = h->reuse[i].back;
  }
  int cls = 0;
  for (int i = 0; i < 2; ++i) {
    for (int qi = 0; qi < INST[i].nq; ++qi, ++cls) {
      const cq_t* q = &h->cq[i][qi];
      uint64_t* o = out + 7 + 12 * cls;
      o[0] = (uint64_t)q->count;
      o[1] = (uint64_t)q->expected;
      o[2] = (uint64_t)q->reserved;
      o[3] = q->front;
      o[4] = q->back;
      o[5] = h->page_based ? 0u : (uint64_t)(int64_t)q->count_;
      if (h->kind == KIND_VL) {
        o[6] = q->front_ptr;
        o[7] = q->back_ptr;
        o[8] = q->old_ptr;
        o[9] = q->old_count;
      }
      if (h->kind == KIND_VA) {
        uint64_t d = 0;
        for (uint32_t v = 0; v < VQ_SIZE; ++v)
          if (q->vq[v] != EMPTY32) d += (uint64_t)(v + 1u) * ((uint64_t)q->vq[v] + 1u);
        o[10] = d;
      }
      o[11] = q->ppc;
    }
  }
  return ORC_OK;
}
