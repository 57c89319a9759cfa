/*
 * ouroboros_b200.h -- C ABI of the B200 Ouroboros allocator.
 *
 * The device-side interface (what kernels call) is the header-only template
 * ouro::Ouroboros<V> in ouroboros_b200/csrc/ouro/ouroboros.cuh, reached from
 * C++/CUDA through include/ouroboros_b200.cuh.  This header is the host side:
 * plain pointers, sizes and status codes, no CUDA or torch types.  Device
 * buffers are passed as pointers to device memory; `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).
 *
 * Each entry point names the reference interface it replaces (paths in the
 * reference project GPUPeople/Ouroboros).
 */
#ifndef OUROBOROS_B200_H
#define OUROBOROS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The six instantiations of include/InstanceDefinitions.cuh:16-34 (the Multi*
 * types: 16 B .. 8 KiB pages in 8 KiB chunks plus 16/32 KiB pages in 32 KiB
 * chunks; larger requests go to the CUDA device heap). */
typedef enum {
  OURO_P = 0,   /* MultiOuroPQ   page-based, standard array queues            */
  OURO_C = 1,   /* MultiOuroCQ   chunk-based, standard array queues           */
  OURO_VAP = 2, /* MultiOuroVAPQ page-based, virtualized array queues         */
  OURO_VAC = 3, /* MultiOuroVACQ chunk-based, virtualized array queues        */
  OURO_VLP = 4, /* MultiOuroVLPQ page-based, virtualized linked-list queues   */
  OURO_VLC = 5  /* MultiOuroVLCQ chunk-based, virtualized linked-list queues  */
} ouro_variant;

/* Host-side status codes.  The reference exits the process on a CUDA error
 * (include/Utility.h:10-36, HANDLE_ERROR); these return instead. */
typedef enum {
  OURO_OK = 0,
  OURO_ERR_ARG = 1,      /* bad argument                                  */
  OURO_ERR_CUDA = 2,     /* a CUDA runtime call failed                    */
  OURO_ERR_NOMEM = 3,    /* cudaMalloc of the heap failed                 */
  OURO_ERR_DEVICE = 4,   /* the device reported an allocator error flag   */
  OURO_ERR_TOO_LARGE = 5, /* beyond the fixed scratch of a no-alloc entry */
  OURO_ERR_FULL = 6       /* the serving loop's submission ring is full    */
} ouro_status;

/* Device-side error flags (ouro_heap_status.flags). */
#define OURO_FLAG_OOM 1u        /* some malloc returned nullptr (heap exhausted)    */
#define OURO_FLAG_TIMEOUT 2u    /* a bounded wait gave up; the heap needs a reset   */
#define OURO_FLAG_CORRUPT 4u    /* a structural check failed                        */
#define OURO_FLAG_QUEUE_FULL 8u /* a size class reached its queue capacity          */

typedef struct ouro_heap ouro_heap;

/* Ouroboros<...>::initialize(instantiation_size)  (include/device/Ouroboros.cuh:281,
 * include/device/MemoryInitialization.cuh:123-219).  Allocates and initializes a
 * heap of `heap_bytes` on the current device; the number of usable 8 KiB chunks
 * is the reference's for the same size.  Synchronous. */
int ouro_create(int variant, uint64_t heap_bytes, ouro_heap** out);

/* Run-time allocator parameters.  The reference fixes all of them at compile
 * time (include/Parameters.h:9-18); ouro_config_default fills in its values,
 * and ouro_create is ouro_create_config with them.
 *   chunk_bytes            CHUNK_SIZE (Parameters.h:17, 16 B << 9 = 8192).  Only
 *                          8192 is accepted: the 9 page bits of a queue entry
 *                          (MemoryIndex.cuh:6-51) and the 512-bit occupancy
 *                          mask of a chunk are sized for 8 KiB / 16 B.
 *   page_queue_entries     page_queue_size (Parameters.h:11, 2^23): ring entries
 *                          per size class of the standard queues (P, C); a power
 *                          of two in [2^16, 2^23].
 *   virtual_queue_entries  virtual_queue_size (Parameters.h:12, 16384): entries of
 *                          the per-class index of queue chunks of the virtualized-
 *                          array queues (VAP, VAC), each queue chunk holding 2048
 *                          queue entries; a power of two in [32, 16384].
 *   agg_width              lanes whose requests of one size class are aggregated
 *                          into one group (one semaphore and one queue atomic per
 *                          group): 1, 2, 4, 8, 16 or 32.  The reference
 *                          aggregates over the whole warp (__match_any_sync over
 *                          __activemask(), BulkSemaphore_impl.cuh:124-127): 32.
 * The number of usable chunks follows the reference's capacity formula
 * (MemoryInitialization.cuh:156-166) on the configured queue sizes, so with
 * the defaults it is the reference's.  The linked-list variants have no queue
 * arrays; the two queue sizes do not apply to them. */
typedef struct {
  uint32_t chunk_bytes;
  uint32_t page_queue_entries;
  uint32_t virtual_queue_entries;
  uint32_t agg_width;
} ouro_config;

int ouro_config_default(ouro_config* out);
/* ouro_create with explicit parameters (cfg NULL = the defaults). */
int ouro_create_config(int variant, uint64_t heap_bytes, const ouro_config* cfg, ouro_heap** out);
/* The parameters a heap was created with. */
int ouro_get_config(const ouro_heap* h, ouro_config* out);

/* Memory::~Memory  (include/device/Ouroboros.cuh:11-15): frees the heap. */
int ouro_destroy(ouro_heap* h);

/* Ouroboros<...>::getDeviceMemoryManager()  (include/device/Ouroboros.cuh:297):
 * the device pointer kernels call malloc/free on (an ouro::Ouroboros<V>*). */
void* ouro_device_handle(const ouro_heap* h);

typedef struct {
  int32_t variant;
  uint64_t heap_bytes;
  uint64_t max_chunks;   /* Memory::maxChunks (MemoryInitialization.cuh:161) */
  uint64_t alloc_bytes;  /* device bytes held                                 */
  uint64_t data_base;    /* device address of chunk 0's data (8 KiB aligned)  */
  uint64_t data_end;
} ouro_heap_info;
int ouro_get_info(const ouro_heap* h, ouro_heap_info* out);

/* The per-thread drop-in path, one launch of n threads (src/main.cu:10-18
 * d_testAllocation): thread i stores malloc(size) -- or malloc(d_sizes[i]) when
 * d_sizes is not NULL -- into d_out[i]; nullptr when out of memory. */
int ouro_alloc(ouro_heap* h, uint32_t n, uint32_t size, const uint32_t* d_sizes, void** d_out, int block,
               void* stream);

/* src/main.cu:55-63 d_testFree: thread i frees d_ptrs[i] (nullptr is a no-op). */
int ouro_free(ouro_heap* h, uint32_t n, void* const* d_ptrs, int block, void* stream);

/* ouro_alloc / ouro_free for requests held in HOST memory (no counterpart in
 * the reference, whose callers are device code: this is the entry point for a
 * host-side caller).  ouro_alloc_host: request i is malloc(size), or
 * malloc(h_sizes[i]) when h_sizes is not NULL; its pointer goes to h_out[i]
 * and, when d_out is not NULL, to d_out[i] (device) too.  ouro_free_host:
 * frees h_ptrs[i].  The requests are cut into `slices` pieces (0: 1 to 4 by
 * n, at least 2^17 requests each; at most 8) whose host<->device copies, on
 * two streams of the heap's own, overlap the launches of the other pieces.
 * The work is ordered after what `stream` holds at the call and after the
 * previous host-buffer call on this heap, and it ends on `stream`:
 * synchronise `stream` before reading h_out or reusing the host buffers.
 * Pinned host memory makes the copies asynchronous; pageable memory works,
 * with copies that do not overlap.  Calls on one heap from several host
 * threads take turns. */
int ouro_alloc_host(ouro_heap* h, uint32_t n, uint32_t size, const uint32_t* h_sizes, void** h_out, void** d_out,
                    int block, int slices, void* stream);
int ouro_free_host(ouro_heap* h, uint32_t n, void* const* h_ptrs, int block, int slices, void* stream);
/* Makes the host-buffer calls' streams, events and device staging for batches
 * of up to n requests now, so that no later call of up to n requests creates
 * them (the first call on a heap otherwise does, synchronously). */
int ouro_host_reserve(ouro_heap* h, uint32_t n);

/* Sequential replay of an op trace by one GPU thread (threadIdx.x = tid,
 * blockIdx.x = bid) for parity with the reference.  Op kinds, ops[2i] with
 * argument a = ops[2i+1]:
 *   0: malloc(a);  1: free(the result of op a);
 *   2: allocate_chunk();  3: enqueue_initial_chunk(a & 15, the chunk of op
 *      a >> 14, (a >> 4) & 1023 available pages);  4: free page a & 1023 of the
 *      chunk of op a >> 10.
 * results[i] (host array): for mallocs class << 32 | chunk << 9 | page, bit 63 =
 * null, bit 62 = CUDA device heap; for op 2 the chunk index; bit 63 for a failed
 * op 2 or 3; otherwise 0.  No counterpart in the reference, whose only caller is
 * its benchmark. */
int ouro_trace(ouro_heap* h, const uint32_t* ops, uint64_t n_ops, uint64_t* results, uint32_t tid, uint32_t bid);

/* The reference's updateMemoryManagerHost (include/device/Ouroboros_impl.cuh:137-144)
 * reduced to counters: 151 words, laid out as the oracle's state (see
 * oracle/ouro_oracle.h).  Synchronizes the device. */
int ouro_state(ouro_heap* h, uint64_t* out151);

typedef struct {
  uint32_t flags;             /* OURO_FLAG_*                               */
  uint64_t null_results;      /* mallocs that returned nullptr (OOM)        */
  uint64_t timeouts;          /* bounded waits that gave up                 */
  uint64_t chunk_allocs;      /* chunk allocations (Statistics.h:11)        */
  uint64_t next_free_chunk;   /* Memory::next_free_chunk                    */
  uint32_t timeout_sites;     /* one bit per kind of wait that gave up: 1, 2 unused, 4 a group
                                 in deficit waiting for its pages, 8 queue slot still
                                 full, 16 queue slot never written, 32 array index entry,
                                 64 linked successor, 128 walk length, 256 walks meeting
                                 recycled chunks, 512 / 1024 chunk reuse ring read / write,
                                 2048 chunk-queue scan */
} ouro_heap_status;
/* Device-side status; clear != 0 resets flags and counters afterwards. */
int ouro_get_status(ouro_heap* h, ouro_heap_status* out, int clear);

/* Harness kernels (src/main.cu:20-53 d_testWriteToMemory / d_testReadFromMemory
 * with a seeded pattern): word w of allocation i holds xorshift32((i ^ seed) | 1) + w,
 * written and checked with 16-byte vector accesses.  d_counters[0] += null
 * pointers, d_counters[1] += mismatching words. */
int ouro_write_pattern(void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed,
                       void* stream);
int ouro_verify_pattern(void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed,
                        unsigned long long* d_counters, void* stream);

/* Invariants of a set of live allocations (no counterpart in the reference):
 * every pointer inside the heap, aligned to its size class (up to the 8 KiB
 * chunk size: 16/32 KiB pages are 8 KiB aligned), and no 16-byte unit owned
 * twice (device ownership bitmap over the heap).  Synchronous. */
typedef struct {
  uint64_t checked;
  uint64_t nulls;
  uint64_t out_of_heap;
  uint64_t misaligned;
  uint64_t overlaps;
} ouro_alloc_report;
int ouro_check_allocations(ouro_heap* h, void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes,
                           ouro_alloc_report* out);

/* The checks of ouro_check_allocations without allocating anything: no
 * cudaMalloc, no cudaFree, no allocating library call.  For callers that
 * cannot allocate device memory -- a serving loop that must not stall its
 * other streams (cudaFree waits for the whole device), or a process whose
 * allocator heap already holds nearly all of HBM, so that the checker's own
 * bitmap allocation would fail.  No counterpart in the reference.
 *
 * The ownership bitmap is a fixed 8 MiB array inside this library
 * (OURO_NOALLOC_BITMAP_BYTES; every GPU that loads the library holds it until
 * exit).  It covers heaps of up to 1 GiB of chunk data (max_chunks <= 131072);
 * larger heaps return OURO_ERR_TOO_LARGE.  The current device must be the
 * heap's.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it with the device's current context; make
 * that first call before any stream capture.  A call in a new context (after
 * cudaDeviceReset) looks the address up again.  Each call clears the bitmap
 * words its heap uses and *d_report
 * (an ouro_alloc_report in DEVICE memory, filled in stream order; nothing is
 * synchronized).  All calls share the one array: calls whose work overlaps on
 * the GPU (other streams, or other host threads without ordering) race and
 * give wrong counts. */
#define OURO_NOALLOC_BITMAP_BYTES (8u << 20)
int ouro_check_allocations_noalloc(ouro_heap* h, void* const* d_ptrs, uint32_t n, uint32_t size,
                                   const uint32_t* d_sizes, ouro_alloc_report* d_report, void* stream);

/* Heap accounting invariants at quiescence (no allocation in flight), per
 * class: pages owned by the class's chunks, free pages recorded in chunk
 * metadata, the semaphore's count / expected / reserved and the queue length.
 * `bad` counts chunks whose count disagrees with their bitmask or whose
 * bitmask has bits beyond its pages.  Synchronous. */
typedef struct {
  uint64_t owned_pages[12];
  uint64_t free_pages_meta[12];   /* chunk-based: sum of chunk counts; page-based: queue length */
  int64_t sem_count[12];
  uint64_t sem_expected[12];
  uint64_t sem_reserved[12];
  uint64_t data_chunks;
  uint64_t bad;
} ouro_heap_report;
int ouro_check_heap(ouro_heap* h, ouro_heap_report* out);

/* Bulk pre-population of one size class (the reference's preFillQueue /
 * enqueueInitialChunk, include/device/queues/page/PageQueue.cuh:42-49,
 * PageQueue_impl.cuh:40-53, include/device/queues/chunk/ChunkQueue_impl.cuh:
 * 69-77): adds ceil(pages / pages-per-chunk) fresh chunks to the class of
 * `size` and publishes all their pages as free, warps adding 32 chunks at a
 * time through the path an elected allocation takes.  A later burst of that
 * class then starts without creating chunks.  *out_pages (may be NULL)
 * receives the pages added: fewer when the heap runs out.  Sizes above
 * 32 KiB (CUDA device heap) are refused.  Synchronizes `stream`. */
int ouro_prefill(ouro_heap* h, uint64_t size, uint64_t pages, uint64_t* out_pages, void* stream);

/* Ouroboros<...>::memory_manager.allocateChunk<false>  (include/device/Ouroboros.cuh:
 * 108-136), the call a caller of enqueueInitialChunk makes first: one 8 KiB chunk
 * of the heap (reuse queue first, then the bump pointer) into *out_chunk, or
 * UINT32_MAX when none is left.  Its pages start at data_base + chunk x 8192
 * (ouro_get_info).  Synchronous, default stream. */
int ouro_allocate_chunk(ouro_heap* h, uint32_t* out_chunk);

/* Ouroboros<...>::enqueueInitialChunk(queue_index, chunk_index, available_pages,
 * pages_per_chunk)  (include/device/Ouroboros.cuh:291-295; PageQueue_impl.cuh:40-53,
 * PageQueueVA_impl.cuh:94-125, PageQueueVL_impl.cuh:54-63, ChunkQueue_impl.cuh:
 * 69-77, ChunkQueueVA_impl.cuh:54-72, ChunkQueueVL_impl.cuh:49-56), together with
 * the chunk initializer its callers run first (PageIndexChunk.cuh:82-86,
 * ChunkIndexChunk.cuh:73-78): chunk_index, from ouro_allocate_chunk, joins size
 * class queue_index (0..9: 16 B << queue_index, the first instance, as in the
 * reference) with its last available_pages pages free and the pages before them
 * in the caller's use; they are freed like any page.  pages_per_chunk follows
 * from the class (8192 / page size).  Page-based heaps queue the free pages in
 * page order, chunk-based heaps queue the chunk; the class's semaphore gains
 * available_pages.  The reference's standard and virtualized-array chunk queues
 * accept this only as the class's first operation; here it may come at any
 * time.  OURO_ERR_ARG for a class, chunk or page count out of range,
 * OURO_ERR_DEVICE when the class's queue or the chunk budget has no room.
 * Synchronous, default stream. */
int ouro_enqueue_initial_chunk(ouro_heap* h, uint32_t queue_index, uint32_t chunk_index, uint32_t available_pages);

/* The batched path (no counterpart in the reference, whose only caller is its
 * per-thread benchmark): a batch is counting-sorted by size class on the
 * device (per-tile histograms in shared memory, a scan, a scatter of request
 * indices) and then served by one launch with a thread per request in sorted
 * order, so every warp but the one at each class boundary asks for one class
 * with all 32 lanes.  Frees are sorted by the class of the page they release.
 * block (of the serving launch) = 0 takes the size ouro_autotune_batch picked
 * (256 until then); else 128, 256, 512 or 1024.  Stream-ordered; the sort
 * uses the heap's batch scratch (4 bytes per request plus 64 per 4,096),
 * which a call for more requests than before allocates (cudaMalloc, so not
 * during stream capture: call ouro_batch_reserve first).  A reserved batch
 * cycle can be captured in a CUDA graph and replayed; calls on one heap
 * share the scratch, so concurrent batch calls on one heap must be ordered.
 *   ouro_batch_reserve: scratch for batches of up to n requests.
 *   ouro_alloc_batch:   d_out[i] = malloc(d_sizes[i])
 *   ouro_free_batch:    free(d_ptrs[i]) (nullptr skipped)
 *   ouro_realloc_batch: one churn cycle over a live set: request i is picked
 *     with probability fraction_permille / 1000 (a hash of seed, cycle and i);
 *     a picked request frees d_ptrs[i], draws a new size from *dist into
 *     d_sizes[i] and allocates it into d_ptrs[i]. */
typedef struct {
  int kind;       /* 0: log-uniform in [lo, hi] rounded up to 16 B;
                     1: Zipf(zipf_s) over the ten 16 B .. 8 KiB classes (rank 1 = 16 B) */
  uint32_t lo, hi;
  float zipf_s;
} ouro_size_dist;
int ouro_batch_reserve(ouro_heap* h, uint32_t n);
int ouro_alloc_batch(ouro_heap* h, const uint32_t* d_sizes, void** d_out, uint32_t n, int block, void* stream);
int ouro_free_batch(ouro_heap* h, void* const* d_ptrs, uint32_t n, int block, void* stream);
int ouro_realloc_batch(ouro_heap* h, void** d_ptrs, uint32_t* d_sizes, uint32_t n, uint64_t seed, uint32_t cycle,
                       uint32_t fraction_permille, const ouro_size_dist* dist, int block, void* stream);
/* Autotuner of the batched path: times alloc + free batches of n log-uniform
 * sizes in [lo, hi] on this heap for every block size of the serving launch
 * (128 .. 1024), keeps the fastest as the heap's batched launch shape and
 * reports it (Mops/s counts mallocs + frees; *out_per_sm is 0: the serving
 * launch is not persistent).  Uses the heap: call it on an idle heap.
 * Allocates scratch; synchronous. */
int ouro_autotune_batch(ouro_heap* h, uint32_t n, uint32_t lo, uint32_t hi, int* out_block, int* out_per_sm,
                        double* out_mops);
/* Autotuner over the run-time configuration and the launch shape (no
 * counterpart in the reference, whose parameters are compile-time,
 * include/Parameters.h:9-18).  Every candidate gets a fresh heap of
 * `variant` and `heap_bytes`, on which n requests with seeded log-uniform
 * sizes in [lo, hi] are allocated and freed through the batched path: one
 * untimed repetition, then `reps` timed ones (alloc + free, event-timed).
 * Candidates: the queue capacities queue_entries[0..n_queue) (queue entries per
 * size class: a standard ring of that many entries, a virtualized-array index
 * of that many / 2048 queue chunks; not swept for the linked-list variants),
 * the aggregation widths agg_widths[0..n_agg) and the block sizes of the
 * serving launch blocks[0..n_blocks).  A candidate that returns a nullptr or
 * raises an error flag is rejected (ok = 0).  points, if not NULL, receives
 * every candidate (n_queue x n_agg x n_blocks entries, in that nesting
 * order); *best the fastest accepted one (Mops/s counts mallocs + frees).
 * OURO_ERR_DEVICE when no candidate is accepted.  Allocates its heaps and
 * buffers; synchronous. */
typedef struct {
  ouro_config cfg;
  int block;
  int ok;
  double mops;
} ouro_tune_point;
int ouro_autotune_config(int variant, uint64_t heap_bytes, uint32_t n, uint32_t lo, uint32_t hi, uint32_t reps,
                         const uint32_t* queue_entries, uint32_t n_queue, const uint32_t* agg_widths,
                         uint32_t n_agg, const int* blocks, uint32_t n_blocks, ouro_tune_point* points,
                         ouro_tune_point* best);

/* The dynamic-graph workload of the serving loop (no counterpart in the
 * reference; its consumer, ouroGraph, lives outside the reference tree).  A
 * graph of nv vertices keeps vertex v's out-edges, degree[v] uint32 ids, in
 * one allocation vptr[v] of 4 x degree[v] bytes.  Edge j of v is a hash of
 * (seed, v, j), so a vertex's content depends only on its degree.
 *   ouro_graph_init:  degrees from a power law P(d) ~ d^-alpha (1 <= d <= 1024),
 *     blocks allocated through the batched path and filled; d_scratch holds nv
 *     uint32; d_failed[0] += vertices left without a block.
 *   ouro_graph_grow:  each named vertex moves to a block of twice its edges
 *     (8 x d bytes, at most 8 KiB): malloc, copy, append, free.  Vertices may
 *     repeat within and across concurrent calls: a growing vertex is locked
 *     (bounded wait).  d_failed[0] += allocations that returned nullptr,
 *     d_failed[1] += requests that gave up waiting for a vertex.
 *   ouro_graph_check: d_out2[0] += a checksum of the named vertices' edges,
 *     d_out2[1] += vertices whose edges differ from their recipe.
 *   ouro_free_bytes_to: the heap's free bytes (free pages x page size + chunks
 *     never handed out or pooled x 8 KiB) written by a kernel to *dst (device
 *     or mapped pinned host memory) -- the admission watermark read without
 *     synchronizing the device.
 * All stream-ordered, no allocation. */
int ouro_graph_init(ouro_heap* h, void** d_vptr, uint32_t* d_degree, uint32_t* d_scratch, uint32_t nv, uint64_t seed,
                    float alpha, unsigned long long* d_failed, void* stream);
int ouro_graph_grow(ouro_heap* h, void** d_vptr, uint32_t* d_degree, const uint32_t* d_vertices, uint32_t n, uint32_t nv,
                    uint64_t seed, unsigned long long* d_failed, void* stream);
int ouro_graph_check(void* const* d_vptr, const uint32_t* d_degree, const uint32_t* d_vertices, uint32_t n, uint32_t nv,
                     uint64_t seed, unsigned long long* d_out2, void* stream);
int ouro_free_bytes_to(ouro_heap* h, unsigned long long* dst, void* stream);

/* The serving loop (no counterpart in the reference; its consumer, ouroGraph,
 * lives outside the reference tree): a persistent kernel that stays on the GPU
 * and serves batches of graph-growth requests (ouro_graph_grow's work) that
 * clients submit while it runs -- continuous batching without a host round
 * trip per batch.
 *   ouro_serve_start: launches the loop on its own non-blocking stream over the
 *     graph (d_vptr / d_degree of ouro_graph_init).  Batches are taken in
 *     submission order and admitted while the heap's free bytes, computed on
 *     the device from allocator state, stay at or above watermark x heap bytes
 *     (a batch is always admitted when none is in flight); at most
 *     max_inflight batches run at once, split into tiles of 1,024 requests
 *     that all blocks work on side by side.
 *   ouro_serve_submit: one batch, n vertex ids already in device memory
 *     (d_vertices stays valid until the batch is reported done).  A host store
 *     into a pinned, mapped ring: no CUDA call.  OURO_ERR_FULL when `ring`
 *     batches are submitted and not yet reported by ouro_serve_poll.
 *   ouro_serve_poll: up to max finished batches into out (any order), with
 *     device timestamps (%globaltimer, ns) taken when the loop saw the batch,
 *     admitted it and finished it.  Never blocks.
 *   ouro_serve_stop: no more submissions; waits until every submitted batch
 *     is done and the kernel has returned.  OURO_ERR_DEVICE when the loop
 *     ended on its own first (status: 1 = idle longer than idle_seconds).
 *     Batches can still be polled afterwards.
 *   ouro_serve_close: stops if needed and frees the loop's memory.
 * While the loop runs it occupies every SM: calls that synchronize the device
 * (ouro_state, ouro_check_heap, ...) wait for ouro_serve_stop. */
typedef struct ouro_server ouro_server;
typedef struct {
  uint32_t ring;           /* submission ring: batches outstanding at once (default 4096)   */
  uint32_t max_inflight;   /* batches admitted and unfinished at once (default 64)          */
  int blocks_per_sm;       /* resident blocks of the loop per SM, 0: as many as fit          */
  double watermark;        /* admission waits below this fraction of free heap (0.10)        */
  double idle_seconds;     /* the loop returns after this long with nothing to do (10)       */
} ouro_serve_config;
typedef struct {
  uint64_t seq;                 /* submission number, from 0                       */
  uint32_t client, n;
  uint64_t t_seen_ns, t_start_ns, t_done_ns;
  uint64_t failed_allocs;       /* requests whose malloc returned nullptr           */
  uint64_t lock_giveups;        /* requests that gave up waiting for their vertex   */
  uint32_t held_back;           /* 1 when the watermark deferred its admission      */
} ouro_serve_result;
typedef struct {
  uint64_t batches_seen, batches_admitted, held_back;
  uint32_t status;
} ouro_serve_stats;
int ouro_serve_start(ouro_heap* h, void** d_vptr, uint32_t* d_degree, uint32_t nv, uint64_t seed,
                     const ouro_serve_config* cfg, ouro_server** out);
int ouro_serve_submit(ouro_server* s, const uint32_t* d_vertices, uint32_t n, uint32_t client, uint64_t* out_seq);
int ouro_serve_poll(ouro_server* s, ouro_serve_result* out, uint32_t max, uint32_t* got);
int ouro_serve_stop(ouro_server* s, ouro_serve_stats* out);
int ouro_serve_close(ouro_server* s);

/* Free resources of a heap (include/device/MemoryQueries.cuh:8-88
 * printFreeResources, include/device/Statistics.h:30-57), as numbers instead
 * of printf: per class its page size, the free pages its semaphore counts and
 * the entries between its queue's front and back; overall the chunks in use
 * (bump pointer minus pooled chunks), the chunks never handed out, the
 * pooled ones, and free_bytes = sum of free pages x page size + (never handed
 * out + pooled) x chunk size -- the figure an admission watermark compares
 * against.  Reads the control block only; meaningful when no allocation is in
 * flight.  Synchronous. */
typedef struct {
  uint32_t page_size[12];
  int64_t free_pages[12];
  uint64_t queue_entries[12];
  uint64_t chunks_in_use;
  uint64_t chunks_untouched;
  uint64_t chunks_pooled;
  uint64_t free_bytes;
  uint64_t heap_chunks;     /* usable base chunks: max_chunks - 1 */
} ouro_free_report;
int ouro_free_resources(ouro_heap* h, ouro_free_report* out);

/* Measured L2 atomic throughput of the current device, the roofline
 * reference of the allocator kernels (no counterpart in the reference):
 * mode 0 distinct addresses (atomics/s over all lanes), mode 1 one hot 32-bit
 * address, mode 2 one hot 64-bit address (requests/s, one per warp), modes 3
 * and 4 two hot 32-bit addresses 128 B apart (one 256 B block) and 256 B apart,
 * alternate warps on each (requests/s in total).  Result in G operations per
 * second. */
int ouro_measure_atomics(int mode, double* gops);

/* Diagnostic counters, 12 words.  Chunk-based heaps: groups, probes, misses,
 * next-fit runs; for groups slower than 2^19 SM cycles the cycles their
 * leaders spent in the semaphore, the scan, dequeues and page claims; the
 * number of such groups; the slowest group's cycles; their probes and misses.
 * Page-based heaps: allocating groups, their cycles in the semaphore and in
 * taking entries, -, freeing groups, their cycles, the slowest free, -,
 * allocating groups slower than 2^20 cycles, the slowest allocation.  All zero unless the library
 * was built with -DOURO_SCAN_STATS.  No counterpart in the reference. */
int ouro_scan_stats(ouro_heap* h, uint64_t* out12, int clear);

const char* ouro_status_string(int code);

#ifdef __cplusplus
}
#endif
#endif
