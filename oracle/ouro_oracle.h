/*
 * ouro_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A sequential, single-threaded CPU restatement of the Ouroboros device
 * allocator (GPUPeople/Ouroboros, the MultiOuro{PQ,CQ,VAPQ,VACQ,VLPQ,VLCQ}
 * instantiations of include/InstanceDefinitions.cuh:16-34).  It exists to
 * check the CUDA allocator in ouroboros_b200/: only tests/, the smoke check
 * and the CPU-baseline leg of bench.py may load it.  Nothing in the product
 * path calls it.
 *
 * Pinning: the layout arithmetic (maxChunks, allocation size) and every trace
 * result and counter are checked against tests/golden/trace_*.npz: the
 * reference's own sm_100a build running the same traces with one GPU thread on
 * a 1 GiB heap (generator: tests/golden/make_golden.py), plus the reference's
 * maxChunks at 1..32 GiB from a host probe of its types.
 *
 * Result encoding (shared with the CUDA allocator's trace entry point):
 *   bits  0..31  MemoryIndex = chunk << 9 | page        (MemoryIndex.cuh:6-51)
 *   bits 32..39  class id = instance * 16 + queue index
 *   bit  62      served by the CUDA device heap (size > 32 KiB)
 *   bit  63      allocation failed (null)
 */
#ifndef OURO_ORACLE_H
#define OURO_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_P = 0, ORC_C = 1, ORC_VAP = 2, ORC_VAC = 3, ORC_VLP = 4, ORC_VLC = 5 };

enum {
  ORC_OK = 0,
  ORC_ERR_ARG = 1,
  ORC_ERR_UB = 2,       /* the reference would run into undefined behaviour here */
  ORC_ERR_TRAP = 3,     /* the reference would __trap() here */
  ORC_ERR_HANG = 4      /* the reference would spin forever here */
};

#define ORC_RES_FAIL    (1ull << 63)
#define ORC_RES_DEVHEAP (1ull << 62)
#define ORC_STATE_WORDS 151
#define ORC_NUM_CLASSES 12

typedef struct {
  uint64_t object_bytes;      /* Ouroboros<...>::size_()                         */
  uint64_t queue_bytes;       /* totalMemoryManagerSize()                        */
  uint64_t total_required;    /* MemoryInitialization.cuh:159                    */
  uint64_t max_chunks;        /* MemoryInitialization.cuh:161                    */
  uint64_t locator_bytes;     /* MemoryInitialization.cuh:163                    */
  uint64_t allocation_bytes;  /* MemoryInitialization.cuh:164                    */
} orc_layout;

typedef struct orc_heap orc_heap;

int orc_layout_of(int variant, uint64_t heap_bytes, orc_layout* out);

/* tid/bid: the threadIdx.x / blockIdx.x of the single GPU thread being
 * restated (they seed the bitmask search of the chunk-based variants). */
orc_heap* orc_create(int variant, uint64_t heap_bytes, uint32_t tid, uint32_t bid);
void orc_destroy(orc_heap* h);

/* One malloc.  *res gets the encoded result, *ref_off the byte offset of the
 * page from the reference's d_data (or -1 / -2 for null / device heap). */
int orc_malloc(orc_heap* h, uint64_t size, uint64_t* res, int64_t* ref_off);
/* One free of a result previously returned by orc_malloc. */
int orc_free(orc_heap* h, uint64_t res);

/* allocateChunk<false> of the first instance (Ouroboros.cuh:108-136). */
int orc_allocate_chunk(orc_heap* h, uint32_t* chunk);
/* enqueueInitialChunk (Ouroboros.cuh:291-295) of chunk c into class queue_index
 * of the first instance, after the chunk initializer its callers run: the last
 * `available` pages free, the ones before them in the caller's use. */
int orc_enqueue_initial(orc_heap* h, uint32_t queue_index, uint32_t c, uint32_t available);

/* Trace replay.  ops[2i] = 0 -> malloc(a); 1 -> free(result of op a);
 * 2 -> allocate a chunk; 3 -> enqueue_initial(a & 15, chunk of op a >> 14,
 * (a >> 4) & 1023 pages); 4 -> free page a & 1023 of the chunk of op a >> 10
 * (a = ops[2i+1]).  res[i] / ref_off[i] as for orc_malloc, the chunk index for
 * op 2, 0 otherwise.  Stops at the first error and reports the failing op index
 * in *failed_at. */
int orc_run_trace(orc_heap* h, const uint32_t* ops, uint64_t n_ops,
                  uint64_t* res, int64_t* ref_off, uint64_t* failed_at);

/* Counter snapshot, ORC_STATE_WORDS words:
 *   [0] next_free_chunk  [1..3] reuse queue 0 count/front/back  [4..6] reuse queue 1
 *   then per class (12 classes, 12 words each):
 *   sem count, sem expected, sem reserved, front, back, chunk count_,
 *   VL front/back/old chunk index, VL old_count, VA index-array digest, pages per chunk */
int orc_state(const orc_heap* h, uint64_t* out);

/* Aggregate statistics of a heap (chunks touched, pages in queues). */
uint64_t orc_next_free_chunk(const orc_heap* h);

#ifdef __cplusplus
}
#endif
#endif
