// ouroboros.cuh -- the device-side allocator object.
//
// Ouroboros<V> is what device code holds: `mm->malloc(size)` and
// `mm->free(ptr)` from any thread of any kernel, the interface of the
// reference's Ouroboros<...> (Ouroboros.cuh:285-287, Ouroboros_impl.cuh:83-125).
// V picks one of the six instantiations of InstanceDefinitions.cuh:16-34
// (always with the second 16-32 KiB instance, as the Multi* types the
// reference's benchmark uses):
//   0 page-based standard (MultiOuroPQ)     1 chunk-based standard (MultiOuroCQ)
//   2 page-based virtualized array (VAPQ)   3 chunk-based virtualized array (VACQ)
//   4 page-based virtualized list (VLPQ)    5 chunk-based virtualized list (VLCQ)
// Requests above 32 KiB go to the CUDA device heap, as in the reference
// (Ouroboros.cuh:401-408).  Out of memory yields nullptr.
#pragma once

#include <type_traits>

#include "queues.cuh"

namespace ouro {

template <int V>
struct Ouroboros : HeapCore {
  static_assert(V >= 0 && V < 6, "variant 0..5");
  static constexpr bool kPageBased = (V % 2) == 0;
  static constexpr int kKind = V / 2;
  using Store = std::conditional_t<kKind == 0, FlatStore, std::conditional_t<kKind == 1, VaStore, VlStore>>;

  // The lanes of this lane's aggregation segment (agg_width consecutive lanes;
  // the whole warp by default): requests are aggregated within it only.
  __device__ __forceinline__ uint32_t segment() const {
    const uint32_t w = this->agg_width;
    if (w - 1u >= 31u) return 0xFFFFFFFFu;   // 32 (or an unset 0): the whole warp
    return ((1u << w) - 1u) << (lane_id() & ~(w - 1u));
  }

  __device__ __forceinline__ void* malloc(size_t size) {
    const int cls = size_class(size);
    const uint32_t active = __activemask() & segment();
    const Group g = group_by(active, static_cast<uint64_t>(cls + 1));
    if (cls < 0) {
      // Ouroboros<>::malloc: next power of two from the CUDA device heap
      // (a size whose power of two does not fit in size_t cannot be served)
      const int p2 = next_pow2_pow(size);
      if (p2 >= 63) return nullptr;
      return ::malloc(static_cast<size_t>(1) << p2);
    }
    ClassState* q = &this->cls[cls];
    if constexpr (kPageBased) return page_alloc<Store>(this, q, g);
    else return chunk_alloc<Store>(this, q, g);
  }

  // Bulk pre-population (the reference's preFillQueue / enqueueInitialChunk,
  // PageQueue.cuh:42-49, PageQueue_impl.cuh:40-53, ChunkQueue_impl.cuh:69-77):
  // the group adds k fresh chunks to class cls and publishes all their pages
  // as free, through the path a group in deficit takes to add chunks.
  // Collective over the calling lanes of one warp, k <= their number.
  // Returns the chunks added.
  __device__ __forceinline__ uint32_t prefill(uint32_t cls, uint32_t k) {
    const Group g = make_group(__activemask());
    ClassState* q = &this->cls[cls];
    if constexpr (kPageBased) return page_grow<Store>(this, q, g, k, false);
    else return chunk_grow<Store>(this, q, g, k, false);
  }

  // allocateChunk<false> of the first instance (Ouroboros.cuh:108-136), the
  // call that callers of enqueueInitialChunk make first: one 8 KiB chunk from
  // the reuse queue or the bump pointer, kEmpty when none is left.  One lane.
  __device__ __forceinline__ uint32_t allocate_chunk() {
    const Group self = make_group(1u << lane_id());
    uint32_t c = kEmpty;
    const uint32_t got = alloc_chunks(this, self, 1u, 0u, false, &c);
    return got ? c : kEmpty;
  }

  // Ouroboros.cuh:291-295 enqueueInitialChunk(queue_index, chunk_index,
  // available_pages, pages_per_chunk) with the chunk initializer its callers
  // run before it: chunk `chunk` (from allocate_chunk) joins class
  // queue_index (0..9, the first instance, as in the reference) with pages
  // [ppc - available_pages, ppc) free and the pages before them in the
  // caller's use (they are freed like any page); pages-per-chunk follows from
  // the class.  One lane; false for bad arguments or when the class's queue or
  // the chunk budget has no room.  The reference's standard and virtualized-
  // array chunk queues accept it only as their class's first operation; here
  // it may come at any time.
  __device__ __forceinline__ bool enqueue_initial_chunk(uint32_t queue_index, uint32_t chunk, uint32_t available_pages) {
    if (queue_index >= 10u) return false;
    ClassState* q = &this->cls[queue_index];
    if (available_pages == 0u || available_pages > q->ppc || chunk >= this->max_chunks - 1u) return false;
    return enqueue_initial<Store, kPageBased>(this, q, chunk, available_pages);
  }

  __device__ __forceinline__ void free(void* ptr) {
    const uint32_t active = __activemask() & segment();
    char* p = static_cast<char*>(ptr);
    const bool in_heap = p >= this->data && p < this->data_end;
    const uint32_t heap_mask = __ballot_sync(active, in_heap);
    if (!in_heap) {
      if (ptr) ::free(ptr);   // foreign pointer: the CUDA device heap (Ouroboros_impl.cuh:97-103)
      return;
    }
    const size_t off = static_cast<size_t>(p - this->data);
    uint32_t c = static_cast<uint32_t>(off >> kChunkShift);
    uint2 ph = ld_relaxed_v2(&this->meta[c].page_size);   // page_size, head
    if (ph.y) c -= ph.y;
    const uint32_t page_size = ph.x;
    int cls = page_size ? size_class(page_size) : -1;
    const uint32_t shift = cls >= 0 ? class_page_shift(static_cast<uint32_t>(cls)) : 0u;
    const uint32_t page = static_cast<uint32_t>((off - (static_cast<size_t>(c) << kChunkShift)) >> shift);
    const Group g = group_by(heap_mask, static_cast<uint64_t>(cls + 1));
    if (cls < 0) {
      set_status(this, kErrCorrupt);
      return;
    }
    ClassState* q = &this->cls[cls];
    if constexpr (kPageBased) page_free<Store>(this, q, g, mem_index(c, page));
    else chunk_free<Store, kKind == 0>(this, q, g, c, page);
  }
};

}  // namespace ouro
