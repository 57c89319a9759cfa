// common.cuh -- constants, memory-order primitives and warp-group helpers of
// the B200 allocator.  Everything here is hand-written for sm_100a.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ouro {

// ---------------------------------------------------------------- geometry
// The logical geometry follows the reference so that capacities and the
// (chunk, page) index space are identical: 8 KiB base chunks, 10 size classes
// of 16 B .. 8 KiB in the first instance, 2 classes of 16/32 KiB in 4-chunk
// chunks in the second (Parameters.h:9-19, InstanceDefinitions.cuh:16-34).
// Physically the 128 B metadata record of a chunk lives out of band in a
// dense array, so chunk data sits on an 8 KiB stride: page addresses are
// size-class aligned and pointer -> chunk is a shift, not a 64-bit divide.
constexpr uint32_t kChunkBytes = 8192u;
constexpr uint32_t kChunkShift = 13u;
constexpr uint32_t kMetaBytes = 128u;
constexpr uint32_t kRefStride = 8320u;      // reference chunk stride, capacity formula only
constexpr uint32_t kNumClasses = 12u;       // 10 + 2
constexpr uint32_t kQcSpots = 2048u;        // entries per queue chunk
// Queue sizes: the reference's, the defaults of the run-time configuration
// (each heap carries its own in ClassState::ring_mask / seg_mask).
constexpr uint32_t kVqSize = 16384u;        // virtual-array index entries
constexpr uint32_t kRingSize = 1u << 23;    // standard ring entries per class
constexpr uint32_t kReuseSize = 65536u;     // chunk reuse ring
constexpr uint32_t kOldHold = 10u;          // linked queue chunks held back before reuse
constexpr int kLowerFillC = 838860;         // chunk flashing threshold of the standard chunk queue
constexpr uint32_t kPageBits = 9u;          // MemoryIndex page bits

constexpr uint32_t kEmpty = 0xFFFFFFFFu;    // free slot / no chunk
constexpr uint32_t kTomb = 0xFFFFFFFEu;     // removed chunk-queue entry, front may pass it
constexpr uint32_t kPending = 0xFFFFFFFEu;  // queue_pos while an enqueue is in flight
constexpr uint32_t kInstalling = 0xFFFFFFFCu;  // queue-chunk link being installed by a waiting lane
// A lane that waits this many polls for a queue chunk that should have been
// pre-allocated installs one itself (the pre-allocation failed for lack of
// chunks, or its lane is slow).
constexpr uint32_t kInstallAfter = 256u;
// Queue chunks per class, beyond those holding its entries, that the chunk
// budget of the virtualized queues keeps free: partial chunks at both ends
// of the window, the pre-allocated successor, one more for a front that
// recycles late, and for linked queues the hold-back of drained chunks.
__host__ __device__ constexpr uint32_t queue_margin(int kind) { return kind == 1 ? 4u : kind == 2 ? 4u + kOldHold : 0u; }
// Removed entries a chunk queue may hold between front and back before a
// free helps the front (frees alone never move it).
constexpr uint32_t kFrontSlack = 4u * kQcSpots;
// Slots of the linked queues' chunk index (recently linked queue chunks).
constexpr uint32_t kSkipSlots = 1024u;

// class id -> instance properties
__host__ __device__ constexpr uint32_t class_instance(uint32_t cls) { return cls < 10u ? 0u : 1u; }
__host__ __device__ constexpr uint32_t class_page_size(uint32_t cls) {
  return cls < 10u ? (16u << cls) : (16384u << (cls - 10u));
}
__host__ __device__ constexpr uint32_t class_pages_per_chunk(uint32_t cls) {
  return cls < 10u ? (512u >> cls) : (2u >> (cls - 10u));
}
__host__ __device__ constexpr uint32_t class_page_shift(uint32_t cls) { return cls < 10u ? 4u + cls : 14u + (cls - 10u); }
__host__ __device__ constexpr uint32_t instance_factor(uint32_t inst) { return inst == 0u ? 1u : 4u; }
__host__ __device__ constexpr uint32_t instance_mask_words(uint32_t inst) { return inst == 0u ? 16u : 1u; }

// Helper.cuh:11-18 + 42-45: the queue index of a request size, restated, on
// the full 64-bit size (a request above 4 GiB must not wrap to a small power
// of two).  n = 0 gives -1.
__host__ __device__ inline int next_pow2_pow(uint64_t n) {
#ifdef __CUDA_ARCH__
  int lz = __clzll(static_cast<long long>(n));
#else
  int lz = n ? __builtin_clzll(n) : 64;
#endif
  return ((n & (n - 1u)) == 0u) ? 64 - lz - 1 : 64 - lz;
}

// Size -> class id (0..11), or -1 for sizes served by the CUDA device heap.
__host__ __device__ inline int size_class(uint64_t size) {
  if (size <= 8192u) {
    int q = next_pow2_pow(size) - 4;
    return q < 0 ? 0 : q;
  }
  if (size <= 32768u) {
    int q = next_pow2_pow(size) - 14;
    return 10 + (q < 0 ? 0 : q);
  }
  return -1;
}

__host__ __device__ constexpr uint32_t mem_index(uint32_t chunk, uint32_t page) { return (chunk << kPageBits) + page; }

// --------------------------------------------------------------- status
enum Status : uint32_t {
  kOk = 0u,
  kErrOom = 1u,         // an allocation found no chunk (not sticky in the product sense: nullptr returned)
  kErrTimeout = 2u,     // a bounded wait ran out: the heap may be inconsistent
  kErrCorrupt = 4u,     // a structural check failed (virtual start mismatch, bad pointer)
  kErrQueueFull = 8u,   // a size class reached its queue capacity
};

// Spin limits: every wait in this allocator gives up after this many polls
// (with nanosleep backoff capped at 1 us, roughly a quarter second) and
// reports kErrTimeout instead of hanging the GPU.
constexpr uint32_t kSpinLimit = 1u << 18;

__device__ __forceinline__ void backoff(uint32_t& iter) {
  uint32_t ns = 32u << (iter < 5u ? iter : 5u);
  __nanosleep(ns);
  ++iter;
}

// ------------------------------------------------------ PTX memory access
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int32_t ld_relaxed(const int32_t* p) {
  int32_t v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint2 ld_relaxed_v2(const uint32_t* p) {
  uint2 v;
  asm volatile("ld.relaxed.gpu.global.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint4 ld_relaxed_v4(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(int32_t* p, int32_t v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_v4(uint32_t* p, uint4 v) {
  asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};"
               :: "l"(p), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
}

// ------------------------------------------------------------ warp groups
// A group is the set of active lanes of a warp that share a key (a size
// class, a chunk, ...).  The lowest lane leads: it issues the group's single
// atomic on a hot counter and broadcasts the result.
struct Group {
  uint32_t mask;
  int leader;
  int rank;
  int size;
  __device__ __forceinline__ bool is_leader() const { return rank == 0; }
};

__device__ __forceinline__ uint32_t lane_id() {
  uint32_t l;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

__device__ __forceinline__ Group make_group(uint32_t mask) {
  Group g;
  g.mask = mask;
  g.leader = __ffs(mask) - 1;
  g.rank = __popc(mask & ((1u << lane_id()) - 1u));
  g.size = __popc(mask);
  return g;
}

__device__ __forceinline__ Group group_by(uint32_t within, uint64_t key) {
  return make_group(__match_any_sync(within, key));
}

template <typename T>
__device__ __forceinline__ T bcast(const Group& g, T v) {
  return __shfl_sync(g.mask, v, g.leader);
}
__device__ __forceinline__ unsigned long long bcast64(const Group& g, unsigned long long v) {
  return __shfl_sync(g.mask, v, g.leader);
}

}  // namespace ouro
