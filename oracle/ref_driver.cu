// ref_driver.cu -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference allocator (GPUPeople/Ouroboros, included read-only from
// its own headers at build time; see oracle/Makefile) through a small C ABI so
// that tests and the reference leg of bench.py can run it on the same inputs as
// the CUDA allocator of this repository.  The reference sources are not copied:
// this file only instantiates MultiOuro{PQ,CQ,VAPQ,VACQ,VLPQ,VLCQ}
// (include/InstanceDefinitions.cuh:16-34, the types src/main.cu:8 selects) and
// calls their public interface: initialize(), getDeviceMemoryManager() and the
// device malloc()/free().  The per-thread kernels mirror src/main.cu:10-63.
#include <iostream>
#include <cstdint>
#include <cstdio>
#include <type_traits>

#include "device/Ouroboros_impl.cuh"
#include "device/MemoryInitialization.cuh"
#include "InstanceDefinitions.cuh"

namespace {

constexpr uint32_t kStateWords = 151;

template <typename T, typename = void> struct has_count : std::false_type {};
template <typename T> struct has_count<T, std::void_t<decltype(std::declval<T&>().count_)>> : std::true_type {};
template <typename T, typename = void> struct has_vq_ptrs : std::false_type {};
template <typename T> struct has_vq_ptrs<T, std::void_t<decltype(std::declval<T&>().old_count_)>> : std::true_type {};

// One thread of the grid replays the whole trace (src/main.cu style device calls).
template <typename MM>
__global__ void k_trace(MM* mm, const uint32_t* ops, uint64_t n, int64_t* off, void** ptrs, uint32_t tid,
                        uint32_t bid) {
  if (threadIdx.x != tid || blockIdx.x != bid) return;
  char* d_data = reinterpret_cast<char*>(mm->memory.d_data);
  char* d_mem = reinterpret_cast<char*>(mm->memory.d_memory);
  size_t asz = mm->memory.allocationSize;
  using ChunkType = typename MM::ChunkType;
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t op = ops[2 * i], arg = ops[2 * i + 1];
    ptrs[i] = nullptr;
    off[i] = 0;
    if (op == 0u) {
      void* p = mm->malloc(arg);
      ptrs[i] = p;
      char* c = reinterpret_cast<char*>(p);
      if (!p) off[i] = -1;
      else if (c > d_mem && c < d_mem + asz) off[i] = c - d_data;
      else off[i] = -2;
    } else if (op == 1u) {
      mm->free(ptrs[arg]);
    } else if (op == 2u) {
      // the first instance's allocateChunk (Ouroboros.cuh:108-136), as a
      // caller of enqueueInitialChunk does before it
      index_t c = 0;
      mm->memory_manager.template allocateChunk<false>(c);
      off[i] = c;
    } else if (op == 3u) {
      // chunk initializer (PageIndexChunk.cuh:82-86 / ChunkIndexChunk.cuh:73-78)
      // then Ouroboros.cuh:291-295 enqueueInitialChunk
      const index_t c = static_cast<index_t>(off[arg >> 14]);
      const uint32_t qi = arg & 15u, avail = (arg >> 4) & 1023u, ppc = 512u >> qi;
      ChunkType::initializeChunk(mm->memory.d_data, c, static_cast<int>(avail), ppc);
      __threadfence();
      mm->enqueueInitialChunk(qi, c, static_cast<int>(avail), ppc);
    } else {
      // free of a page the caller held from an initial chunk
      const index_t c = static_cast<index_t>(off[arg >> 10]);
      const unsigned int ps = ChunkType::getAccess(mm->memory.d_data, c)->page_size;
      mm->free(ChunkType::getPage(mm->memory.d_data, c, arg & 1023u, ps));
    }
  }
}

// src/main.cu:10-18 d_testAllocation with a fixed size, or per-thread sizes.
template <typename MM>
__global__ void k_alloc(MM* mm, void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes) {
  uint32_t tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  ptrs[tid] = mm->malloc(sizes ? sizes[tid] : size);
}

// src/main.cu:55-63 d_testFree
template <typename MM>
__global__ void k_free(MM* mm, void** ptrs, uint32_t n) {
  uint32_t tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  mm->free(ptrs[tid]);
}

__device__ __forceinline__ uint32_t xorshift32(uint32_t x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

// src/main.cu:20-53 write/verify, with a seeded pattern and a mismatch counter
// in place of printf.  counters[0] = null results, counters[1] = bad words.
__global__ void k_write(void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, uint32_t seed) {
  uint32_t tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  uint32_t* p = reinterpret_cast<uint32_t*>(ptrs[tid]);
  if (!p) return;
  uint32_t words = (sizes ? sizes[tid] : size) / 4u;
  uint32_t v = xorshift32((tid ^ seed) | 1u);
  for (uint32_t i = 0; i < words; ++i) p[i] = v + i;
}

__global__ void k_verify(void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, uint32_t seed,
                         unsigned long long* counters) {
  uint32_t tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  uint32_t* p = reinterpret_cast<uint32_t*>(ptrs[tid]);
  if (!p) { atomicAdd(&counters[0], 1ull); return; }
  uint32_t words = (sizes ? sizes[tid] : size) / 4u;
  uint32_t v = xorshift32((tid ^ seed) | 1u);
  uint32_t bad = 0;
  for (uint32_t i = 0; i < words; ++i) bad += p[i] != v + i;
  if (bad) atomicAdd(&counters[1], (unsigned long long)bad);
}

// The harness writes through, and the reference frees, the pointers the
// reference's malloc returned.  A pointer outside the reference's chunk
// region [d_data, d_data + maxChunks * 8320) -- which its code has no business
// returning for requests of at most 8 KiB -- is replaced by nullptr here and
// counted in counters[1], so that neither the pattern kernels nor the
// reference's own free ever dereference it.
__global__ void k_sanitize(void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, const char* lo,
                           const char* hi, unsigned long long* counters) {
  uint32_t tid = threadIdx.x + blockIdx.x * blockDim.x;
  if (tid >= n) return;
  const char* p = reinterpret_cast<const char*>(ptrs[tid]);
  if (!p) return;
  const uint32_t sz = sizes ? sizes[tid] : size;
  if (sz > 8192u) return;   // served by the CUDA device heap
  if (p < lo || p + sz > hi) {
    ptrs[tid] = nullptr;
    atomicAdd(&counters[1], 1ull);
  }
}

struct RefBase {
  virtual ~RefBase() {}
  virtual int sanitize(void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, unsigned long long* counters,
                       cudaStream_t s) = 0;
  virtual int trace(const uint32_t* ops, uint64_t n, int64_t* off, uint32_t tid, uint32_t bid) = 0;
  virtual int state(uint64_t* out) = 0;
  virtual int alloc(uint32_t n, uint32_t size, const uint32_t* sizes, void** ptrs, int block, cudaStream_t s) = 0;
  virtual int free_(uint32_t n, void** ptrs, int block, cudaStream_t s) = 0;
  virtual void info(uint64_t* out) = 0;
};

template <typename Q>
void queue_state(const Q& q, char* d_data, uint64_t* o) {
  int count, expected, reserved;
  uint64_t v = q.semaphore.value;
  count = static_cast<int>(v & BulkSemaphore::highest_value_mask) - static_cast<int>(BulkSemaphore::null_value);
  expected = static_cast<int>((v >> BulkSemaphore::middle_mask_shift) & BulkSemaphore::highest_value_mask);
  reserved = static_cast<int>((v >> BulkSemaphore::upper_mask_shift) & BulkSemaphore::highest_value_mask);
  o[0] = static_cast<uint64_t>(static_cast<int64_t>(count));
  o[1] = static_cast<uint64_t>(static_cast<int64_t>(expected));
  o[2] = static_cast<uint64_t>(static_cast<int64_t>(reserved));
  o[3] = q.front_;
  o[4] = q.back_;
  if constexpr (has_vq_ptrs<Q>::value) {
    auto idx = [&](const void* p) -> uint64_t {
      return p ? static_cast<uint64_t>((reinterpret_cast<const char*>(p) - d_data) / 8320) : ~0ull;
    };
    o[6] = idx(q.front_ptr_);
    o[7] = idx(q.back_ptr_);
    o[8] = idx(q.old_ptr_);
    o[9] = q.old_count_;
  }
  if constexpr (Q::virtualized && !has_vq_ptrs<Q>::value) {
    static uint32_t vq[virtual_queue_size];
    cudaMemcpy(vq, q.queue_, sizeof(vq), cudaMemcpyDeviceToHost);
    uint64_t d = 0;
    for (uint32_t i = 0; i < virtual_queue_size; ++i)
      if (vq[i] != 0xFFFFFFFFu) d += static_cast<uint64_t>(i + 1u) * (static_cast<uint64_t>(vq[i]) + 1u);
    o[10] = d;
  }
}

template <typename Q>
void count_state(const Q& q, uint64_t* o) {
  if constexpr (has_count<Q>::value) o[5] = static_cast<uint64_t>(static_cast<int64_t>(q.count_));
}

template <typename MM, bool ChunkBased>
struct RefHeap : RefBase {
  MM mm;
  explicit RefHeap(size_t heap) { mm.initialize(heap); }

  int trace(const uint32_t* ops, uint64_t n, int64_t* off, uint32_t tid, uint32_t bid) override {
    uint32_t* d_ops = nullptr;
    int64_t* d_off = nullptr;
    void** d_ptrs = nullptr;
    if (cudaMalloc(&d_ops, 8 * n) || cudaMalloc(&d_off, 8 * n) || cudaMalloc(&d_ptrs, 8 * n)) return 3;
    cudaMemcpy(d_ops, ops, 8 * n, cudaMemcpyHostToDevice);
    uint32_t block = (tid / 32u + 1u) * 32u;
    k_trace<MM><<<bid + 1u, block>>>(mm.getDeviceMemoryManager(), d_ops, n, d_off, d_ptrs, tid, bid);
    cudaError_t e = cudaDeviceSynchronize();
    cudaMemcpy(off, d_off, 8 * n, cudaMemcpyDeviceToHost);
    cudaFree(d_ops);
    cudaFree(d_off);
    cudaFree(d_ptrs);
    return e == cudaSuccess ? 0 : 4;
  }

  int state(uint64_t* out) override {
    if (cudaDeviceSynchronize() != cudaSuccess) return 4;
    updateMemoryManagerHost(mm);
    for (uint32_t i = 0; i < kStateWords; ++i) out[i] = 0;
    char* d_data = reinterpret_cast<char*>(mm.memory.d_data);
    out[0] = mm.memory.next_free_chunk;
    auto& i0 = mm.memory_manager;
    auto& i1 = mm.next_memory_manager.memory_manager;
    out[1] = static_cast<uint64_t>(static_cast<int64_t>(i0.d_chunk_reuse_queue.count_));
    out[2] = i0.d_chunk_reuse_queue.front_;
    out[3] = i0.d_chunk_reuse_queue.back_;
    out[4] = static_cast<uint64_t>(static_cast<int64_t>(i1.d_chunk_reuse_queue.count_));
    out[5] = i1.d_chunk_reuse_queue.front_;
    out[6] = i1.d_chunk_reuse_queue.back_;
    int cls = 0;
    for (int q = 0; q < 10; ++q, ++cls) {
      uint64_t* o = out + 7 + 12 * cls;
      queue_state(i0.d_storage_reuse_queue[q], d_data, o);
      if constexpr (ChunkBased) count_state(i0.d_storage_reuse_queue[q], o);
      o[11] = 512u >> q;
    }
    for (int q = 0; q < 2; ++q, ++cls) {
      uint64_t* o = out + 7 + 12 * cls;
      queue_state(i1.d_storage_reuse_queue[q], d_data, o);
      if constexpr (ChunkBased) count_state(i1.d_storage_reuse_queue[q], o);
      o[11] = 2u >> q;
    }
    return 0;
  }

  int alloc(uint32_t n, uint32_t size, const uint32_t* sizes, void** ptrs, int block, cudaStream_t s) override {
    if (n == 0) return 0;
    k_alloc<MM><<<(n + block - 1) / block, block, 0, s>>>(mm.getDeviceMemoryManager(), ptrs, n, size, sizes);
    return cudaGetLastError() == cudaSuccess ? 0 : 4;
  }

  int free_(uint32_t n, void** ptrs, int block, cudaStream_t s) override {
    if (n == 0) return 0;
    k_free<MM><<<(n + block - 1) / block, block, 0, s>>>(mm.getDeviceMemoryManager(), ptrs, n);
    return cudaGetLastError() == cudaSuccess ? 0 : 4;
  }

  int sanitize(void** ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, unsigned long long* counters,
               cudaStream_t s) override {
    if (n == 0) return 0;
    const char* lo = reinterpret_cast<const char*>(mm.memory.d_data);
    const char* hi = lo + static_cast<size_t>(mm.memory.maxChunks) * 8320u;
    k_sanitize<<<(n + 255) / 256, 256, 0, s>>>(ptrs, n, size, sizes, lo, hi, counters);
    return cudaGetLastError() == cudaSuccess ? 0 : 4;
  }

  void info(uint64_t* out) override {
    out[0] = mm.memory.maxChunks;
    out[1] = mm.memory.allocationSize;
    out[2] = reinterpret_cast<uint64_t>(mm.memory.d_memory);
    out[3] = reinterpret_cast<uint64_t>(mm.memory.d_data);
  }
};

}  // namespace

extern "C" {

// variant: 0 P, 1 C, 2 VAP, 3 VAC, 4 VLP, 5 VLC
int ref_create(int variant, uint64_t heap_bytes, void** out) {
  if (!out) return 1;
  RefBase* h = nullptr;
  switch (variant) {
    case 0: h = new RefHeap<MultiOuroPQ, false>(heap_bytes); break;
    case 1: h = new RefHeap<MultiOuroCQ, true>(heap_bytes); break;
    case 2: h = new RefHeap<MultiOuroVAPQ, false>(heap_bytes); break;
    case 3: h = new RefHeap<MultiOuroVACQ, true>(heap_bytes); break;
    case 4: h = new RefHeap<MultiOuroVLPQ, false>(heap_bytes); break;
    case 5: h = new RefHeap<MultiOuroVLCQ, true>(heap_bytes); break;
    default: return 1;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) { delete h; return 4; }
  // initialize() sets cudaLimitMallocHeapSize once per type without checking;
  // after an earlier type has launched kernels that call device malloc the
  // call fails with a non-sticky error that would surface at the next
  // cudaGetLastError().  Clear it here.
  (void)cudaGetLastError();
  *out = h;
  return 0;
}

int ref_destroy(void* h) {
  delete static_cast<RefBase*>(h);
  return 0;
}

int ref_trace(void* h, const uint32_t* ops, uint64_t n, int64_t* off, uint32_t tid, uint32_t bid) {
  if (!h || !ops || !off || n == 0) return 1;
  return static_cast<RefBase*>(h)->trace(ops, n, off, tid, bid);
}

int ref_state(void* h, uint64_t* out) {
  if (!h || !out) return 1;
  return static_cast<RefBase*>(h)->state(out);
}

// out[0] maxChunks, out[1] allocationSize, out[2] d_memory, out[3] d_data
int ref_info(void* h, uint64_t* out) {
  if (!h || !out) return 1;
  static_cast<RefBase*>(h)->info(out);
  return 0;
}

int ref_alloc(void* h, uint32_t n, uint32_t size, const uint32_t* d_sizes, void** d_ptrs, int block, void* stream) {
  if (!h || !d_ptrs || block <= 0) return 1;
  return static_cast<RefBase*>(h)->alloc(n, size, d_sizes, d_ptrs, block, static_cast<cudaStream_t>(stream));
}

int ref_free(void* h, uint32_t n, void** d_ptrs, int block, void* stream) {
  if (!h || !d_ptrs || block <= 0) return 1;
  return static_cast<RefBase*>(h)->free_(n, d_ptrs, block, static_cast<cudaStream_t>(stream));
}

int ref_sanitize(void* h, void** d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes,
                 unsigned long long* d_counters, void* stream) {
  if (!h || !d_ptrs || !d_counters) return 1;
  return static_cast<RefBase*>(h)->sanitize(d_ptrs, n, size, d_sizes, d_counters, static_cast<cudaStream_t>(stream));
}

int ref_write(void** d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed, void* stream) {
  if (n == 0) return 0;
  k_write<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_ptrs, n, size, d_sizes, seed);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

int ref_verify(void** d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed,
               unsigned long long* d_counters, void* stream) {
  if (n == 0) return 0;
  k_verify<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_ptrs, n, size, d_sizes, seed, d_counters);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

// The src/main.cu:146-167 loop for one (variant, size) cell: `reps` times
// {timed alloc, write, verify, timed free}, each followed by a synchronize.
// ms[0] = total alloc ms, ms[1] = total free ms.  d_counters as for ref_verify.
int ref_run_cell(void* h, uint32_t n, uint32_t size, int block, int reps, void** d_ptrs, uint32_t seed,
                 unsigned long long* d_counters, float* ms) {
  if (!h || !d_ptrs || !ms || reps <= 0) return 1;
  RefBase* r = static_cast<RefBase*>(h);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  ms[0] = ms[1] = 0.0f;
  int rc = 0;
  for (int i = 0; i < reps && rc == 0; ++i) {
    float t = 0.0f;
    cudaEventRecord(a, 0);
    rc |= r->alloc(n, size, nullptr, d_ptrs, block, 0);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&t, a, b);
    ms[0] += t;
    rc |= r->sanitize(d_ptrs, n, size, nullptr, d_counters, 0);
    rc |= ref_write(d_ptrs, n, size, nullptr, seed + static_cast<uint32_t>(i), nullptr);
    rc |= ref_verify(d_ptrs, n, size, nullptr, seed + static_cast<uint32_t>(i), d_counters, nullptr);
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 4;
    cudaEventRecord(a, 0);
    rc |= r->free_(n, d_ptrs, block, 0);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&t, a, b);
    ms[1] += t;
    if (cudaDeviceSynchronize() != cudaSuccess) rc = 4;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

}  // extern "C"
