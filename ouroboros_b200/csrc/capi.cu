// capi.cu -- host side of the B200 allocator behind the C ABI of
// include/ouroboros_b200.h: heap creation (the reference's initialize()),
// the per-thread launch path, sequential trace replay, state readback and the
// invariant checkers.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "handle.h"

using namespace ouro;

namespace {

// ------------------------------------------------------------------ kernels

// Bulk pre-population: warps take up to 32 chunks of work at a time from a
// counter and add them to class cls; d_done[0] counts the chunks added.
template <int V>
__global__ void k_prefill(Ouroboros<V>* mm, uint32_t cls, uint32_t chunks, uint32_t* d_next,
                          unsigned long long* d_done) {
  for (;;) {
    uint32_t base = 0;
    if (lane_id() == 0u) base = atomicAdd(d_next, 32u);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (base >= chunks) return;
    const uint32_t k = chunks - base < 32u ? chunks - base : 32u;
    const uint32_t got = mm->prefill(cls, k);
    if (lane_id() == 0u) atomicAdd(d_done, static_cast<unsigned long long>(got));
    if (got < k) return;   // out of chunks (or budget)
  }
}

// Queue initialization of the virtualized variants (MemoryInitialization.cuh:91-119
// with PageQueueVA_impl.cuh:11-28 / PageQueueVL_impl.cuh:11-30): one queue chunk
// per class, allocated in class order by a single thread.
template <int V>
__global__ void k_init_queues(Ouroboros<V>* mm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (uint32_t cls = 0; cls < kNumClasses; ++cls) {
    ClassState* q = &mm->cls[cls];
    uint32_t c = new_queue_chunk(mm, q->inst, 0u, queue_tag(q));
    if (c == kEmpty) return;
    if constexpr (Ouroboros<V>::kKind == 1) {
      st_relaxed(q->ring, c);
    } else {
      q->front_ptr = c;
      q->back_ptr = c;
      q->old_ptr = c;
      VlStore::remember(mm, q, c, 0u);
    }
  }
  __threadfence();
}

template <int V>
__global__ void k_alloc(Ouroboros<V>* mm, uint32_t n, uint32_t size, const uint32_t* sizes, void** out) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n) return;
  out[tid] = mm->malloc(sizes ? sizes[tid] : size);
}

template <int V>
__global__ void k_free(Ouroboros<V>* mm, uint32_t n, void* const* ptrs) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= n) return;
  mm->free(ptrs[tid]);
}

// class id of the oracle's encoding: instance * 16 + queue index
__device__ __forceinline__ uint64_t encode_result(HeapCore* h, void* p) {
  if (!p) return 1ull << 63;
  char* c = static_cast<char*>(p);
  if (c < h->data || c >= h->data_end) return 1ull << 62;
  size_t off = static_cast<size_t>(c - h->data);
  uint32_t chunk = static_cast<uint32_t>(off >> kChunkShift);
  uint32_t head = ld_relaxed(&h->meta[chunk].head);
  chunk -= head;
  uint32_t ps = ld_relaxed(&h->meta[chunk].page_size);
  int cls = ps ? size_class(ps) : -1;
  if (cls < 0) return (1ull << 63) | 1ull;
  uint32_t page = static_cast<uint32_t>((off - (static_cast<size_t>(chunk) << kChunkShift)) >> class_page_shift(cls));
  uint64_t cid = cls < 10 ? static_cast<uint64_t>(cls) : 16ull + static_cast<uint64_t>(cls - 10);
  return (cid << 32) | mem_index(chunk, page);
}

template <int V>
__global__ void k_trace(Ouroboros<V>* mm, const uint32_t* ops, uint64_t n, uint64_t* res, void** ptrs, uint32_t tid,
                        uint32_t bid) {
  if (threadIdx.x != tid || blockIdx.x != bid) return;
  for (uint64_t i = 0; i < n; ++i) {
    const uint32_t op = ops[2 * i], arg = ops[2 * i + 1];
    ptrs[i] = nullptr;
    res[i] = 0;
    if (op == 0u) {
      void* p = mm->malloc(arg);
      ptrs[i] = p;
      res[i] = encode_result(mm, p);
    } else if (op == 1u) {
      mm->free(ptrs[arg]);
    } else if (op == 2u) {
      const uint32_t c = mm->allocate_chunk();
      res[i] = c == kEmpty ? (1ull << 63) : c;
    } else if (op == 3u) {
      const bool ok = mm->enqueue_initial_chunk(arg & 15u, static_cast<uint32_t>(res[arg >> 14]), (arg >> 4) & 1023u);
      res[i] = ok ? 0ull : (1ull << 63);
    } else {
      const uint32_t c = static_cast<uint32_t>(res[arg >> 10]);
      const uint32_t ps = ld_relaxed(&mm->meta[c].page_size);
      mm->free(mm->data + (static_cast<size_t>(c) << kChunkShift) + static_cast<size_t>(arg & 1023u) * ps);
    }
  }
}

// One lane runs the reference's allocateChunk / enqueueInitialChunk for the
// host (r: the chunk, or 1 for success).
template <int V>
__global__ void k_allocate_chunk(Ouroboros<V>* mm, unsigned long long* r) {
  const uint32_t c = mm->allocate_chunk();
  *r = c == kEmpty ? ~0ull : c;
}
template <int V>
__global__ void k_enqueue_initial(Ouroboros<V>* mm, uint32_t queue_index, uint32_t chunk, uint32_t avail,
                                  unsigned long long* r) {
  *r = mm->enqueue_initial_chunk(queue_index, chunk, avail) ? 1ull : 0ull;
}

__device__ __forceinline__ uint32_t pattern_seed(uint32_t i, uint32_t seed) {
  uint32_t x = (i ^ seed) | 1u;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

// One thread per allocation, 16 B stores (pages are at least 16 B aligned).
__global__ void k_write_pattern(void* const* ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, uint32_t seed) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t* p = static_cast<uint32_t*>(ptrs[i]);
  if (!p) return;
  const uint32_t words = (sizes ? sizes[i] : size) / 4u;
  const uint32_t v = pattern_seed(i, seed);
  uint32_t w = 0;
  for (; w + 4u <= words; w += 4u)
    *reinterpret_cast<uint4*>(p + w) = make_uint4(v + w, v + w + 1u, v + w + 2u, v + w + 3u);
  for (; w < words; ++w) p[w] = v + w;
}

__global__ void k_verify_pattern(void* const* ptrs, uint32_t n, uint32_t size, const uint32_t* sizes, uint32_t seed,
                                 unsigned long long* counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t nulls = 0, bad = 0;
  if (i < n) {
    const uint32_t* p = static_cast<const uint32_t*>(ptrs[i]);
    if (!p) {
      nulls = 1;
    } else {
      const uint32_t words = (sizes ? sizes[i] : size) / 4u;
      const uint32_t v = pattern_seed(i, seed);
      uint32_t w = 0;
      for (; w + 4u <= words; w += 4u) {
        uint4 x = *reinterpret_cast<const uint4*>(p + w);
        bad += (x.x != v + w) + (x.y != v + w + 1u) + (x.z != v + w + 2u) + (x.w != v + w + 3u);
      }
      for (; w < words; ++w) bad += p[w] != v + w;
    }
  }
  nulls = __reduce_add_sync(0xFFFFFFFFu, nulls);
  bad = __reduce_add_sync(0xFFFFFFFFu, bad);
  if ((threadIdx.x & 31u) == 0u) {
    if (nulls) atomicAdd(&counters[0], static_cast<unsigned long long>(nulls));
    if (bad) atomicAdd(&counters[1], static_cast<unsigned long long>(bad));
  }
}

// Ownership bitmap over the heap data at 16 B granularity.
// r[0] checked, r[1] nulls, r[2] out of heap, r[3] misaligned, r[4] overlapping units
__global__ void k_check_allocs(const HeapCore* h, void* const* ptrs, uint32_t n, uint32_t size, const uint32_t* sizes,
                               uint32_t* bitmap, unsigned long long* r) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const char* p = static_cast<const char*>(ptrs[i]);
  if (!p) { atomicAdd(&r[1], 1ull); return; }
  atomicAdd(&r[0], 1ull);
  const uint32_t sz = sizes ? sizes[i] : size;
  const int cls = size_class(sz);
  if (cls < 0) return;   // CUDA device heap
  if (p < h->data || p + sz > h->data_end) { atomicAdd(&r[2], 1ull); return; }
  const size_t off = static_cast<size_t>(p - h->data);
  // pages are aligned to their size class up to the 8 KiB chunk: 16/32 KiB
  // pages sit in 4-chunk chunks that start at any chunk index
  const uint32_t align = class_page_size(static_cast<uint32_t>(cls)) < kChunkBytes
                             ? class_page_size(static_cast<uint32_t>(cls)) : kChunkBytes;
  if (off & (align - 1u)) atomicAdd(&r[3], 1ull);
  const size_t u0 = off >> 4;
  const size_t units = (sz + 15u) >> 4 ? (sz + 15u) >> 4 : 1u;
  unsigned long long dup = 0;
  for (size_t u = u0; u < u0 + units;) {
    const uint32_t bit = static_cast<uint32_t>(u & 31u);
    const uint32_t take = (32u - bit) < (u0 + units - u) ? (32u - bit) : static_cast<uint32_t>(u0 + units - u);
    const uint32_t m = take == 32u ? 0xFFFFFFFFu : (((1u << take) - 1u) << bit);
    const uint32_t old = atomicOr(&bitmap[u >> 5], m);
    dup += __popc(old & m);
    u += take;
  }
  if (dup) atomicAdd(&r[4], dup);
}

// Per-chunk accounting.  r layout: [0..11] owned pages, [12..23] free pages
// (chunk counts), [24] data chunks, [25] bad chunks.
__global__ void k_check_heap(const HeapCore* h, uint64_t nchunks, bool chunk_based, unsigned long long* r) {
  for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < nchunks;
       c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const ChunkMeta* m = h->meta + c;
    if (m->page_size == 0u || m->head != 0u) continue;
    const int cls = size_class(m->page_size);
    if (cls < 0) { atomicAdd(&r[25], 1ull); continue; }
    atomicAdd(&r[24], 1ull);
    atomicAdd(&r[cls], static_cast<unsigned long long>(m->size));
    if (!chunk_based) continue;
    const uint32_t words = instance_mask_words(class_instance(static_cast<uint32_t>(cls)));
    uint32_t ones = 0, stray = 0;
    for (uint32_t w = 0; w < words; ++w) {
      const uint32_t lo = w * 32u;
      const uint32_t valid = m->size >= lo + 32u ? 0xFFFFFFFFu : (m->size > lo ? ((1u << (m->size - lo)) - 1u) : 0u);
      ones += __popc(*m->mask(w) & valid);
      stray += __popc(*m->mask(w) & ~valid);
    }
    if (m->count >= 0) atomicAdd(&r[12 + cls], static_cast<unsigned long long>(m->count));
    if (stray || static_cast<int32_t>(ones) != m->count) atomicAdd(&r[25], 1ull);
  }
}


// L2 atomic throughput references for the roofline (no counterpart in the
// reference).  mode 0: distinct addresses, every lane one atomicAdd with return
// on an L2-resident array; mode 1: one hot address, one atomicAdd per warp;
// mode 2: one hot 64-bit address, one atomicAdd per warp.
__global__ void k_peak_distinct(uint32_t* a, uint32_t mask, int iters, uint32_t* sink) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t acc = 0;
  for (int i = 0; i < iters; ++i) acc += atomicAdd(&a[(t + static_cast<uint32_t>(i) * stride) & mask], 1u);
  if (acc == 0x9E3779B9u) *sink = acc;
}
// stride > 0: two hot addresses `stride` words apart, alternate warps on each
// (mode 3: 128 B apart, one 256 B block; mode 4: 256 B apart).
__global__ void k_peak_hot(uint32_t* a, unsigned long long* a64, int iters, int wide, uint32_t stride, uint32_t* sink) {
  if ((threadIdx.x & 31u) != 0u) return;
  uint32_t* p = a + (((blockIdx.x * blockDim.x + threadIdx.x) >> 5) & 1u) * stride;
  uint32_t acc = 0;
  for (int i = 0; i < iters; ++i) {
    if (wide) acc += static_cast<uint32_t>(atomicAdd(a64, 32ull));
    else acc += atomicAdd(p, 32u);
  }
  if (acc == 0x9E3779B9u) *sink = acc;
}

// Devices whose CUDA device-heap limit was raised (the limit is per device).
constexpr int kMaxDevices = 64;
bool g_heap_limit_set[kMaxDevices] = {};
std::mutex g_heap_limit_mu;

}  // namespace

extern "C" {

const char* ouro_status_string(int code) {
  switch (code) {
    case OURO_OK: return "ok";
    case OURO_ERR_ARG: return "bad argument";
    case OURO_ERR_CUDA: return "CUDA runtime error";
    case OURO_ERR_NOMEM: return "device out of memory";
    case OURO_ERR_DEVICE: return "allocator reported an error on the device";
    case OURO_ERR_TOO_LARGE:
      return "heap too large for the fixed scratch of ouro_check_allocations_noalloc (at most 1 GiB of chunk data)";
    case OURO_ERR_FULL: return "the serving loop's submission ring is full";
    default: return "unknown status";
  }
}

int ouro_config_default(ouro_config* out) {
  if (!out) return OURO_ERR_ARG;
  out->chunk_bytes = kChunkBytes;
  out->page_queue_entries = kRingSize;
  out->virtual_queue_entries = kVqSize;
  out->agg_width = 32u;
  return OURO_OK;
}

int ouro_create(int variant, uint64_t heap_bytes, ouro_heap** out) {
  return ouro_create_config(variant, heap_bytes, nullptr, out);
}

int ouro_get_config(const ouro_heap* h, ouro_config* out) {
  if (!h || !out) return OURO_ERR_ARG;
  *out = h->cfg;
  return OURO_OK;
}

int ouro_create_config(int variant, uint64_t heap_bytes, const ouro_config* cfg_in, ouro_heap** out) {
  if (!out || variant < 0 || variant > 5) return OURO_ERR_ARG;
  *out = nullptr;
  ouro_config cfg;
  ouro_config_default(&cfg);
  if (cfg_in) cfg = *cfg_in;
  auto pow2 = [](uint32_t v) { return v && (v & (v - 1u)) == 0u; };
  if (cfg.chunk_bytes != kChunkBytes || !pow2(cfg.page_queue_entries) || cfg.page_queue_entries < (1u << 16) ||
      cfg.page_queue_entries > kRingSize || !pow2(cfg.virtual_queue_entries) || cfg.virtual_queue_entries < 32u ||
      cfg.virtual_queue_entries > kVqSize || !pow2(cfg.agg_width) || cfg.agg_width > 32u)
    return OURO_ERR_ARG;
  Layout L;
  if (!compute_layout(variant / 2, heap_bytes, &L, cfg.page_queue_entries, cfg.virtual_queue_entries))
    return OURO_ERR_ARG;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return OURO_ERR_CUDA;
  {
    // the reference reserves 500 MiB of CUDA device heap for requests > 32 KiB
    // (Parameters.h:49, MemoryInitialization.cuh:130-134); a per-device
    // limit, only settable before that device's first kernel that calls
    // device malloc
    std::lock_guard<std::mutex> lock(g_heap_limit_mu);
    if (device >= 0 && device < kMaxDevices && !g_heap_limit_set[device]) {
      size_t cur = 0;
      cudaDeviceGetLimit(&cur, cudaLimitMallocHeapSize);
      if (cur < (500ull << 20)) cudaDeviceSetLimit(cudaLimitMallocHeapSize, 500ull << 20);
      (void)cudaGetLastError();
      g_heap_limit_set[device] = true;
    }
  }
  ouro_heap* h = new (std::nothrow) ouro_heap();
  if (!h) return OURO_ERR_NOMEM;
  h->variant = variant;
  h->heap_bytes = heap_bytes;
  h->L = L;
  h->cfg = cfg;
  h->device = device;
  if (cudaMalloc(&h->raw, L.alloc_bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    delete h;
    return OURO_ERR_NOMEM;
  }
  h->base = reinterpret_cast<char*>(align_up(reinterpret_cast<unsigned long long>(h->raw), kChunkBytes));
  h->dev = reinterpret_cast<HeapCore*>(h->base);
  // metadata zero; chunk data and queues flooded with kEmpty (queue chunks are
  // taken from the data region without rewriting their entries)
  cudaError_t e = cudaMemset(h->base, 0, L.data_off);
  if (e == cudaSuccess) e = cudaMemset(h->base + L.data_off, 0xFF, L.ring_off - L.data_off);
  const unsigned long long q_end = L.reuse_off + 2ull * kReuseSize * 4u;
  if (e == cudaSuccess) e = cudaMemset(h->base + L.ring_off, 0xFF, q_end - L.ring_off);
  const uint32_t ring = static_cast<uint32_t>(L.ring_entries), vq = static_cast<uint32_t>(L.vq_entries);
  const uint32_t segs = ring / kQcSpots;
  if (e == cudaSuccess && variant / 2 == 0) e = cudaMemset(h->base + L.seg_off, 0, kNumClasses * segs * 4ull);
  std::unique_ptr<HeapCore> core_buf(new HeapCore());   // ~0.5 MiB: not on the stack
  HeapCore& core = *core_buf;
  std::memset(&core, 0, sizeof(core));
  core.variant = variant;
  core.max_chunks = static_cast<uint32_t>(L.max_chunks);
  core.meta = reinterpret_cast<ChunkMeta*>(h->base + L.meta_off);
  core.data = h->base + L.data_off;
  core.data_end = core.data + L.max_chunks * kChunkBytes;
  core.base = h->base;
  core.alloc_bytes = L.alloc_bytes;
  core.heap_bytes = heap_bytes;
  core.agg_width = cfg.agg_width;
  const int kind = variant / 2;
  if (kind != 0) {
    // usable base chunks (index + 1 < max_chunks); every class starts with
    // one queue chunk and keeps its margin
    core.budget_limit = L.max_chunks - 1u;
    core.budget.v = static_cast<unsigned long long>(kNumClasses) * (1u + queue_margin(kind));
  }
  for (int i = 0; i < 2; ++i) core.reuse[i].ring = reinterpret_cast<uint32_t*>(h->base + L.reuse_off) + i * kReuseSize;
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    ClassState& q = core.cls[c];
    q.sem.v = SemWord::kInit;
    q.cls = c;
    q.inst = class_instance(c);
    q.page_size = class_page_size(c);
    q.page_shift = class_page_shift(c);
    q.ppc = class_pages_per_chunk(c);
    q.words = instance_mask_words(q.inst);
    q.front_ptr = q.back_ptr = q.old_ptr = kEmpty;
    q.clean_on_recycle = (variant % 2) == 1 ? 1u : 0u;
    if (kind == 0) {
      q.ring = reinterpret_cast<uint32_t*>(h->base + L.ring_off) + static_cast<size_t>(c) * ring;
      q.ring_mask = ring - 1u;
      q.page_cap = ring;
      q.seg = reinterpret_cast<uint32_t*>(h->base + L.seg_off) + static_cast<size_t>(c) * segs;
      q.seg_mask = segs - 1u;
    } else if (kind == 1) {
      q.ring = reinterpret_cast<uint32_t*>(h->base + L.vq_off) + static_cast<size_t>(c) * vq;
      q.ring_mask = vq - 1u;
      q.page_cap = vq * kQcSpots;
    } else {
      q.page_cap = 1u << 30;   // linked queues are unbounded; positions are 32-bit
      q.skip = reinterpret_cast<uint32_t*>(h->base + L.skip_off) + static_cast<size_t>(c) * kSkipSlots;
    }
  }
  if (e == cudaSuccess) e = cudaMemcpy(h->base, &core, sizeof(core), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && kind != 0) {
    dispatch(variant, [&](auto v) {
      constexpr int V = decltype(v)::value;
      k_init_queues<V><<<1, 32>>>(reinterpret_cast<Ouroboros<V>*>(h->dev));
      return 0;
    });
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaFree(h->raw);
    delete h;
    return OURO_ERR_CUDA;
  }
  *out = h;
  return OURO_OK;
}

static void host_release(ouro_heap* h);

int ouro_destroy(ouro_heap* h) {
  if (!h) return OURO_ERR_ARG;
  host_release(h);
  if (h->batch_scratch) cudaFree(h->batch_scratch);
  cudaError_t e = cudaFree(h->raw);
  delete h;
  return cuda_rc(e);
}

void* ouro_device_handle(const ouro_heap* h) { return h ? static_cast<void*>(h->dev) : nullptr; }

int ouro_get_info(const ouro_heap* h, ouro_heap_info* out) {
  if (!h || !out) return OURO_ERR_ARG;
  out->variant = h->variant;
  out->heap_bytes = h->heap_bytes;
  out->max_chunks = h->L.max_chunks;
  out->alloc_bytes = h->L.alloc_bytes;
  out->data_base = reinterpret_cast<uint64_t>(h->base + h->L.data_off);
  out->data_end = out->data_base + h->L.max_chunks * kChunkBytes;
  return OURO_OK;
}

int ouro_alloc(ouro_heap* h, uint32_t n, uint32_t size, const uint32_t* d_sizes, void** d_out, int block,
               void* stream) {
  if (!h || !d_out || block <= 0 || block > 1024) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_alloc<V><<<grid_for(n, block), block, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<Ouroboros<V>*>(h->dev), n, size, d_sizes, d_out);
    return cuda_rc(cudaGetLastError());
  });
}

int ouro_free(ouro_heap* h, uint32_t n, void* const* d_ptrs, int block, void* stream) {
  if (!h || !d_ptrs || block <= 0 || block > 1024) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_free<V><<<grid_for(n, block), block, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<Ouroboros<V>*>(h->dev), n, d_ptrs);
    return cuda_rc(cudaGetLastError());
  });
}

// ------------------------------------------------------------ host buffers
// Requests and results in host memory.  The n requests are cut into slices:
// a slice's request sizes (or pointers) go host->device on host_in, its launch
// runs on the caller's stream once they are there, and (alloc) its pointers
// come back device->host on host_out once the launch is done, so the copies of
// one slice overlap the launches of the others.  Everything is ordered after
// the work queued on `stream` before the call, and after the previous
// host-buffer call on this heap (they share the staging), and it ends on
// `stream`: the caller synchronises `stream` before reading the results.
using ouro_host::host_slice_plan;
using ouro_host::kHostSlicesMax;

namespace {

int host_prepare(ouro_heap* h, size_t bytes) {
  if (!h->host_ready) {
    bool ok = cudaStreamCreateWithFlags(&h->host_in, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&h->host_out, cudaStreamNonBlocking) == cudaSuccess;
    cudaEvent_t* evs[3] = {&h->host_entry, &h->host_done, &h->host_joined};
    for (cudaEvent_t* e : evs) ok = ok && cudaEventCreateWithFlags(e, cudaEventDisableTiming) == cudaSuccess;
    for (uint32_t k = 0; k < kHostSlicesMax; ++k)
      ok = ok && cudaEventCreateWithFlags(&h->host_slice_in[k], cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&h->host_slice_run[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      (void)cudaGetLastError();
      return OURO_ERR_CUDA;
    }
    h->host_ready = true;
  }
  if (h->host_stage_bytes < bytes) {
    // cudaFree waits for the work still reading the old staging
    if (h->host_stage) cudaFree(h->host_stage);
    h->host_stage = nullptr;
    h->host_stage_bytes = 0;
    if (cudaMalloc(&h->host_stage, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return OURO_ERR_NOMEM;
    }
    h->host_stage_bytes = bytes;
  }
  return OURO_OK;
}

// The helper streams start after the caller's queued work and after the
// previous host-buffer call's copies.
void host_enter(ouro_heap* h, cudaStream_t s) {
  cudaEventRecord(h->host_entry, s);
  cudaStreamWaitEvent(h->host_in, h->host_entry, 0);
  cudaStreamWaitEvent(h->host_in, h->host_done, 0);
  cudaStreamWaitEvent(h->host_out, h->host_entry, 0);
  cudaStreamWaitEvent(h->host_out, h->host_done, 0);
}

}  // namespace

static void host_release(ouro_heap* h) {
  if (h->host_ready) {
    cudaStreamSynchronize(h->host_in);
    cudaStreamSynchronize(h->host_out);
    cudaStreamDestroy(h->host_in);
    cudaStreamDestroy(h->host_out);
    cudaEventDestroy(h->host_entry);
    cudaEventDestroy(h->host_done);
    cudaEventDestroy(h->host_joined);
    for (uint32_t k = 0; k < kHostSlicesMax; ++k) {
      cudaEventDestroy(h->host_slice_in[k]);
      cudaEventDestroy(h->host_slice_run[k]);
    }
    h->host_ready = false;
  }
  if (h->host_stage) cudaFree(h->host_stage);
  h->host_stage = nullptr;
  h->host_stage_bytes = 0;
}

int ouro_host_reserve(ouro_heap* h, uint32_t n) {
  if (!h) return OURO_ERR_ARG;
  std::lock_guard<std::mutex> lock(h->host_mu);
  // enough for ouro_alloc_host with per-request sizes and staged pointers
  return host_prepare(h, ((4ull * n + 255u) & ~size_t(255)) + 8ull * n);
}

int ouro_alloc_host(ouro_heap* h, uint32_t n, uint32_t size, const uint32_t* h_sizes, void** h_out, void** d_out,
                    int block, int slices, void* stream) {
  if (!h || !h_out || block <= 0 || block > 1024 || slices < 0 || slices > static_cast<int>(kHostSlicesMax))
    return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  std::lock_guard<std::mutex> lock(h->host_mu);
  const size_t sizes_bytes = h_sizes ? (4ull * n + 255u) & ~size_t(255) : 0u;
  int rc = host_prepare(h, sizes_bytes + (d_out ? 0u : 8ull * n));
  if (rc) return rc;
  uint32_t* d_sizes = h_sizes ? static_cast<uint32_t*>(h->host_stage) : nullptr;
  void** d_ptrs = d_out ? d_out : reinterpret_cast<void**>(static_cast<char*>(h->host_stage) + sizes_bytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t k = 0, m = 0;
  host_slice_plan(n, slices, &k, &m);
  host_enter(h, s);
  rc = dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    for (uint32_t j = 0; j < k; ++j) {
      const uint32_t o = j * m, c = n - o < m ? n - o : m;
      if (h_sizes) {
        cudaMemcpyAsync(d_sizes + o, h_sizes + o, 4ull * c, cudaMemcpyHostToDevice, h->host_in);
        cudaEventRecord(h->host_slice_in[j], h->host_in);
        cudaStreamWaitEvent(s, h->host_slice_in[j], 0);
      }
      k_alloc<V><<<grid_for(c, block), block, 0, s>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), c, size,
                                                         h_sizes ? d_sizes + o : nullptr, d_ptrs + o);
      cudaEventRecord(h->host_slice_run[j], s);
      cudaStreamWaitEvent(h->host_out, h->host_slice_run[j], 0);
      cudaMemcpyAsync(h_out + o, d_ptrs + o, 8ull * c, cudaMemcpyDeviceToHost, h->host_out);
    }
    return OURO_OK;
  });
  cudaEventRecord(h->host_joined, h->host_out);
  cudaStreamWaitEvent(s, h->host_joined, 0);   // host_in's copies all precede launches on s
  cudaEventRecord(h->host_done, s);
  return rc ? rc : cuda_rc(cudaGetLastError());
}

int ouro_free_host(ouro_heap* h, uint32_t n, void* const* h_ptrs, int block, int slices, void* stream) {
  if (!h || !h_ptrs || block <= 0 || block > 1024 || slices < 0 || slices > static_cast<int>(kHostSlicesMax))
    return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  std::lock_guard<std::mutex> lock(h->host_mu);
  int rc = host_prepare(h, 8ull * n);
  if (rc) return rc;
  void** d_ptrs = static_cast<void**>(h->host_stage);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t k = 0, m = 0;
  host_slice_plan(n, slices, &k, &m);
  host_enter(h, s);
  rc = dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    for (uint32_t j = 0; j < k; ++j) {
      const uint32_t o = j * m, c = n - o < m ? n - o : m;
      cudaMemcpyAsync(d_ptrs + o, h_ptrs + o, 8ull * c, cudaMemcpyHostToDevice, h->host_in);
      cudaEventRecord(h->host_slice_in[j], h->host_in);
      cudaStreamWaitEvent(s, h->host_slice_in[j], 0);
      k_free<V><<<grid_for(c, block), block, 0, s>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), c, d_ptrs + o);
    }
    return OURO_OK;
  });
  cudaEventRecord(h->host_done, s);
  return rc ? rc : cuda_rc(cudaGetLastError());
}

int ouro_trace(ouro_heap* h, const uint32_t* ops, uint64_t n_ops, uint64_t* results, uint32_t tid, uint32_t bid) {
  if (!h || !ops || !results || n_ops == 0 || tid >= 1024u) return OURO_ERR_ARG;
  for (uint64_t i = 0; i < n_ops; ++i) {
    // a free must name an earlier malloc; an initial-chunk enqueue or a page
    // free of such a chunk must name an earlier chunk allocation
    const uint32_t op = ops[2 * i], arg = ops[2 * i + 1];
    if (op > 4u) return OURO_ERR_ARG;
    if (op == 1u && (arg >= i || ops[2 * arg] != 0u)) return OURO_ERR_ARG;
    const uint64_t src = op == 3u ? (arg >> 14) : (arg >> 10);
    if ((op == 3u || op == 4u) && (src >= i || ops[2 * src] != 2u)) return OURO_ERR_ARG;
  }
  uint32_t* d_ops = nullptr;
  uint64_t* d_res = nullptr;
  void** d_ptrs = nullptr;
  if (cudaMalloc(&d_ops, 8 * n_ops) != cudaSuccess || cudaMalloc(&d_res, 8 * n_ops) != cudaSuccess ||
      cudaMalloc(&d_ptrs, 8 * n_ops) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(d_ops);
    cudaFree(d_res);
    return OURO_ERR_NOMEM;
  }
  cudaError_t e = cudaMemcpy(d_ops, ops, 8 * n_ops, cudaMemcpyHostToDevice);
  const uint32_t block = (tid / 32u + 1u) * 32u;
  if (e == cudaSuccess) {
    dispatch(h->variant, [&](auto v) {
      constexpr int V = decltype(v)::value;
      k_trace<V><<<bid + 1u, block>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), d_ops, n_ops, d_res, d_ptrs, tid, bid);
      return 0;
    });
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(results, d_res, 8 * n_ops, cudaMemcpyDeviceToHost);
  cudaFree(d_ops);
  cudaFree(d_res);
  cudaFree(d_ptrs);
  return cuda_rc(e);
}

int ouro_state(ouro_heap* h, uint64_t* out) {
  if (!h || !out) return OURO_ERR_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return OURO_ERR_CUDA;
  std::unique_ptr<HeapCore> core_buf(new HeapCore());   // ~0.5 MiB: not on the stack
  HeapCore& core = *core_buf;
  if (cudaMemcpy(&core, h->dev, sizeof(core), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  std::memset(out, 0, 151 * sizeof(uint64_t));
  out[0] = core.next_free_chunk.v;
  for (int i = 0; i < 2; ++i) {
    out[1 + 3 * i] = static_cast<uint64_t>(static_cast<int64_t>(core.reuse[i].count.v));
    out[2 + 3 * i] = core.reuse[i].front.v;
    out[3 + 3 * i] = core.reuse[i].back.v;
  }
  const int kind = h->variant / 2;
  const bool chunk_based = (h->variant % 2) == 1;
  const uint32_t vq_entries = static_cast<uint32_t>(h->L.vq_entries);
  std::vector<uint32_t> vq(vq_entries);
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    const ClassState& q = core.cls[c];
    uint64_t* o = out + 7 + 12 * c;
    o[0] = static_cast<uint64_t>(SemWord::count(q.sem.v));
    o[1] = 0;   // expected and reserved pages of the reference's semaphore: none at quiescence
    o[2] = q.holes > 0 ? static_cast<uint64_t>(q.holes) : 0u;
    o[3] = q.front.v;
    o[4] = q.back.v;
    o[5] = chunk_based && kind != 2 ? static_cast<uint64_t>(static_cast<int64_t>(q.entries.v)) : 0u;
    if (kind == 2) {
      o[6] = q.front_ptr;
      o[7] = q.back_ptr;
      o[8] = q.old_ptr;
      o[9] = q.old_count;
    }
    if (kind == 1) {
      if (cudaMemcpy(vq.data(), q.ring, vq_entries * 4u, cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
      uint64_t d = 0;
      for (uint32_t v = 0; v < vq_entries; ++v)
        if (vq[v] != kEmpty) d += static_cast<uint64_t>(v + 1u) * (static_cast<uint64_t>(vq[v]) + 1u);
      o[10] = d;
    }
    o[11] = q.ppc;
  }
  return OURO_OK;
}

int ouro_get_status(ouro_heap* h, ouro_heap_status* out, int clear) {
  if (!h || !out) return OURO_ERR_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return OURO_ERR_CUDA;
  std::unique_ptr<HeapCore> core_buf(new HeapCore());   // ~0.5 MiB: not on the stack
  HeapCore& core = *core_buf;
  if (cudaMemcpy(&core, h->dev, sizeof(core), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  out->flags = core.status.v;
  out->null_results = core.oom.v;
  out->timeouts = core.timeouts.v;
  out->chunk_allocs = core.chunk_allocs.v;
  out->next_free_chunk = core.next_free_chunk.v;
  out->timeout_sites = core.timeout_sites.v;
  if (clear) {
    const size_t off = offsetof(HeapCore, status);
    const size_t len = offsetof(HeapCore, chunk_allocs) - off;
    if (cudaMemset(reinterpret_cast<char*>(h->dev) + off, 0, len) != cudaSuccess) return OURO_ERR_CUDA;
  }
  return OURO_OK;
}

int ouro_write_pattern(void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed,
                       void* stream) {
  if (!d_ptrs) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  k_write_pattern<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_ptrs, n, size, d_sizes, seed);
  return cuda_rc(cudaGetLastError());
}

int ouro_verify_pattern(void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes, uint32_t seed,
                        unsigned long long* d_counters, void* stream) {
  if (!d_ptrs || !d_counters) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  k_verify_pattern<<<grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(d_ptrs, n, size, d_sizes, seed,
                                                                                    d_counters);
  return cuda_rc(cudaGetLastError());
}

int ouro_check_allocations(ouro_heap* h, void* const* d_ptrs, uint32_t n, uint32_t size, const uint32_t* d_sizes,
                           ouro_alloc_report* out) {
  if (!h || !d_ptrs || !out) return OURO_ERR_ARG;
  const size_t units = h->L.max_chunks * (kChunkBytes / 16u);
  const size_t words = (units + 31u) / 32u;
  uint32_t* bitmap = nullptr;
  unsigned long long* r = nullptr;
  if (cudaMalloc(&bitmap, words * 4u) != cudaSuccess || cudaMalloc(&r, 5 * sizeof(unsigned long long)) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(bitmap);
    return OURO_ERR_NOMEM;
  }
  cudaError_t e = cudaMemset(bitmap, 0, words * 4u);
  if (e == cudaSuccess) e = cudaMemset(r, 0, 5 * sizeof(unsigned long long));
  if (e == cudaSuccess && n) {
    k_check_allocs<<<grid_for(n, 256), 256>>>(h->dev, d_ptrs, n, size, d_sizes, bitmap, r);
    e = cudaGetLastError();
  }
  unsigned long long hr[5] = {0, 0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(hr, r, sizeof(hr), cudaMemcpyDeviceToHost);
  cudaFree(bitmap);
  cudaFree(r);
  out->checked = hr[0];
  out->nulls = hr[1];
  out->out_of_heap = hr[2];
  out->misaligned = hr[3];
  out->overlaps = hr[4];
  return cuda_rc(e);
}

int ouro_check_heap(ouro_heap* h, ouro_heap_report* out) {
  if (!h || !out) return OURO_ERR_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return OURO_ERR_CUDA;
  std::unique_ptr<HeapCore> core_buf(new HeapCore());   // ~0.5 MiB: not on the stack
  HeapCore& core = *core_buf;
  if (cudaMemcpy(&core, h->dev, sizeof(core), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  uint64_t nchunks = core.next_free_chunk.v < h->L.max_chunks ? core.next_free_chunk.v : h->L.max_chunks;
  unsigned long long* r = nullptr;
  if (cudaMalloc(&r, 26 * sizeof(unsigned long long)) != cudaSuccess) return OURO_ERR_NOMEM;
  cudaError_t e = cudaMemset(r, 0, 26 * sizeof(unsigned long long));
  const bool chunk_based = (h->variant % 2) == 1;
  if (e == cudaSuccess && nchunks) {
    k_check_heap<<<1184, 256>>>(h->dev, nchunks, chunk_based, r);
    e = cudaGetLastError();
  }
  unsigned long long hr[26];
  if (e == cudaSuccess) e = cudaMemcpy(hr, r, sizeof(hr), cudaMemcpyDeviceToHost);
  cudaFree(r);
  if (e != cudaSuccess) return OURO_ERR_CUDA;
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    const ClassState& q = core.cls[c];
    out->owned_pages[c] = hr[c];
    out->free_pages_meta[c] = chunk_based ? hr[12 + c] : static_cast<uint64_t>(q.back.v - q.front.v);
    out->sem_count[c] = SemWord::count(q.sem.v);
    out->sem_expected[c] = 0;   // no expected pages: groups in deficit own the chunks they add
    out->sem_reserved[c] = 0;   // no reservations either: groups wait on supply
  }
  out->data_chunks = hr[24];
  out->bad = hr[25];
  return OURO_OK;
}


int ouro_prefill(ouro_heap* h, uint64_t size, uint64_t pages, uint64_t* out_pages, void* stream) {
  if (!h) return OURO_ERR_ARG;
  const int cls = size_class(size);
  if (cls < 0) return OURO_ERR_ARG;   // served by the CUDA device heap, nothing to pre-populate
  const uint32_t ppc = class_pages_per_chunk(static_cast<uint32_t>(cls));
  const unsigned long long chunks = (pages + ppc - 1u) / ppc;
  if (chunks >= h->L.max_chunks) return OURO_ERR_ARG;
  if (out_pages) *out_pages = 0;
  if (chunks == 0) return OURO_OK;
  // the work counter and the result live in the heap's control block: no
  // allocation, so no device-wide synchronization
  uint32_t* d_next = &h->dev->prefill_next.v;
  unsigned long long* d_done = &h->dev->prefill_done.v;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(d_next, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_done, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) {
    dispatch(h->variant, [&](auto v) {
      constexpr int V = decltype(v)::value;
      const unsigned warps = static_cast<unsigned>((chunks + 31u) / 32u);
      const unsigned blocks = warps < 148u * 8u ? (warps + 7u) / 8u : 148u;
      k_prefill<V><<<blocks, 256, 0, s>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), static_cast<uint32_t>(cls),
                                          static_cast<uint32_t>(chunks), d_next, d_done);
      return 0;
    });
    e = cudaGetLastError();
  }
  unsigned long long done = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&done, d_done, sizeof(done), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (out_pages) *out_pages = done * ppc;
  return cuda_rc(e);
}

int ouro_allocate_chunk(ouro_heap* h, uint32_t* out_chunk) {
  if (!h || !out_chunk) return OURO_ERR_ARG;
  unsigned long long* d_r = &h->dev->prefill_done.v;
  dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_allocate_chunk<V><<<1, 1>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), d_r);
    return 0;
  });
  unsigned long long r = ~0ull;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&r, d_r, sizeof(r), cudaMemcpyDeviceToHost);
  *out_chunk = r == ~0ull ? 0xFFFFFFFFu : static_cast<uint32_t>(r);
  return cuda_rc(e);
}

int ouro_enqueue_initial_chunk(ouro_heap* h, uint32_t queue_index, uint32_t chunk_index, uint32_t available_pages) {
  if (!h || queue_index >= 10u || chunk_index + 1ull >= h->L.max_chunks) return OURO_ERR_ARG;
  const uint32_t ppc = class_pages_per_chunk(queue_index);
  if (available_pages == 0u || available_pages > ppc) return OURO_ERR_ARG;
  unsigned long long* d_r = &h->dev->prefill_done.v;
  dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_enqueue_initial<V><<<1, 1>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), queue_index, chunk_index,
                                   available_pages, d_r);
    return 0;
  });
  unsigned long long r = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&r, d_r, sizeof(r), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return OURO_ERR_CUDA;
  return r ? OURO_OK : OURO_ERR_DEVICE;
}

int ouro_free_resources(ouro_heap* h, ouro_free_report* out) {
  if (!h || !out) return OURO_ERR_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return OURO_ERR_CUDA;
  std::unique_ptr<HeapCore> core_buf(new HeapCore());   // ~0.5 MiB: not on the stack
  HeapCore& core = *core_buf;
  if (cudaMemcpy(&core, h->dev, sizeof(core), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  std::memset(out, 0, sizeof(*out));
  unsigned long long free_bytes = 0;
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    const ClassState& q = core.cls[c];
    out->page_size[c] = q.page_size;
    out->free_pages[c] = SemWord::count(q.sem.v);
    out->queue_entries[c] = static_cast<uint32_t>(q.back.v - q.front.v);
    if (out->free_pages[c] > 0) free_bytes += static_cast<unsigned long long>(out->free_pages[c]) * q.page_size;
  }
  const unsigned long long usable = h->L.max_chunks - 1u;
  const unsigned long long bumped = core.next_free_chunk.v < usable ? core.next_free_chunk.v : usable;
  const long long pooled0 = core.reuse[0].count.v > 0 ? core.reuse[0].count.v : 0;
  const long long pooled1 = core.reuse[1].count.v > 0 ? core.reuse[1].count.v : 0;
  const unsigned long long pooled = static_cast<unsigned long long>(pooled0) + 4ull * static_cast<unsigned long long>(pooled1);
  out->heap_chunks = usable;
  out->chunks_untouched = usable - bumped;
  out->chunks_pooled = pooled;
  out->chunks_in_use = bumped > pooled ? bumped - pooled : 0;
  out->free_bytes = free_bytes + (out->chunks_untouched + pooled) * kChunkBytes;
  return OURO_OK;
}

// Diagnostic counters of the chunk-based allocation path (zero unless the
// library was built with OURO_SCAN_STATS); no counterpart in the reference.
int ouro_scan_stats(ouro_heap* h, uint64_t* out, int clear) {
  if (!h || !out) return OURO_ERR_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return OURO_ERR_CUDA;
  Line<unsigned long long> v[kScanCounters];
  if (cudaMemcpy(v, h->dev->scan, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  for (uint32_t i = 0; i < kScanCounters; ++i) out[i] = v[i].v;
  if (clear && cudaMemset(h->dev->scan, 0, sizeof(v)) != cudaSuccess) return OURO_ERR_CUDA;
  return OURO_OK;
}

int ouro_measure_atomics(int mode, double* gops) {
  if (!gops || mode < 0 || mode > 4) return OURO_ERR_ARG;
  int sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return OURO_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const uint32_t N = 1u << 22;   // 16 MiB: L2 resident
  uint32_t* a = nullptr;
  if (cudaMalloc(&a, N * 4u + 256u) != cudaSuccess) return OURO_ERR_NOMEM;
  uint32_t* sink = a + N;
  unsigned long long* a64 = reinterpret_cast<unsigned long long*>(a + N + 32u);
  cudaMemset(a, 0, N * 4u + 256u);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = sms * 8, block = 256;
  const int iters = mode == 0 ? 64 : 16;
  auto launch = [&]() {
    if (mode == 0) k_peak_distinct<<<grid, block>>>(a, N - 1u, iters, sink);
    else k_peak_hot<<<grid, block>>>(a, a64, iters, mode == 2, mode == 3 ? 32u : mode == 4 ? 64u : 0u, sink);
  };
  launch();
  cudaEventRecord(e0);
  for (int r = 0; r < 5; ++r) launch();
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double ops = 5.0 * grid * block * static_cast<double>(iters) / (mode == 0 ? 1.0 : 32.0);
  *gops = ops / (ms * 1e-3) / 1e9;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  return cuda_rc(e);
}

// ------------------------------------------------ allocation-free checker
//
// ouro_check_allocations takes its ownership bitmap (one bit per 16 bytes of
// the heap) from cudaMalloc and gives it back with cudaFree.  Some callers
// cannot do either: a serving loop that must not stall its other streams
// (cudaFree waits for the whole device), and a process whose allocator heap
// and caching allocator already hold nearly all of HBM, where the bitmap
// allocation itself fails exactly when a check is most wanted.  For them the
// bitmap lives in the fixed array below, part of this library's device image:
// every GPU that loads the library holds its 8 MiB until the process exits.
// 8 MiB covers 2^26 units of 16 bytes, i.e. heaps of up to 1 GiB of chunk
// data; larger heaps are refused.

constexpr size_t kNoAllocBitmapWords = OURO_NOALLOC_BITMAP_BYTES / sizeof(uint32_t);
static __device__ __align__(256) uint32_t ouro_noalloc_bitmap[kNoAllocBitmapWords];

namespace {

// Device address of ouro_noalloc_bitmap on each device.  On the host the
// array's name is only a stand-in for the device object, so the address is
// asked from the runtime once per device, with that device current, and kept
// together with the context it belongs to: after a cudaDeviceReset the
// device's next context loads the library's module again, at an address the
// old one says nothing about, so a changed context means a fresh look-up.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
  void* ctx;
  uint32_t* addr;
};
NoAllocSlot g_noalloc[kNoAllocMaxDevices] = {};

// The driver's cuCtxGetCurrent, reached through the runtime so that the
// library does not link the driver library itself.
using CtxGetCurrent = int (*)(void**);
CtxGetCurrent ctx_get_current() {
  static CtxGetCurrent fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult st;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &st) != cudaSuccess ||
        st != cudaDriverEntryPointSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<CtxGetCurrent>(p);
  }();
  return fn;
}

void* current_context() {
  void* ctx = nullptr;
  const CtxGetCurrent fn = ctx_get_current();
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

int noalloc_bitmap(int device, uint32_t** out) {
  if (device < 0 || device >= kNoAllocMaxDevices) return OURO_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& slot = g_noalloc[device];
  void* ctx = current_context();
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, ouro_noalloc_bitmap);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      return OURO_ERR_CUDA;
    }
    slot.addr = static_cast<uint32_t*>(p);
    slot.ctx = ctx ? ctx : current_context();   // the look-up made the context current
  }
  *out = slot.addr;
  return OURO_OK;
}

}  // namespace

int ouro_check_allocations_noalloc(ouro_heap* h, void* const* d_ptrs, uint32_t n, uint32_t size,
                                   const uint32_t* d_sizes, ouro_alloc_report* d_report, void* stream) {
  if (!h || !d_ptrs || !d_report) return OURO_ERR_ARG;
  int device = -1;
  if (cudaGetDevice(&device) != cudaSuccess) return OURO_ERR_CUDA;
  if (device != h->device) return OURO_ERR_ARG;
  const size_t words = (h->L.max_chunks * (kChunkBytes / 16u) + 31u) / 32u;
  if (words > kNoAllocBitmapWords) return OURO_ERR_TOO_LARGE;
  uint32_t* bitmap = nullptr;
  const int rc = noalloc_bitmap(device, &bitmap);
  if (rc != OURO_OK) return rc;
  // The array keeps what the previous call left: clear the part this heap
  // uses, and the caller's report, which the kernel accumulates into.
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(bitmap, 0, words * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_report, 0, sizeof(ouro_alloc_report), s);
  if (e == cudaSuccess && n) {
    k_check_allocs<<<grid_for(n, 256), 256, 0, s>>>(h->dev, d_ptrs, n, size, d_sizes, bitmap,
                                                    reinterpret_cast<unsigned long long*>(d_report));
    e = cudaGetLastError();
  }
  return cuda_rc(e);
}

}  // extern "C"
