// batch.cu -- the batched path: kernels that serve large arrays of mixed-size
// requests (no counterpart in the reference, whose only caller is its
// per-thread benchmark).
//
// The per-thread path forms warp groups from whatever sizes a warp's 32
// threads happen to ask for; with mixed sizes that is ~10 classes per warp,
// so every class's semaphore and queue work is done by groups of ~3 lanes,
// and the chunk queues in particular pay for every small group with its own
// scan run.  Measured on 2^22 log-uniform 16 B .. 8 KiB requests in a VAC
// heap, the same requests issued in class order allocate 5-7x faster.  So a
// batch is sorted by size class first -- a counting sort over the whole
// array: per-tile histograms in shared memory, one scan of the (class, tile)
// counts, a scatter of request indices -- and then served by one launch with
// a thread per request in sorted order: every warp but the one at each class
// boundary asks for one class with all 32 lanes.  Frees are sorted by the
// class of the page they release.  All launches are stream-ordered and keep
// no state outside the heap's scratch, so a whole batch cycle can be
// captured in a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <cmath>

#include "handle.h"

using namespace ouro;

namespace {

constexpr uint32_t kBins = kNumClasses + 1u;   // + the CUDA device heap
constexpr uint32_t kNone = 15u;                // a slot without a request
constexpr uint32_t kSortThreads = 256u;
constexpr uint32_t kSortPer = 16u;             // requests per thread in the sort kernels
constexpr uint32_t kSortTile = kSortThreads * kSortPer;

__device__ __forceinline__ uint32_t bin_of_size(uint64_t size) {
  const int c = size_class(size);
  return c < 0 ? kNumClasses : static_cast<uint32_t>(c);
}

// Class of the page p points into (kNumClasses for foreign pointers).
template <int V>
__device__ __forceinline__ uint32_t bin_of_ptr(const Ouroboros<V>* mm, const void* ptr) {
  const char* p = static_cast<const char*>(ptr);
  if (!p || p < mm->data || p >= mm->data_end) return kNumClasses;
  uint32_t c = static_cast<uint32_t>(static_cast<size_t>(p - mm->data) >> kChunkShift);
  const uint2 ph = ld_relaxed_v2(&mm->meta[c].page_size);   // page_size, head
  const int cls = ph.x ? size_class(ph.x) : -1;
  return cls < 0 ? kNumClasses : static_cast<uint32_t>(cls);
}

// splitmix64: a counter-based hash, so a cycle's choices need no stored state.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct SizeDist {
  int kind;          // 0 log-uniform [lo, hi] rounded up to 16 B; 1 Zipf over first-instance classes
  uint32_t lo, hi;
  float cdf[10];     // kind 1: cumulative class probabilities
};

__device__ __forceinline__ uint32_t draw_size(const SizeDist& d, uint64_t r) {
  const float u = static_cast<float>(r >> 40) * (1.0f / 16777216.0f);   // 24 random bits in [0, 1)
  if (d.kind == 1) {
    uint32_t k = 0;
    while (k < 9u && u >= d.cdf[k]) ++k;
    return 16u << k;
  }
  const float s = static_cast<float>(d.lo) * expf(u * logf(static_cast<float>(d.hi) / static_cast<float>(d.lo)));
  uint32_t v = static_cast<uint32_t>(s);
  v = v < d.lo ? d.lo : (v > d.hi ? d.hi : v);
  return (v + 15u) & ~15u;
}

// The sort key of request i, one functor per kind of batch.
struct AllocKey {
  const uint32_t* sizes;
  __device__ uint32_t operator()(uint64_t i) const { return bin_of_size(sizes[i]); }
};
template <int V>
struct FreeKey {
  const Ouroboros<V>* mm;
  void* const* ptrs;
  __device__ uint32_t operator()(uint64_t i) const {
    const void* p = ptrs[i];
    return p ? bin_of_ptr(mm, p) : kNone;
  }
};
// A churn cycle picks request i with probability fraction / 1000 (hash of
// seed, cycle and i).  Free phase: a picked request's old page; alloc phase:
// the picked request's new size, drawn and stored here.
struct Churn {
  uint64_t seed;
  uint32_t cycle, fraction;
  SizeDist dist;
  __device__ bool picked(uint64_t i, uint64_t* r) const {
    *r = mix64(seed ^ (static_cast<uint64_t>(cycle) << 32) ^ i);
    return (*r & 0x3FFu) < fraction * 1024u / 1000u;
  }
};
template <int V>
struct ChurnFreeKey {
  const Ouroboros<V>* mm;
  void* const* ptrs;
  Churn ch;
  __device__ uint32_t operator()(uint64_t i) const {
    uint64_t r;
    if (!ch.picked(i, &r)) return kNone;
    const void* p = ptrs[i];
    return p ? bin_of_ptr(mm, p) : kNone;
  }
};
struct ChurnAllocKey {
  uint32_t* sizes;
  Churn ch;
  __device__ uint32_t operator()(uint64_t i) const {
    uint64_t r;
    if (!ch.picked(i, &r)) return kNone;
    const uint32_t sz = draw_size(ch.dist, mix64(r));
    sizes[i] = sz;
    return bin_of_size(sz);
  }
};

// Scratch of a sort (in the heap's batch scratch): for every tile of
// kSortTile requests 16 counters, then one total, then the permutation.
struct SortScratch {
  uint32_t* counts;   // [tiles][16]: counts, then start positions
  uint32_t* total;    // requests with a key (not kNone)
  uint32_t* perm;     // [n]: request indices grouped by key
};

// Pass 1: per-tile histogram of the keys, in shared memory.
template <typename Key>
__global__ void __launch_bounds__(kSortThreads) k_sort_count(Key key, uint32_t n, uint32_t* counts) {
  __shared__ uint32_t hist[16];
  if (threadIdx.x < 16u) hist[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
  for (uint32_t j = 0; j < kSortPer; ++j) {
    const uint64_t i = base + j * kSortThreads + threadIdx.x;
    const uint32_t k = i < n ? key(i) : kNone;
    const uint32_t m = __match_any_sync(0xFFFFFFFFu, k);
    if (k != kNone && (m & ((1u << lane_id()) - 1u)) == 0u) atomicAdd(&hist[k], static_cast<uint32_t>(__popc(m)));
  }
  __syncthreads();
  if (threadIdx.x < 16u) counts[blockIdx.x * 16u + threadIdx.x] = hist[threadIdx.x];
}

// Pass 2 (one block): start position of every (key, tile) in key-major
// order, and the total.  Warp k scans key k's counts over the tiles.
__global__ void __launch_bounds__(512) k_sort_scan(uint32_t* counts, uint32_t tiles, uint32_t* total) {
  __shared__ uint32_t bin_total[16], bin_base[16];
  const uint32_t w = threadIdx.x >> 5, lane = lane_id();
  if (w < kBins) {
    uint32_t run = 0;
    for (uint32_t t0 = 0; t0 < tiles; t0 += 32u) {
      const uint32_t t = t0 + lane;
      const uint32_t c = t < tiles ? counts[t * 16u + w] : 0u;
      uint32_t incl = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (static_cast<int>(lane) >= d) incl += o;
      }
      if (t < tiles) counts[t * 16u + w] = run + incl - c;   // exclusive, within the key
      run += __shfl_sync(0xFFFFFFFFu, incl, 31);
    }
    if (lane == 0) bin_total[w] = run;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b < kBins; ++b) {
      bin_base[b] = acc;
      acc += bin_total[b];
    }
    *total = acc;
  }
  __syncthreads();
  if (w < kBins)
    for (uint32_t t = lane; t < tiles; t += 32u) counts[t * 16u + w] += bin_base[w];
}

// Pass 3: every request index to its place in the permutation.  Within a
// (key, tile) the order follows shared-memory atomics, so it is not stable;
// nothing depends on it.
template <typename Key>
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(Key key, uint32_t n, const uint32_t* counts,
                                                               uint32_t* perm) {
  __shared__ uint32_t cur[16];
  if (threadIdx.x < 16u) cur[threadIdx.x] = counts[blockIdx.x * 16u + threadIdx.x];
  __syncthreads();
  const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile;
  for (uint32_t j = 0; j < kSortPer; ++j) {
    const uint64_t i = base + j * kSortThreads + threadIdx.x;
    const uint32_t k = i < n ? key(i) : kNone;
    const uint32_t m = __match_any_sync(0xFFFFFFFFu, k);
    const int leader = __ffs(m) - 1;
    uint32_t pos = 0;
    if (k != kNone && static_cast<int>(lane_id()) == leader) pos = atomicAdd(&cur[k], static_cast<uint32_t>(__popc(m)));
    pos = __shfl_sync(m, pos, leader) + static_cast<uint32_t>(__popc(m & ((1u << lane_id()) - 1u)));
    if (k != kNone) perm[pos] = static_cast<uint32_t>(i);
  }
}

// Serving in sorted order: thread k takes the k-th request of the sort.
template <int V>
__global__ void k_alloc_sorted(Ouroboros<V>* mm, const uint32_t* perm, const uint32_t* total, const uint32_t* sizes,
                               void** out) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *total) return;
  const uint32_t i = perm[k];
  out[i] = mm->malloc(sizes[i]);
}

template <int V>
__global__ void k_free_sorted(Ouroboros<V>* mm, const uint32_t* perm, const uint32_t* total, void** ptrs,
                              bool clear) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= *total) return;
  const uint32_t i = perm[k];
  mm->free(ptrs[i]);
  if (clear) ptrs[i] = nullptr;
}

// Batch scratch of the heap, grown on demand: 16 counters per sort tile, the
// total and the permutation.  A call that needs more allocates it anew
// (cudaMalloc, so not while its stream is being captured: reserve first).
int batch_scratch(ouro_heap* h, uint32_t n, SortScratch* s) {
  const size_t tiles = (static_cast<size_t>(n) + kSortTile - 1u) / kSortTile;
  const size_t bytes = (tiles * 16u + 32u + static_cast<size_t>(n)) * sizeof(uint32_t);
  if (bytes > h->batch_scratch_bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return OURO_ERR_NOMEM;
    }
    if (h->batch_scratch) {
      cudaDeviceSynchronize();   // the old scratch may still be read by queued work
      cudaFree(h->batch_scratch);
    }
    h->batch_scratch = p;
    h->batch_scratch_bytes = bytes;
  }
  uint32_t* b = static_cast<uint32_t*>(h->batch_scratch);
  s->counts = b;
  s->total = b + tiles * 16u;
  s->perm = b + tiles * 16u + 32u;
  return OURO_OK;
}

// Counting sort of n requests by key into the heap's scratch (3 launches).
template <typename Key>
int sort_requests(const Key& key, uint32_t n, const SortScratch& s, cudaStream_t st) {
  const unsigned tiles = static_cast<unsigned>((static_cast<uint64_t>(n) + kSortTile - 1u) / kSortTile);
  k_sort_count<Key><<<tiles, kSortThreads, 0, st>>>(key, n, s.counts);
  k_sort_scan<<<1, 512, 0, st>>>(s.counts, tiles, s.total);
  k_sort_scatter<Key><<<tiles, kSortThreads, 0, st>>>(key, n, s.counts, s.perm);
  return cuda_rc(cudaGetLastError());
}

// Launch shape of the serving launch: the tuned one of the heap unless the
// caller names a block size.
int serve_block(const ouro_heap* h, int block) {
  const int b = block > 0 ? block : (h->batch_block > 0 ? h->batch_block : 256);
  return (b == 128 || b == 256 || b == 512 || b == 1024) ? b : -1;
}

}  // namespace

extern "C" {

int ouro_batch_reserve(ouro_heap* h, uint32_t n) {
  if (!h) return OURO_ERR_ARG;
  SortScratch s;
  return batch_scratch(h, n, &s);
}

int ouro_alloc_batch(ouro_heap* h, const uint32_t* d_sizes, void** d_out, uint32_t n, int block, void* stream) {
  if (!h || !d_sizes || !d_out) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  const int b = serve_block(h, block);
  if (b < 0) return OURO_ERR_ARG;
  SortScratch s;
  int rc = batch_scratch(h, n, &s);
  if (rc != OURO_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if ((rc = sort_requests(AllocKey{d_sizes}, n, s, st)) != OURO_OK) return rc;
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_alloc_sorted<V><<<grid_for(n, b), b, 0, st>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), s.perm, s.total,
                                                    d_sizes, d_out);
    return cuda_rc(cudaGetLastError());
  });
}

int ouro_free_batch(ouro_heap* h, void* const* d_ptrs, uint32_t n, int block, void* stream) {
  if (!h || !d_ptrs) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  const int b = serve_block(h, block);
  if (b < 0) return OURO_ERR_ARG;
  SortScratch s;
  int rc = batch_scratch(h, n, &s);
  if (rc != OURO_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    Ouroboros<V>* mm = reinterpret_cast<Ouroboros<V>*>(h->dev);
    int r = sort_requests(FreeKey<V>{mm, d_ptrs}, n, s, st);
    if (r != OURO_OK) return r;
    k_free_sorted<V><<<grid_for(n, b), b, 0, st>>>(mm, s.perm, s.total, const_cast<void**>(d_ptrs), false);
    return cuda_rc(cudaGetLastError());
  });
}

int ouro_realloc_batch(ouro_heap* h, void** d_ptrs, uint32_t* d_sizes, uint32_t n, uint64_t seed, uint32_t cycle,
                       uint32_t fraction_permille, const ouro_size_dist* dist, int block, void* stream) {
  if (!h || !d_ptrs || !d_sizes || !dist || fraction_permille > 1000u) return OURO_ERR_ARG;
  SizeDist d{};
  d.kind = dist->kind;
  d.lo = dist->lo;
  d.hi = dist->hi;
  if (d.kind == 0) {
    if (d.lo < 1u || d.hi < d.lo) return OURO_ERR_ARG;
  } else if (d.kind == 1) {
    if (!(dist->zipf_s > 0.0f)) return OURO_ERR_ARG;
    double w[10], total = 0;
    for (int k = 0; k < 10; ++k) total += (w[k] = 1.0 / std::pow(static_cast<double>(k + 1), dist->zipf_s));
    double acc = 0;
    for (int k = 0; k < 10; ++k) d.cdf[k] = static_cast<float>((acc += w[k]) / total);
    d.cdf[9] = 1.0f;
  } else {
    return OURO_ERR_ARG;
  }
  if (n == 0) return OURO_OK;
  const int b = serve_block(h, block);
  if (b < 0) return OURO_ERR_ARG;
  SortScratch s;
  int rc = batch_scratch(h, n, &s);
  if (rc != OURO_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Churn ch{seed, cycle, fraction_permille, d};
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    Ouroboros<V>* mm = reinterpret_cast<Ouroboros<V>*>(h->dev);
    // the picked requests' old pages, sorted by class, freed (pointers cleared)
    int r = sort_requests(ChurnFreeKey<V>{mm, d_ptrs, ch}, n, s, st);
    if (r != OURO_OK) return r;
    k_free_sorted<V><<<grid_for(n, b), b, 0, st>>>(mm, s.perm, s.total, d_ptrs, true);
    // their new sizes (drawn by the sort's key), sorted by class, allocated
    r = sort_requests(ChurnAllocKey{d_sizes, ch}, n, s, st);
    if (r != OURO_OK) return r;
    k_alloc_sorted<V><<<grid_for(n, b), b, 0, st>>>(mm, s.perm, s.total, d_sizes, d_ptrs);
    return cuda_rc(cudaGetLastError());
  });
}

int ouro_autotune_batch(ouro_heap* h, uint32_t n, uint32_t lo, uint32_t hi, int* out_block, int* out_per_sm,
                        double* out_mops) {
  if (!h || n == 0 || lo < 1u || hi < lo) return OURO_ERR_ARG;
  void** ptrs = nullptr;
  uint32_t* sizes = nullptr;
  if (cudaMalloc(&ptrs, static_cast<size_t>(n) * sizeof(void*)) != cudaSuccess ||
      cudaMalloc(&sizes, static_cast<size_t>(n) * sizeof(uint32_t)) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(ptrs);
    return OURO_ERR_NOMEM;
  }
  cudaMemset(ptrs, 0, static_cast<size_t>(n) * sizeof(void*));
  const ouro_size_dist dist{0, lo, hi, 0.0f};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best_b = 256, rc = OURO_OK;
  float best_ms = 1e30f;
  const int blocks[] = {128, 256, 512, 1024};
  for (int b : blocks) {
    h->batch_block = b;
    float ms_total = 0.f;
    for (int rep = 0; rep < 3 && rc == OURO_OK; ++rep) {
      // fresh sizes (one realloc cycle that picks every request), all of them
      // freed, then one timed alloc + free of the whole batch
      if ((rc = ouro_realloc_batch(h, ptrs, sizes, n, 0x5EEDull + static_cast<uint64_t>(rep), 0u, 1000u, &dist, 0,
                                   nullptr)) != OURO_OK)
        break;
      if ((rc = ouro_free_batch(h, ptrs, n, 0, nullptr)) != OURO_OK) break;
      cudaEventRecord(e0);
      rc = ouro_alloc_batch(h, sizes, ptrs, n, 0, nullptr);
      if (rc == OURO_OK) rc = ouro_free_batch(h, ptrs, n, 0, nullptr);
      cudaEventRecord(e1);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = OURO_ERR_CUDA;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) ms_total += ms;   // the first repetition warms the heap
      cudaMemset(ptrs, 0, static_cast<size_t>(n) * sizeof(void*));
    }
    if (rc != OURO_OK) break;
    if (ms_total < best_ms) {
      best_ms = ms_total;
      best_b = b;
    }
  }
  h->batch_block = best_b;
  h->batch_per_sm = 0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ptrs);
  cudaFree(sizes);
  if (out_block) *out_block = best_b;
  if (out_per_sm) *out_per_sm = 0;
  if (out_mops) *out_mops = best_ms > 0.f ? 2.0 * 2.0 * n / (best_ms * 1e-3) / 1e6 : 0.0;
  return rc;
}

int ouro_autotune_config(int variant, uint64_t heap_bytes, uint32_t n, uint32_t lo, uint32_t hi, uint32_t reps,
                         const uint32_t* queue_entries, uint32_t n_queue, const uint32_t* agg_widths,
                         uint32_t n_agg, const int* blocks, uint32_t n_blocks, ouro_tune_point* points,
                         ouro_tune_point* best) {
  if (variant < 0 || variant > 5 || n == 0 || lo < 1u || hi < lo || reps == 0 || !queue_entries || n_queue == 0 ||
      !agg_widths || n_agg == 0 || !blocks || n_blocks == 0 || !best)
    return OURO_ERR_ARG;
  for (uint32_t b = 0; b < n_blocks; ++b)
    if (blocks[b] != 128 && blocks[b] != 256 && blocks[b] != 512 && blocks[b] != 1024) return OURO_ERR_ARG;
  void** ptrs = nullptr;
  uint32_t* sizes = nullptr;
  if (cudaMalloc(&ptrs, static_cast<size_t>(n) * sizeof(void*)) != cudaSuccess ||
      cudaMalloc(&sizes, static_cast<size_t>(n) * sizeof(uint32_t)) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(ptrs);
    return OURO_ERR_NOMEM;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const ouro_size_dist dist{0, lo, hi, 0.0f};
  const bool linked = variant / 2 == 2;
  int rc = OURO_OK;
  best->ok = 0;
  best->mops = 0.0;
  for (uint32_t qi = 0; qi < n_queue && rc == OURO_OK; ++qi) {
    for (uint32_t ai = 0; ai < n_agg && rc == OURO_OK; ++ai) {
      ouro_config cfg;
      ouro_config_default(&cfg);
      if (variant / 2 == 0) cfg.page_queue_entries = queue_entries[qi];
      if (variant / 2 == 1) cfg.virtual_queue_entries = queue_entries[qi] / kQcSpots;
      cfg.agg_width = agg_widths[ai];
      ouro_heap* h = nullptr;
      // the linked-list variants have no queue arrays: one queue candidate
      const bool skip = linked && qi > 0;
      const int crc = skip ? OURO_ERR_ARG : ouro_create_config(variant, heap_bytes, &cfg, &h);
      if (crc == OURO_ERR_CUDA || crc == OURO_ERR_NOMEM) rc = crc;
      for (uint32_t bi = 0; bi < n_blocks; ++bi) {
        ouro_tune_point pt{cfg, blocks[bi], 0, 0.0};
        if (h && rc == OURO_OK) {
          cudaMemset(ptrs, 0, static_cast<size_t>(n) * sizeof(void*));
          // the sizes: one churn cycle that picks every request draws them
          // (and allocates them, which is the untimed repetition)
          int r = ouro_realloc_batch(h, ptrs, sizes, n, 0x5EEDull, 0u, 1000u, &dist, blocks[bi], nullptr);
          if (r == OURO_OK) r = ouro_free_batch(h, ptrs, n, blocks[bi], nullptr);
          float ms_total = 0.f;
          for (uint32_t rep = 0; rep < reps && r == OURO_OK; ++rep) {
            cudaEventRecord(e0);
            r = ouro_alloc_batch(h, sizes, ptrs, n, blocks[bi], nullptr);
            if (r == OURO_OK) r = ouro_free_batch(h, ptrs, n, blocks[bi], nullptr);
            cudaEventRecord(e1);
            if (r == OURO_OK && cudaEventSynchronize(e1) != cudaSuccess) r = OURO_ERR_CUDA;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms_total += ms;
          }
          ouro_heap_status st{};
          if (r == OURO_OK) r = ouro_get_status(h, &st, 0);
          if (r == OURO_ERR_CUDA) rc = r;
          pt.ok = r == OURO_OK && st.flags == 0u && st.null_results == 0u && ms_total > 0.f;
          pt.mops = ms_total > 0.f ? 2.0 * n * reps / (ms_total * 1e-3) / 1e6 : 0.0;
        }
        if (points) points[(qi * n_agg + ai) * n_blocks + bi] = pt;
        if (pt.ok && pt.mops > best->mops) *best = pt;
      }
      if (h) ouro_destroy(h);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ptrs);
  cudaFree(sizes);
  if (rc == OURO_OK && !best->ok) rc = OURO_ERR_DEVICE;
  return rc;
}

}  // extern "C"
