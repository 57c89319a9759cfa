// batch.cu -- the batched path: persistent kernels that serve large arrays of
// mixed-size requests (no counterpart in the reference, whose only caller is
// its per-thread benchmark).
//
// The per-thread path forms warp groups from whatever sizes a warp's 32
// threads happen to ask for; with mixed sizes that is ~10 classes per warp,
// so every class's semaphore and ticket atomics are issued by groups of ~3
// lanes.  Here each block takes tiles of 4 x blockDim requests, bins them by
// size class in shared memory (a histogram, a prefix sum and a scatter of
// request indices), and serves the tile in binned order: consecutive lanes
// of a warp then ask for the same class, and a warp's 32 requests cost one
// semaphore and one ticket atomic.  Tiles are taken grid-stride by a
// persistent grid (no counter to reset, so launches can be captured in CUDA
// graphs).  Frees are binned by the class of the page they release.
#include <cuda_runtime.h>

#include <cmath>

#include "handle.h"

using namespace ouro;

namespace {

constexpr int kPer = 4;                        // requests per thread and tile
constexpr uint32_t kBins = kNumClasses + 1u;   // + the CUDA device heap

__device__ __forceinline__ uint32_t bin_of_size(uint64_t size) {
  const int c = size_class(size);
  return c < 0 ? kNumClasses : static_cast<uint32_t>(c);
}

// Class of the page p points into (kNumClasses for foreign pointers and null).
template <int V>
__device__ __forceinline__ uint32_t bin_of_ptr(const Ouroboros<V>* mm, const void* ptr) {
  const char* p = static_cast<const char*>(ptr);
  if (!p || p < mm->data || p >= mm->data_end) return kNumClasses;
  uint32_t c = static_cast<uint32_t>(static_cast<size_t>(p - mm->data) >> kChunkShift);
  const uint2 ph = ld_relaxed_v2(&mm->meta[c].page_size);   // page_size, head
  const int cls = ph.x ? size_class(ph.x) : -1;
  return cls < 0 ? kNumClasses : static_cast<uint32_t>(cls);
}

// Shared-memory binning of one tile.  bins[j] is the bin of the thread's j-th
// request (kBins: none); the request indices come out in `order`, grouped by
// bin.  Returns the tile's request count.
template <int BLOCK>
__device__ __forceinline__ void bin_tile(const uint32_t (&bins)[kPer], const uint32_t (&req)[kPer], uint32_t* hist,
                                         uint32_t* off, uint32_t* order) {
  uint32_t slot[kPer];
  if (threadIdx.x < kBins) hist[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPer; ++j) slot[j] = bins[j] < kBins ? atomicAdd(&hist[bins[j]], 1u) : 0u;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b < kBins; ++b) {
      off[b] = acc;
      acc += hist[b];
    }
    off[kBins] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPer; ++j)
    if (bins[j] < kBins) order[off[bins[j]] + slot[j]] = req[j];
  __syncthreads();
}

template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_alloc_batch(Ouroboros<V>* mm, const uint32_t* sizes, void** out,
                                                       uint32_t n) {
  constexpr uint32_t T = BLOCK * kPer;
  __shared__ uint32_t hist[kBins], off[kBins + 1];
  __shared__ uint32_t order[T];
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * T; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * T) {
    uint32_t bins[kPer], req[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const uint64_t i = t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x;
      req[j] = static_cast<uint32_t>(i);
      bins[j] = i < n ? bin_of_size(sizes[i]) : kBins;
    }
    bin_tile<BLOCK>(bins, req, hist, off, order);
    const uint32_t cnt = off[kBins];
    for (uint32_t k = threadIdx.x; k < cnt; k += BLOCK) {
      const uint32_t i = order[k];
      out[i] = mm->malloc(sizes[i]);
    }
    __syncthreads();
  }
}

template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_free_batch(Ouroboros<V>* mm, void* const* ptrs, uint32_t n) {
  constexpr uint32_t T = BLOCK * kPer;
  __shared__ uint32_t hist[kBins], off[kBins + 1];
  __shared__ uint32_t order[T];
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * T; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * T) {
    uint32_t bins[kPer], req[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const uint64_t i = t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x;
      req[j] = static_cast<uint32_t>(i);
      bins[j] = i < n && ptrs[i] ? bin_of_ptr(mm, ptrs[i]) : kBins;
    }
    bin_tile<BLOCK>(bins, req, hist, off, order);
    const uint32_t cnt = off[kBins];
    for (uint32_t k = threadIdx.x; k < cnt; k += BLOCK) mm->free(ptrs[order[k]]);
    __syncthreads();
  }
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

// One cycle of churn over a live set: request i is picked with probability
// fraction/1000 (hash of seed, cycle, i); a picked request frees its page and
// allocates one of a freshly drawn size.  Frees of a tile go first (binned by
// the class they release), then its allocations (binned by the new class).
template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_realloc_batch(Ouroboros<V>* mm, void** ptrs, uint32_t* sizes, uint32_t n,
                                                         uint64_t seed, uint32_t cycle, uint32_t fraction,
                                                         SizeDist dist) {
  constexpr uint32_t T = BLOCK * kPer;
  __shared__ uint32_t hist[kBins], off[kBins + 1];
  __shared__ uint32_t order[T];
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * T; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * T) {
    uint32_t bins[kPer], req[kPer], news[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const uint64_t i = t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x;
      req[j] = static_cast<uint32_t>(i);
      bins[j] = kBins;
      news[j] = 0;
      if (i < n) {
        const uint64_t r = mix64(seed ^ (static_cast<uint64_t>(cycle) << 32) ^ i);
        if ((r & 0x3FFu) < fraction * 1024u / 1000u) {
          news[j] = draw_size(dist, mix64(r));
          bins[j] = ptrs[i] ? bin_of_ptr(mm, ptrs[i]) : kBins;
          if (!ptrs[i]) bins[j] = kBins + 1u;   // picked, nothing to free
        }
      }
    }
    // frees (bins >= kBins are skipped by the binning)
    bin_tile<BLOCK>(bins, req, hist, off, order);
    for (uint32_t k = threadIdx.x; k < off[kBins]; k += BLOCK) mm->free(ptrs[order[k]]);
    __syncthreads();
    // allocations of the picked requests
#pragma unroll
    for (int j = 0; j < kPer; ++j) bins[j] = news[j] ? bin_of_size(news[j]) : kBins;
    bin_tile<BLOCK>(bins, req, hist, off, order);
#pragma unroll
    for (int j = 0; j < kPer; ++j)
      if (news[j]) sizes[req[j]] = news[j];
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < off[kBins]; k += BLOCK) {
      const uint32_t i = order[k];
      ptrs[i] = mm->malloc(sizes[i]);
    }
    __syncthreads();
  }
}

// Grid of a persistent batch kernel: resident blocks x SMs, capped by the tiles.
template <typename K>
unsigned batch_grid(K kernel, int block, uint32_t n, int blocks_per_sm) {
  int dev = 0, sms = 148, fit = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, block, 0);
  if (fit < 1) fit = 1;
  if (blocks_per_sm > 0 && blocks_per_sm < fit) fit = blocks_per_sm;
  const uint64_t tiles = (static_cast<uint64_t>(n) + static_cast<uint64_t>(block) * kPer - 1u) /
                         (static_cast<uint64_t>(block) * kPer);
  const uint64_t g = static_cast<uint64_t>(sms) * fit;
  return static_cast<unsigned>(tiles < g ? (tiles ? tiles : 1u) : g);
}

// Launch shape: the tuned one of the heap unless the caller names a block size.
void shape_of(const ouro_heap* h, int block, int* out_block, int* out_per_sm) {
  *out_block = block > 0 ? block : (h->batch_block > 0 ? h->batch_block : 256);
  *out_per_sm = block > 0 ? 0 : h->batch_per_sm;
}

template <typename Launch>
int with_block(int block, Launch&& launch) {
  switch (block) {
    case 128: return launch(std::integral_constant<int, 128>{});
    case 256: return launch(std::integral_constant<int, 256>{});
    case 512: return launch(std::integral_constant<int, 512>{});
    case 1024: return launch(std::integral_constant<int, 1024>{});
    default: return OURO_ERR_ARG;
  }
}

}  // namespace

extern "C" {

int ouro_alloc_batch(ouro_heap* h, const uint32_t* d_sizes, void** d_out, uint32_t n, int block, void* stream) {
  if (!h || !d_sizes || !d_out) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  int b = 0, per_sm = 0;
  shape_of(h, block, &b, &per_sm);
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    return with_block(b, [&](auto bb) {
      constexpr int B = decltype(bb)::value;
      const unsigned g = batch_grid(k_alloc_batch<V, B>, B, n, per_sm);
      k_alloc_batch<V, B><<<g, B, 0, static_cast<cudaStream_t>(stream)>>>(
          reinterpret_cast<Ouroboros<V>*>(h->dev), d_sizes, d_out, n);
      return cuda_rc(cudaGetLastError());
    });
  });
}

int ouro_free_batch(ouro_heap* h, void* const* d_ptrs, uint32_t n, int block, void* stream) {
  if (!h || !d_ptrs) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  int b = 0, per_sm = 0;
  shape_of(h, block, &b, &per_sm);
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    return with_block(b, [&](auto bb) {
      constexpr int B = decltype(bb)::value;
      const unsigned g = batch_grid(k_free_batch<V, B>, B, n, per_sm);
      k_free_batch<V, B><<<g, B, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<Ouroboros<V>*>(h->dev),
                                                                          d_ptrs, n);
      return cuda_rc(cudaGetLastError());
    });
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
  int b = 0, per_sm = 0;
  shape_of(h, block, &b, &per_sm);
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    return with_block(b, [&](auto bb) {
      constexpr int B = decltype(bb)::value;
      const unsigned g = batch_grid(k_realloc_batch<V, B>, B, n, per_sm);
      k_realloc_batch<V, B><<<g, B, 0, static_cast<cudaStream_t>(stream)>>>(
          reinterpret_cast<Ouroboros<V>*>(h->dev), d_ptrs, d_sizes, n, seed, cycle, fraction_permille, d);
      return cuda_rc(cudaGetLastError());
    });
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
  // the sizes of the sample: one realloc cycle that picks every request
  cudaMemset(ptrs, 0, static_cast<size_t>(n) * sizeof(void*));
  const ouro_size_dist dist{0, lo, hi, 0.0f};
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best_b = 256, best_s = 0, rc = OURO_OK;
  float best_ms = 1e30f;
  const int blocks[] = {128, 256, 512, 1024};
  const int per_sm[] = {0, 1, 2, 4};
  for (int b : blocks) {
    for (int s : per_sm) {
      h->batch_block = b;
      h->batch_per_sm = s;
      float ms_total = 0.f;
      for (int rep = 0; rep < 3 && rc == OURO_OK; ++rep) {
        // fresh sizes, all pages allocated, then all freed; only alloc + free timed
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
        best_s = s;
      }
    }
    if (rc != OURO_OK) break;
  }
  h->batch_block = best_b;
  h->batch_per_sm = best_s;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ptrs);
  cudaFree(sizes);
  if (out_block) *out_block = best_b;
  if (out_per_sm) *out_per_sm = best_s;
  if (out_mops) *out_mops = best_ms > 0.f ? 2.0 * 2.0 * n / (best_ms * 1e-3) / 1e6 : 0.0;
  return rc;
}

}  // extern "C"
