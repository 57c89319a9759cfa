// batch.cu -- the batched path: persistent kernels that serve large arrays of
// mixed-size requests (no counterpart in the reference, whose only caller is
// its per-thread benchmark).
//
// The per-thread path forms warp groups from whatever sizes a warp's 32
// threads happen to ask for; with mixed sizes that is ~10 classes per warp,
// so every class's semaphore and queue atomics are issued by groups of ~3
// lanes.  Here every warp takes tiles of 512 requests (16 per lane),
// counting-sorts the tile by size class in its own part of shared memory (a
// histogram and a scatter of request indices, match_any-ranked, no block
// barrier), and serves it in sorted order: the 32 lanes of a round then ask
// for one class (two at a class boundary), so a round costs one semaphore and
// one queue reservation instead of ten.  Each warp starts its sorted order at
// a different class (the class order is rotated by the warp's index), so the
// warps of the grid spread over the classes' hot lines at every moment
// instead of all serving the smallest class first.  Warps never wait for each
// other: a warp whose tile holds the slow large classes does not hold up the
// others.
// Tiles are taken grid-stride by a persistent grid (no counter to reset, so
// launches can be captured in CUDA graphs).  Frees are sorted by the class of
// the page they release.
#include <cuda_runtime.h>

#include <cmath>

#include "handle.h"

using namespace ouro;

namespace {

constexpr uint32_t kBins = kNumClasses + 1u;   // + the CUDA device heap
constexpr uint32_t kNone = 15u;                // a slot without a request
constexpr uint32_t kLaneSlots = 16u;           // requests per lane and tile
constexpr uint32_t kWarpTile = 32u * kLaneSlots;

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

// Shared memory of one warp: the sorted slot indices of its tile and the
// running offsets per bin.
struct WarpBins {
  uint16_t idx[kWarpTile];
  uint32_t cur[16];
};

// Counting sort of the warp's tile slots by key (key[j] of this lane's slot
// j, slot number j x 32 + lane; kNone: no request).  Writes the slot numbers
// grouped by key into w.idx, bins in the order rot, rot + 1, ... (mod kBins),
// and returns how many there are.  Ranks come from match_any, so the order
// within a key is the slot order.
__device__ __forceinline__ uint32_t warp_bin(WarpBins& w, const uint8_t (&key)[kLaneSlots], uint32_t rot) {
  const uint32_t lane = lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  if (lane < 16u) w.cur[lane] = 0;
  __syncwarp();
#pragma unroll
  for (uint32_t j = 0; j < kLaneSlots; ++j) {
    const uint32_t m = __match_any_sync(0xFFFFFFFFu, key[j]);
    if ((m & lt) == 0u && key[j] != kNone) w.cur[key[j]] += __popc(m);
    __syncwarp();
  }
  uint32_t total = 0;
  if (lane == 0) {
    for (uint32_t i = 0; i < kBins; ++i) {
      const uint32_t b = (rot + i) % kBins;
      const uint32_t c = w.cur[b];
      w.cur[b] = total;
      total += c;
    }
  }
  total = __shfl_sync(0xFFFFFFFFu, total, 0);
  __syncwarp();
#pragma unroll
  for (uint32_t j = 0; j < kLaneSlots; ++j) {
    const uint32_t m = __match_any_sync(0xFFFFFFFFu, key[j]);
    const uint32_t base = key[j] != kNone ? w.cur[key[j]] : 0u;
    __syncwarp();
    if (key[j] != kNone) {
      if ((m & lt) == 0u) w.cur[key[j]] = base + __popc(m);
      w.idx[base + __popc(m & lt)] = static_cast<uint16_t>(j * 32u + lane);
    }
    __syncwarp();
  }
  return total;
}

__device__ __forceinline__ uint32_t warp_global() {
  return (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ uint32_t warps_total() { return (gridDim.x * blockDim.x) >> 5; }

template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_alloc_batch(Ouroboros<V>* mm, const uint32_t* sizes, void** out,
                                                       uint32_t n) {
  __shared__ WarpBins bins[BLOCK / 32];
  WarpBins& w = bins[threadIdx.x >> 5];
  const uint32_t lane = lane_id();
  for (uint64_t t0 = static_cast<uint64_t>(warp_global()) * kWarpTile; t0 < n;
       t0 += static_cast<uint64_t>(warps_total()) * kWarpTile) {
    uint8_t key[kLaneSlots];
#pragma unroll
    for (uint32_t j = 0; j < kLaneSlots; ++j) {
      const uint64_t i = t0 + j * 32u + lane;
      key[j] = static_cast<uint8_t>(i < n ? bin_of_size(sizes[i]) : kNone);
    }
    const uint32_t total = warp_bin(w, key, warp_global() % kBins);
    for (uint32_t k = lane; k - lane < total; k += 32u) {
      if (k < total) {
        const uint64_t i = t0 + w.idx[k];
        out[i] = mm->malloc(sizes[i]);
      }
    }
    __syncwarp();
  }
}

template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_free_batch(Ouroboros<V>* mm, void* const* ptrs, uint32_t n) {
  __shared__ WarpBins bins[BLOCK / 32];
  WarpBins& w = bins[threadIdx.x >> 5];
  const uint32_t lane = lane_id();
  for (uint64_t t0 = static_cast<uint64_t>(warp_global()) * kWarpTile; t0 < n;
       t0 += static_cast<uint64_t>(warps_total()) * kWarpTile) {
    uint8_t key[kLaneSlots];
#pragma unroll
    for (uint32_t j = 0; j < kLaneSlots; ++j) {
      const uint64_t i = t0 + j * 32u + lane;
      const void* p = i < n ? ptrs[i] : nullptr;
      key[j] = static_cast<uint8_t>(p ? bin_of_ptr(mm, p) : kNone);
    }
    const uint32_t total = warp_bin(w, key, warp_global() % kBins);
    for (uint32_t k = lane; k - lane < total; k += 32u)
      if (k < total) mm->free(ptrs[t0 + w.idx[k]]);
    __syncwarp();
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
// allocates one of a freshly drawn size.  Per warp tile: the frees first,
// sorted by the class they release, then the allocations, sorted by the new
// class.
template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_realloc_batch(Ouroboros<V>* mm, void** ptrs, uint32_t* sizes, uint32_t n,
                                                         uint64_t seed, uint32_t cycle, uint32_t fraction,
                                                         SizeDist dist) {
  __shared__ WarpBins bins[BLOCK / 32];
  WarpBins& w = bins[threadIdx.x >> 5];
  const uint32_t lane = lane_id();
  for (uint64_t t0 = static_cast<uint64_t>(warp_global()) * kWarpTile; t0 < n;
       t0 += static_cast<uint64_t>(warps_total()) * kWarpTile) {
    uint8_t key[kLaneSlots];
    uint32_t picked = 0;   // bit j: slot j of this lane is picked
#pragma unroll
    for (uint32_t j = 0; j < kLaneSlots; ++j) {
      const uint64_t i = t0 + j * 32u + lane;
      key[j] = kNone;
      if (i < n) {
        const uint64_t r = mix64(seed ^ (static_cast<uint64_t>(cycle) << 32) ^ i);
        if ((r & 0x3FFu) < fraction * 1024u / 1000u) {
          picked |= 1u << j;
          const void* p = ptrs[i];
          if (p) key[j] = static_cast<uint8_t>(bin_of_ptr(mm, p));
        }
      }
    }
    uint32_t total = warp_bin(w, key, warp_global() % kBins);
    for (uint32_t k = lane; k - lane < total; k += 32u)
      if (k < total) mm->free(ptrs[t0 + w.idx[k]]);
    __syncwarp();
    // new sizes of the picked requests, then their allocations
#pragma unroll
    for (uint32_t j = 0; j < kLaneSlots; ++j) {
      key[j] = kNone;
      if (picked & (1u << j)) {
        const uint64_t i = t0 + j * 32u + lane;
        const uint64_t r = mix64(seed ^ (static_cast<uint64_t>(cycle) << 32) ^ i);
        const uint32_t sz = draw_size(dist, mix64(r));
        sizes[i] = sz;
        key[j] = static_cast<uint8_t>(bin_of_size(sz));
      }
    }
    __syncwarp();
    total = warp_bin(w, key, warp_global() % kBins);
    for (uint32_t k = lane; k - lane < total; k += 32u) {
      if (k < total) {
        const uint64_t i = t0 + w.idx[k];
        ptrs[i] = mm->malloc(sizes[i]);
      }
    }
    __syncwarp();
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
  const uint64_t per_block = static_cast<uint64_t>(block / 32) * kWarpTile;
  const uint64_t tiles = (static_cast<uint64_t>(n) + per_block - 1u) / per_block;
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
  const int blocks[] = {128, 256};
  const int per_sm[] = {0, 2, 4};
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
