// serve.cu -- the dynamic-graph workload behind the serving loop (no
// counterpart in the reference; its consumer, ouroGraph, lives outside the
// reference tree).
//
// A graph of nv vertices keeps each vertex's out-edges (uint32 vertex ids) in
// one allocation of this heap: vptr[v] points at degree[v] edges in a block of
// 4 x degree[v] bytes.  A growth request on v allocates a block of twice the
// edges (8 x d bytes, at most 8 KiB, i.e. 2048 edges), copies the d old edges,
// appends the new ones and frees the old block -- adjacency growth as a
// dynamic-graph framework does it.  Edge j of vertex v is a hash of (seed, v,
// j), so the content of a vertex's block depends only on how often it grew:
// the result of a batch is the same whether it runs alone or beside others
// that touch other vertices.  Growth kernels bin each tile by the size class
// of the new blocks, as the batched path does.
#include <cuda_runtime.h>

#include <cmath>

#include "handle.h"

using namespace ouro;

namespace {

constexpr int kPer = 4;
constexpr uint32_t kBins = kNumClasses + 1u;
constexpr uint32_t kMaxEdges = 2048u;   // 8 KiB of uint32 ids
constexpr uint32_t kLock = 1u << 31;     // degree[v] bit held while v grows

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ uint32_t edge_of(uint64_t seed, uint32_t v, uint32_t j, uint32_t nv) {
  return static_cast<uint32_t>(mix64(seed ^ (static_cast<uint64_t>(v) << 24) ^ j) % nv);
}

// Initial degree: a discrete power law P(d) ~ d^-alpha (d >= 1) drawn by
// inversion of the continuous one, capped at kMaxEdges / 2 so that every
// vertex can grow at least once.
__device__ __forceinline__ uint32_t degree_of(uint64_t seed, uint32_t v, float alpha) {
  const float u = (static_cast<float>(mix64(seed ^ 0xD15EA5Eull ^ v) >> 40) + 0.5f) * (1.0f / 16777216.0f);
  const float d = powf(u, -1.0f / (alpha - 1.0f));
  const uint32_t k = d >= static_cast<float>(kMaxEdges / 2u) ? kMaxEdges / 2u : static_cast<uint32_t>(d);
  return k < 1u ? 1u : k;
}

__global__ void k_graph_degrees(uint32_t* degree, uint32_t* bytes, uint32_t nv, uint64_t seed, float alpha) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const uint32_t d = degree_of(seed, v, alpha);
    degree[v] = d;
    bytes[v] = 4u * d;
  }
}

__global__ void k_graph_fill(void* const* vptr, const uint32_t* degree, uint32_t nv, uint64_t seed,
                             unsigned long long* failed) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    uint32_t* e = static_cast<uint32_t*>(vptr[v]);
    if (!e) {
      atomicAdd(failed, 1ull);
      continue;
    }
    for (uint32_t j = 0; j < degree[v]; ++j) e[j] = edge_of(seed, v, j, nv);
  }
}

__device__ __forceinline__ uint32_t bin_of_size(uint64_t size) {
  const int c = size_class(size);
  return c < 0 ? kNumClasses : static_cast<uint32_t>(c);
}

// Growth of the vertices vertices[0..n): tiles binned by the class of the new
// block.  A vertex at kMaxEdges is left as it is.  Batches in flight may name
// the same vertex (and a batch may name one twice): a growing vertex holds
// the top bit of its degree word, and a request that finds it held waits
// (bounded) for the other growth to finish; growth is deterministic, so the
// final content does not depend on the order.  failed[0] counts requests
// whose allocation returned nullptr (the vertex keeps its old block),
// failed[1] requests that gave up waiting for a vertex.
template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_graph_grow(Ouroboros<V>* mm, void** vptr, uint32_t* degree,
                                                      const uint32_t* vertices, uint32_t n, uint32_t nv,
                                                      uint64_t seed, unsigned long long* failed) {
  constexpr uint32_t T = BLOCK * kPer;
  __shared__ uint32_t hist[kBins], off[kBins + 1];
  __shared__ uint32_t order[T];
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * T; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * T) {
    uint32_t bins[kPer], slot[kPer];
    if (threadIdx.x < kBins) hist[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
      const uint64_t i = t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x;
      bins[j] = kBins;
      if (i < n) {
        const uint32_t d = ld_relaxed(&degree[vertices[i]]) & ~kLock;   // a hint: the class of the new block
        bins[j] = bin_of_size(4u * (2u * d < kMaxEdges ? 2u * d : kMaxEdges));
      }
      slot[j] = bins[j] < kBins ? atomicAdd(&hist[bins[j]], 1u) : 0u;
    }
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
      if (bins[j] < kBins) order[off[bins[j]] + slot[j]] = static_cast<uint32_t>(t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x);
    __syncthreads();
    // Warps walk the binned order together: a lane takes a request, locks its
    // vertex (one attempt per round, so two lanes of a warp naming the same
    // vertex cannot wait on each other) and allocates the new block; then the
    // whole warp copies and appends the edges of every request won this round,
    // 32 edges at a time, so a warp does not wait on its largest vertex.
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t kb = threadIdx.x - lane; kb < off[kBins]; kb += BLOCK) {
      const uint32_t k = kb + lane;
      uint32_t v = 0;
      bool pending = k < off[kBins];
      if (pending) v = vertices[order[k]];
      for (uint32_t round = 0, it = 0; __any_sync(0xFFFFFFFFu, pending); ++round) {
        bool won = false;
        uint32_t d = 0, nd = 0;
        uint32_t* p = nullptr;
        const uint32_t* old = nullptr;
        if (pending) {
          d = atomicOr(&degree[v], kLock);
          if (!(d & kLock)) {
            __threadfence();
            pending = false;
            nd = 2u * d < kMaxEdges ? 2u * d : kMaxEdges;
            if (d >= kMaxEdges) {
              st_release(&degree[v], d);   // full: nothing to grow
            } else if ((p = static_cast<uint32_t*>(mm->malloc(4u * nd))) == nullptr) {
              atomicAdd(&failed[0], 1ull);
              st_release(&degree[v], d);
            } else {
              old = static_cast<const uint32_t*>(vptr[v]);
              won = true;
            }
          } else if (round >= kSpinLimit) {   // gave up waiting for the vertex
            atomicAdd(&failed[1], 1ull);
            pending = false;
          }
        }
        for (uint32_t m = __ballot_sync(0xFFFFFFFFu, won); m; m &= m - 1u) {
          const int src = __ffs(m) - 1;
          uint32_t* pl = reinterpret_cast<uint32_t*>(__shfl_sync(0xFFFFFFFFu, reinterpret_cast<unsigned long long>(p), src));
          const uint32_t* ol =
              reinterpret_cast<const uint32_t*>(__shfl_sync(0xFFFFFFFFu, reinterpret_cast<unsigned long long>(old), src));
          const uint32_t dl = __shfl_sync(0xFFFFFFFFu, d, src), ndl = __shfl_sync(0xFFFFFFFFu, nd, src);
          const uint32_t vl = __shfl_sync(0xFFFFFFFFu, v, src);
          for (uint32_t j = lane; j < dl; j += 32u) pl[j] = ol[j];
          for (uint32_t j = dl + lane; j < ndl; j += 32u) pl[j] = edge_of(seed, vl, j, nv);
        }
        __threadfence();   // every lane's edges are visible before a winner publishes its block
        __syncwarp();
        if (won) {
          mm->free(const_cast<uint32_t*>(old));
          vptr[v] = p;
          __threadfence();
          st_release(&degree[v], nd);   // releases the vertex
        }
        if (__any_sync(0xFFFFFFFFu, pending)) backoff(it);
      }
    }
    __syncthreads();
  }
}

// Checksum of the edge blocks of vertices[0..n): the sum over their edges of
// a hash of (vertex, position, id); bad counts blocks whose edges differ from
// the recipe (the content a vertex of that degree must hold).
__global__ void k_graph_check(void* const* vptr, const uint32_t* degree, const uint32_t* vertices, uint32_t n,
                              uint32_t nv, uint64_t seed, unsigned long long* out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = vertices[i];
    const uint32_t* e = static_cast<const uint32_t*>(vptr[v]);
    if (!e) continue;
    unsigned long long sum = 0;
    uint32_t bad = 0;
    const uint32_t deg = degree[v] & ~kLock;
    for (uint32_t j = 0; j < deg; ++j) {
      sum += mix64((static_cast<uint64_t>(v) << 32) ^ (static_cast<uint64_t>(j) << 12) ^ e[j]);
      bad += e[j] != edge_of(seed, v, j, nv);
    }
    atomicAdd(&out[0], sum);
    if (bad) atomicAdd(&out[1], 1ull);
  }
}

template <int V>
__global__ void k_free_bytes(const Ouroboros<V>* mm, unsigned long long* dst) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long bytes = 0;
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    const long long cnt = SemWord::count(ld_relaxed(&mm->cls[c].sem.v));
    if (cnt > 0) bytes += static_cast<unsigned long long>(cnt) * mm->cls[c].page_size;
  }
  const unsigned long long usable = mm->max_chunks - 1u;
  const unsigned long long bumped = ld_relaxed(&mm->next_free_chunk.v);
  const int32_t p0 = ld_relaxed(&mm->reuse[0].count.v), p1 = ld_relaxed(&mm->reuse[1].count.v);
  const unsigned long long pooled = (p0 > 0 ? p0 : 0) + 4ull * (p1 > 0 ? p1 : 0);
  bytes += ((bumped < usable ? usable - bumped : 0ull) + pooled) * kChunkBytes;
  *dst = bytes;
}

template <typename K>
unsigned persistent_grid(K kernel, int block, uint64_t work, uint32_t per_block) {
  int dev = 0, sms = 148, fit = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, block, 0);
  if (fit < 1) fit = 1;
  const uint64_t tiles = (work + per_block - 1u) / per_block;
  const uint64_t g = static_cast<uint64_t>(sms) * fit;
  return static_cast<unsigned>(tiles < g ? (tiles ? tiles : 1u) : g);
}

}  // namespace

extern "C" {

int ouro_graph_init(ouro_heap* h, void** d_vptr, uint32_t* d_degree, uint32_t* d_scratch, uint32_t nv, uint64_t seed,
                    float alpha, unsigned long long* d_failed, void* stream) {
  if (!h || !d_vptr || !d_degree || !d_scratch || !d_failed || nv == 0 || !(alpha > 1.0f)) return OURO_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned grid = grid_for(nv, 256) < 148u * 16u ? grid_for(nv, 256) : 148u * 16u;
  k_graph_degrees<<<grid, 256, 0, s>>>(d_degree, d_scratch, nv, seed, alpha);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return OURO_ERR_CUDA;
  const int rc = ouro_alloc_batch(h, d_scratch, d_vptr, nv, 0, stream);
  if (rc != OURO_OK) return rc;
  k_graph_fill<<<grid, 256, 0, s>>>(d_vptr, d_degree, nv, seed, d_failed);
  return cuda_rc(cudaGetLastError());
}

int ouro_graph_grow(ouro_heap* h, void** d_vptr, uint32_t* d_degree, const uint32_t* d_vertices, uint32_t n, uint32_t nv,
                    uint64_t seed, unsigned long long* d_failed, void* stream) {
  if (!h || !d_vptr || !d_degree || !d_vertices || !d_failed) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    constexpr int B = 256;
    const unsigned g = persistent_grid(k_graph_grow<V, B>, B, n, B * kPer);
    k_graph_grow<V, B><<<g, B, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<Ouroboros<V>*>(h->dev), d_vptr, d_degree, d_vertices, n, nv, seed, d_failed);
    return cuda_rc(cudaGetLastError());
  });
}

int ouro_graph_check(void* const* d_vptr, const uint32_t* d_degree, const uint32_t* d_vertices, uint32_t n, uint32_t nv,
                     uint64_t seed, unsigned long long* d_out2, void* stream) {
  if (!d_vptr || !d_degree || !d_vertices || !d_out2) return OURO_ERR_ARG;
  if (n == 0) return OURO_OK;
  const unsigned grid = grid_for(n, 256) < 148u * 16u ? grid_for(n, 256) : 148u * 16u;
  k_graph_check<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(d_vptr, d_degree, d_vertices, n, nv, seed, d_out2);
  return cuda_rc(cudaGetLastError());
}

int ouro_free_bytes_to(ouro_heap* h, unsigned long long* dst, void* stream) {
  if (!h || !dst) return OURO_ERR_ARG;
  return dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    k_free_bytes<V><<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const Ouroboros<V>*>(h->dev), dst);
    return cuda_rc(cudaGetLastError());
  });
}

}  // extern "C"
