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

#include <atomic>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

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
// Shared memory of one growth tile.
template <int BLOCK>
struct GrowTile {
  uint32_t hist[kBins], off[kBins + 1];
  uint32_t order[BLOCK * kPer];
};

// One tile of requests vertices[t0 .. t0 + BLOCK x kPer) (bounded by n):
// binned by the class of the new blocks in shared memory, then grown.  Every
// thread of the block calls it.
template <int V, int BLOCK>
__device__ __forceinline__ void grow_tile(Ouroboros<V>* mm, void** vptr, uint32_t* degree, const uint32_t* vertices,
                                          uint64_t t0, uint32_t n, uint32_t nv, uint64_t seed,
                                          unsigned long long* failed, GrowTile<BLOCK>& sm) {
  uint32_t bins[kPer], slot[kPer];
  if (threadIdx.x < kBins) sm.hist[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const uint64_t i = t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x;
    bins[j] = kBins;
    if (i < n) {
      const uint32_t d = ld_relaxed(&degree[vertices[i]]) & ~kLock;   // a hint: the class of the new block
      bins[j] = bin_of_size(4u * (2u * d < kMaxEdges ? 2u * d : kMaxEdges));
    }
    slot[j] = bins[j] < kBins ? atomicAdd(&sm.hist[bins[j]], 1u) : 0u;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t b = 0; b < kBins; ++b) {
      sm.off[b] = acc;
      acc += sm.hist[b];
    }
    sm.off[kBins] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPer; ++j)
    if (bins[j] < kBins) sm.order[sm.off[bins[j]] + slot[j]] = static_cast<uint32_t>(t0 + static_cast<uint64_t>(j) * BLOCK + threadIdx.x);
  __syncthreads();
  // Warps walk the binned order together: a lane takes a request, locks its
  // vertex (one attempt per round, so two lanes of a warp naming the same
  // vertex cannot wait on each other) and allocates the new block; then the
  // whole warp copies and appends the edges of every request won this round,
  // 32 edges at a time, so a warp does not wait on its largest vertex.
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t total = sm.off[kBins];
  for (uint32_t kb = threadIdx.x - lane; kb < total; kb += BLOCK) {
    const uint32_t k = kb + lane;
    uint32_t v = 0;
    bool pending = k < total;
    if (pending) v = vertices[sm.order[k]];
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
  __shared__ GrowTile<BLOCK> sm;
  for (uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * T; t0 < n; t0 += static_cast<uint64_t>(gridDim.x) * T)
    grow_tile<V, BLOCK>(mm, vptr, degree, vertices, t0, n, nv, seed, failed, sm);
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

// =============================================================== serving loop
// A persistent kernel serves batches of growth requests that host clients
// submit while it runs.  The host writes a batch descriptor into a ring in
// pinned, mapped host memory and then its sequence number; the kernel polls
// that ring (system-scope acquire loads), admits batches in arrival order while
// the heap's free bytes -- computed on the device from allocator state -- stay
// above a watermark (a batch is always admitted when none is in flight), and
// splits each admitted batch into tiles of 1,024 requests.  Every block takes
// tickets on the tile sequence, so tiles of different batches run side by
// side; the block that finishes a batch's last tile writes its completion,
// with %globaltimer stamps taken when the batch was seen, admitted and done,
// into a second mapped ring that the host polls.  No CUDA call sits between a
// client and the GPU: submitting is a host store.
struct ServeDesc {                 // host -> device, one per batch slot
  unsigned long long vertices;     // device address of n uint32 vertex ids
  uint32_t n, client;
  uint32_t ready;                  // sequence number + 1 once the fields are written
  uint32_t pad_;
};
struct ServeDone {                 // device -> host
  unsigned long long t_seen, t_start, t_done;   // ns, %globaltimer
  unsigned long long failed_allocs, lock_giveups;
  uint32_t n, client, held_back;
  uint32_t done;                   // sequence number + 1 once the fields are written
};
struct ServeBatch {                // device copy of a seen batch
  const uint32_t* vertices;
  uint32_t n, client, first_tile, ntiles, held_back;
  uint32_t done_tiles;
  unsigned long long t_seen, t_start;
  unsigned long long failed[2];
};
struct ServeState {
  Line<uint32_t> grabbed;          // tickets handed out on the tile sequence
  Line<uint32_t> admitted_tiles;   // tiles admitted so far (published by the scheduler)
  Line<uint32_t> tiles_done;
  Line<uint32_t> inflight;         // batches admitted and not finished
  Line<uint32_t> lock;             // scheduler try-lock
  Line<uint32_t> status;           // kServe* bits
  // owned by the lock holder
  uint32_t seen, admitted;
  unsigned long long held_back, batches_done, requests_done;
};
constexpr uint32_t kServeIdle = 1u;   // nothing to do for longer than the idle limit

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire_sys(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_sys(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_relaxed_sys(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys(uint32_t* p, uint32_t v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

// The heap's free bytes: free pages x page size over the classes, plus the
// chunks never handed out and the pooled ones (the figure of ouro_free_resources).
template <int V>
__device__ unsigned long long heap_free_bytes(const Ouroboros<V>* mm) {
  unsigned long long bytes = 0;
  for (uint32_t c = 0; c < kNumClasses; ++c) {
    const long long cnt = SemWord::count(ld_relaxed(&mm->cls[c].sem.v));
    if (cnt > 0) bytes += static_cast<unsigned long long>(cnt) * mm->cls[c].page_size;
  }
  const unsigned long long usable = mm->max_chunks - 1u;
  const unsigned long long bumped = ld_relaxed(&mm->next_free_chunk.v);
  const int32_t p0 = ld_relaxed(&mm->reuse[0].count.v), p1 = ld_relaxed(&mm->reuse[1].count.v);
  const unsigned long long pooled = (p0 > 0 ? p0 : 0) + 4ull * (p1 > 0 ? p1 : 0);
  return bytes + ((bumped < usable ? usable - bumped : 0ull) + pooled) * kChunkBytes;
}

struct ServeArgs {
  void** vptr;
  uint32_t* degree;
  uint32_t nv;
  uint64_t seed;
  ServeDesc* desc;                 // mapped host memory
  ServeDone* done;                 // mapped host memory
  const uint32_t* stop;            // mapped host memory: 1 once the host submits nothing more
  ServeState* st;
  ServeBatch* batches;             // ring entries, slot = sequence % ring
  uint32_t* tile_batch;            // tile_cap entries, slot = tile % tile_cap: the batch of a tile
  uint32_t ring, tile_cap, max_inflight;
  unsigned long long watermark_bytes, idle_ns;
};

// One round of the scheduler, run by one thread under the try-lock: take the
// batches that arrived, then admit in order.  Returns whether it did anything.
template <int V, uint32_t T>
__device__ bool serve_schedule(Ouroboros<V>* mm, const ServeArgs& a) {
  ServeState* st = a.st;
  if (atomicCAS(&st->lock.v, 0u, 1u) != 0u) return false;
  __threadfence();
  bool progress = false;
  uint32_t seen = st->seen, admitted = st->admitted;
  for (uint32_t k = 0; k < 64u; ++k) {
    ServeDesc* d = a.desc + (seen % a.ring);
    if (ld_acquire_sys(&d->ready) != seen + 1u) break;
    ServeBatch* b = a.batches + (seen % a.ring);
    b->vertices = reinterpret_cast<const uint32_t*>(ld_relaxed_sys(&d->vertices));
    b->n = ld_relaxed_sys(&d->n);
    b->client = ld_relaxed_sys(&d->client);
    b->t_seen = globaltimer();
    b->held_back = 0;
    b->done_tiles = 0;
    b->failed[0] = b->failed[1] = 0;
    ++seen;
    progress = true;
  }
  uint32_t A = st->admitted_tiles.v;
  while (admitted != seen) {
    ServeBatch* b = a.batches + (admitted % a.ring);
    const uint32_t ntiles = (b->n + T - 1u) / T;
    const uint32_t inflight = ld_relaxed(&st->inflight.v);
    if (inflight >= a.max_inflight) break;
    if (A + ntiles - ld_relaxed(&st->tiles_done.v) > a.tile_cap) break;
    if (inflight > 0u && heap_free_bytes(mm) < a.watermark_bytes) {
      if (!b->held_back) {   // deferred by the watermark: counted once per batch
        b->held_back = 1u;
        ++st->held_back;
      }
      break;
    }
    b->first_tile = A;
    b->ntiles = ntiles;
    b->t_start = globaltimer();
    for (uint32_t i = 0; i < ntiles; ++i) a.tile_batch[(A + i) % a.tile_cap] = admitted;
    atomicAdd(&st->inflight.v, 1u);
    A += ntiles;
    ++admitted;
    progress = true;
  }
  st->seen = seen;
  st->admitted = admitted;
  __threadfence();
  st_release(&st->admitted_tiles.v, A);
  __threadfence();
  atomicExch(&st->lock.v, 0u);
  return progress;
}

// Nothing more will come: the host has stopped submitting, every batch it
// submitted was seen and admitted, and none is in flight.
__device__ bool serve_drained(const ServeArgs& a) {
  ServeState* st = a.st;
  if (ld_acquire_sys(a.stop) == 0u) return false;
  if (atomicCAS(&st->lock.v, 0u, 1u) != 0u) return false;
  __threadfence();
  const uint32_t seen = st->seen;
  const bool more = ld_acquire_sys(&a.desc[seen % a.ring].ready) == seen + 1u;
  const bool idle = !more && st->admitted == seen && ld_relaxed(&st->inflight.v) == 0u;
  __threadfence();
  atomicExch(&st->lock.v, 0u);
  return idle;
}

template <int V, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_serve(Ouroboros<V>* mm, ServeArgs a) {
  constexpr uint32_t T = BLOCK * kPer;
  __shared__ GrowTile<BLOCK> sm;
  __shared__ uint32_t s_ticket, s_exit, s_n, s_first;
  __shared__ const uint32_t* s_vertices;
  __shared__ unsigned long long* s_failed;
  ServeState* st = a.st;
  for (;;) {
    if (threadIdx.x == 0) {
      // a ticket on the tile sequence; wait (bounded by the idle limit) until
      // that tile is admitted, doing scheduler rounds meanwhile
      const uint32_t t = atomicAdd(&st->grabbed.v, 1u);
      uint32_t ex = 0, it = 0;
      unsigned long long idle_since = globaltimer();
      while (static_cast<int32_t>(ld_acquire(&st->admitted_tiles.v) - t) <= 0) {
        if (serve_schedule<V, T>(mm, a)) {
          idle_since = globaltimer();
          it = 0;
          continue;
        }
        if (serve_drained(a)) {
          ex = 1u;
          break;
        }
        if (globaltimer() - idle_since > a.idle_ns) {
          atomicOr(&st->status.v, kServeIdle);
          ex = 1u;
          break;
        }
        backoff(it);
        if (it > 5u) it = 5u;   // keep polling every microsecond or so
      }
      s_ticket = t;
      s_exit = ex;
      if (!ex) {
        const uint32_t seq = ld_relaxed(&a.tile_batch[t % a.tile_cap]);
        ServeBatch* b = a.batches + (seq % a.ring);
        s_vertices = b->vertices;
        s_n = b->n;
        s_first = b->first_tile;
        s_failed = b->failed;
      }
    }
    __syncthreads();
    if (s_exit) return;
    grow_tile<V, BLOCK>(mm, a.vptr, a.degree, s_vertices, static_cast<uint64_t>(s_ticket - s_first) * T, s_n, a.nv,
                        a.seed, s_failed, sm);
    if (threadIdx.x == 0) {
      const uint32_t t = s_ticket;
      const uint32_t seq = ld_relaxed(&a.tile_batch[t % a.tile_cap]);
      ServeBatch* b = a.batches + (seq % a.ring);
      __threadfence();
      atomicAdd(&st->tiles_done.v, 1u);
      if (atomicAdd(&b->done_tiles, 1u) + 1u == b->ntiles) {
        // the batch's last tile: its completion goes to the host
        __threadfence();
        ServeDone* d = a.done + (seq % a.ring);
        d->t_seen = b->t_seen;
        d->t_start = b->t_start;
        d->t_done = globaltimer();
        d->failed_allocs = ld_relaxed(&b->failed[0]);
        d->lock_giveups = ld_relaxed(&b->failed[1]);
        d->n = b->n;
        d->client = b->client;
        d->held_back = b->held_back;
        __threadfence_system();
        st_release_sys(&d->done, seq + 1u);
        atomicAdd(&st->inflight.v, 0xFFFFFFFFu);
      }
    }
    __syncthreads();
  }
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

struct ouro_server {
  ouro_heap* h;
  cudaStream_t stream;
  char* host;                      // pinned, mapped: desc[ring] | done[ring] | stop
  ServeDesc* desc;
  ServeDone* done;
  volatile uint32_t* stop;
  char* dev;                       // ServeState | batches[ring] | tile_batch[tile_cap]
  uint32_t ring;
  uint64_t next_seq;               // host: sequence number of the next submission
  uint64_t oldest;                 // host: oldest submission not yet reported by poll
  std::vector<uint8_t> reported;
  bool stopped;
  cudaError_t launch_error;
};

namespace {
constexpr uint32_t kServeTileCap = 1u << 16;
}

extern "C" {

int ouro_serve_start(ouro_heap* h, void** d_vptr, uint32_t* d_degree, uint32_t nv, uint64_t seed,
                     const ouro_serve_config* cfg, ouro_server** out) {
  if (!h || !d_vptr || !d_degree || nv == 0 || !out) return OURO_ERR_ARG;
  *out = nullptr;
  ouro_serve_config c{4096u, 64u, 0, 0.10, 10.0};
  if (cfg) c = *cfg;
  if (c.ring == 0u || c.ring > (1u << 20) || c.max_inflight == 0u || c.watermark < 0.0 || c.watermark >= 1.0 ||
      !(c.idle_seconds > 0.0))
    return OURO_ERR_ARG;
  ouro_server* sv = new (std::nothrow) ouro_server();
  if (!sv) return OURO_ERR_NOMEM;
  sv->h = h;
  sv->ring = c.ring;
  sv->reported.assign(c.ring, 0u);
  const size_t host_bytes = c.ring * (sizeof(ServeDesc) + sizeof(ServeDone)) + 64u;
  const size_t dev_bytes = sizeof(ServeState) + c.ring * sizeof(ServeBatch) + kServeTileCap * sizeof(uint32_t);
  cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&sv->host), host_bytes, cudaHostAllocMapped);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    delete sv;
    return OURO_ERR_NOMEM;
  }
  std::memset(sv->host, 0, host_bytes);
  sv->desc = reinterpret_cast<ServeDesc*>(sv->host);
  sv->done = reinterpret_cast<ServeDone*>(sv->host + c.ring * sizeof(ServeDesc));
  sv->stop = reinterpret_cast<volatile uint32_t*>(sv->host + c.ring * (sizeof(ServeDesc) + sizeof(ServeDone)));
  char* host_d = nullptr;
  e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&host_d), sv->host, 0);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&sv->dev), dev_bytes);
  if (e == cudaSuccess) e = cudaMemset(sv->dev, 0, dev_bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFree(sv->dev);
    cudaFreeHost(sv->host);
    delete sv;
    return OURO_ERR_CUDA;
  }
  ServeArgs a;
  a.vptr = d_vptr;
  a.degree = d_degree;
  a.nv = nv;
  a.seed = seed;
  a.desc = reinterpret_cast<ServeDesc*>(host_d);
  a.done = reinterpret_cast<ServeDone*>(host_d + c.ring * sizeof(ServeDesc));
  a.stop = reinterpret_cast<const uint32_t*>(host_d + c.ring * (sizeof(ServeDesc) + sizeof(ServeDone)));
  a.st = reinterpret_cast<ServeState*>(sv->dev);
  a.batches = reinterpret_cast<ServeBatch*>(sv->dev + sizeof(ServeState));
  a.tile_batch = reinterpret_cast<uint32_t*>(sv->dev + sizeof(ServeState) + c.ring * sizeof(ServeBatch));
  a.ring = c.ring;
  a.tile_cap = kServeTileCap;
  a.max_inflight = c.max_inflight;
  a.watermark_bytes = static_cast<unsigned long long>(c.watermark * static_cast<double>(h->heap_bytes));
  a.idle_ns = static_cast<unsigned long long>(c.idle_seconds * 1e9);
  const int rc = dispatch(h->variant, [&](auto v) {
    constexpr int V = decltype(v)::value;
    constexpr int B = 256;
    int dev = 0, sms = 148, fit = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, k_serve<V, B>, B, 0);
    if (fit < 1) fit = 1;
    if (c.blocks_per_sm > 0 && c.blocks_per_sm < fit) fit = c.blocks_per_sm;
    k_serve<V, B><<<static_cast<unsigned>(sms * fit), B, 0, sv->stream>>>(reinterpret_cast<Ouroboros<V>*>(h->dev), a);
    return cuda_rc(cudaGetLastError());
  });
  if (rc != OURO_OK) {
    cudaStreamDestroy(sv->stream);
    cudaFree(sv->dev);
    cudaFreeHost(sv->host);
    delete sv;
    return rc;
  }
  *out = sv;
  return OURO_OK;
}

int ouro_serve_submit(ouro_server* sv, const uint32_t* d_vertices, uint32_t n, uint32_t client, uint64_t* out_seq) {
  if (!sv || !d_vertices || n == 0 || sv->stopped) return OURO_ERR_ARG;
  if (sv->next_seq - sv->oldest >= sv->ring) return OURO_ERR_FULL;
  const uint64_t seq = sv->next_seq;
  ServeDesc* d = sv->desc + (seq % sv->ring);
  d->vertices = reinterpret_cast<unsigned long long>(d_vertices);
  d->n = n;
  d->client = client;
  std::atomic_thread_fence(std::memory_order_release);
  reinterpret_cast<volatile uint32_t*>(&d->ready)[0] = static_cast<uint32_t>(seq + 1u);
  sv->next_seq = seq + 1u;
  if (out_seq) *out_seq = seq;
  return OURO_OK;
}

int ouro_serve_poll(ouro_server* sv, ouro_serve_result* out, uint32_t max, uint32_t* got) {
  if (!sv || !got || (max && !out)) return OURO_ERR_ARG;
  *got = 0;
  for (uint64_t seq = sv->oldest; seq < sv->next_seq && *got < max; ++seq) {
    const uint32_t slot = static_cast<uint32_t>(seq % sv->ring);
    if (sv->reported[slot]) continue;
    const volatile ServeDone* d = sv->done + slot;
    if (d->done != static_cast<uint32_t>(seq + 1u)) continue;
    std::atomic_thread_fence(std::memory_order_acquire);
    ouro_serve_result& r = out[(*got)++];
    r.seq = seq;
    r.client = d->client;
    r.n = d->n;
    r.t_seen_ns = d->t_seen;
    r.t_start_ns = d->t_start;
    r.t_done_ns = d->t_done;
    r.failed_allocs = d->failed_allocs;
    r.lock_giveups = d->lock_giveups;
    r.held_back = d->held_back;
    sv->reported[slot] = 1u;
  }
  while (sv->oldest < sv->next_seq && sv->reported[sv->oldest % sv->ring]) {
    sv->reported[sv->oldest % sv->ring] = 0u;
    ++sv->oldest;
  }
  return OURO_OK;
}

int ouro_serve_stop(ouro_server* sv, ouro_serve_stats* out) {
  if (!sv) return OURO_ERR_ARG;
  if (!sv->stopped) {
    std::atomic_thread_fence(std::memory_order_release);
    *sv->stop = 1u;
    sv->launch_error = cudaStreamSynchronize(sv->stream);
    sv->stopped = true;
  }
  if (sv->launch_error != cudaSuccess) return OURO_ERR_CUDA;
  ServeState st;
  if (cudaMemcpy(&st, sv->dev, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess) return OURO_ERR_CUDA;
  if (out) {
    out->batches_seen = st.seen;
    out->batches_admitted = st.admitted;
    out->held_back = st.held_back;
    out->status = st.status.v;
  }
  return st.status.v ? OURO_ERR_DEVICE : OURO_OK;
}

int ouro_serve_close(ouro_server* sv) {
  if (!sv) return OURO_ERR_ARG;
  int rc = OURO_OK;
  if (!sv->stopped) rc = ouro_serve_stop(sv, nullptr);
  cudaStreamDestroy(sv->stream);
  cudaFree(sv->dev);
  cudaFreeHost(sv->host);
  delete sv;
  return rc == OURO_ERR_DEVICE ? OURO_OK : rc;
}

}  // extern "C"
