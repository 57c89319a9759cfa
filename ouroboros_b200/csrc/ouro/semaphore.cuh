// semaphore.cuh -- the per-class page semaphore.
//
// Same protocol as the reference's BulkSemaphore (BulkSemaphore_impl.cuh:
// 116-232): a packed word of (count, expected, reserved); a fast path that
// subtracts the group's demand, and a CAS path that either claims, reserves
// and waits, or elects the group to allocate chunks.  Differences: the fields
// are repacked (count 26 bits biased by 2^25, expected counted in whole chunks
// with 19 bits, reserved 19 bits) so that neither expected nor reserved can
// overflow at B200 thread counts; a group may allocate several chunks in one
// election; every wait is bounded; allocation failure ends in a partial grant
// instead of undefined behaviour.
#pragma once

#include "heap.cuh"

namespace ouro {

struct SemWord {
  static constexpr unsigned long long kCntMask = (1ull << 26) - 1u;
  static constexpr unsigned long long kBias = 1ull << 25;
  static constexpr uint32_t kExpShift = 26u;
  static constexpr uint32_t kResShift = 45u;
  static constexpr unsigned long long kFieldMask = (1ull << 19) - 1u;
  static constexpr unsigned long long kInit = kBias;
  static constexpr long long kMaxCount = (1ll << 25) - 1;

  __host__ __device__ static long long count(unsigned long long v) {
    return static_cast<long long>(v & kCntMask) - static_cast<long long>(kBias);
  }
  __host__ __device__ static uint32_t exp_chunks(unsigned long long v) {
    return static_cast<uint32_t>((v >> kExpShift) & kFieldMask);
  }
  __host__ __device__ static uint32_t reserved(unsigned long long v) {
    return static_cast<uint32_t>((v >> kResShift) & kFieldMask);
  }
  __host__ __device__ static unsigned long long make(long long c, uint32_t e, uint32_t r) {
    return static_cast<unsigned long long>(c + static_cast<long long>(kBias)) |
           (static_cast<unsigned long long>(e) << kExpShift) | (static_cast<unsigned long long>(r) << kResShift);
  }
  __host__ __device__ static unsigned long long sub(uint32_t n) { return ~static_cast<unsigned long long>(n) + 1ull; }
};

// count += pages (a free, or pages that arrived)
__device__ __forceinline__ void sem_signal(ClassState* q, uint32_t pages) {
  if (pages) atomicAdd(&q->sem.v, static_cast<unsigned long long>(pages));
}

// Chunks promised earlier arrived: count += got_pages, expected -= promised.
__device__ __forceinline__ void sem_fulfil(ClassState* q, uint32_t got_pages, uint32_t promised_chunks) {
  unsigned long long d = static_cast<unsigned long long>(got_pages) -
                         (static_cast<unsigned long long>(promised_chunks) << SemWord::kExpShift);
  atomicAdd(&q->sem.v, d);
}

// BulkSemaphore_impl.cuh:7-17 tryReduce
__device__ __forceinline__ bool sem_try_reduce(ClassState* q, uint32_t n) {
  if (n == 0) return true;
  unsigned long long old = atomicAdd(&q->sem.v, SemWord::sub(n));
  if (SemWord::count(old) - static_cast<long long>(n) < 0) {
    atomicAdd(&q->sem.v, static_cast<unsigned long long>(n));
    return false;
  }
  return true;
}

// Acquire g.size pages of class q for the group.  Collective over the group;
// the leader issues the atomics.  `grow(k)` is called collectively when the
// group is elected to add k chunks; it must publish the new pages and call
// sem_fulfil(q, pages, k), and return the number of chunks obtained.
// Returns the number of pages granted (g.size, or fewer after an allocation
// failure, 0 after a timeout).
template <typename Grow>
__device__ inline uint32_t sem_acquire(HeapCore* h, ClassState* q, const Group& g, Grow&& grow) {
  enum : uint32_t { kTake = 0, kAlloc = 1, kReserve = 2, kFail = 3 };
  const uint32_t n = static_cast<uint32_t>(g.size);
  const uint32_t ppc = q->ppc;
  bool first = true;
  bool failed_alloc = false;
  for (uint32_t round = 0;; ++round) {
    uint32_t mode = kFail, arg = 0;
    if (g.is_leader()) {
      if (round > kSpinLimit) {
        note_timeout(h, kWaitSemRounds);
        mode = kFail;
      } else {
        // fast path: one subtract (optimistic on the first round)
        bool try_fast = first || SemWord::count(ld_relaxed(&q->sem.v)) >= static_cast<long long>(n);
        first = false;
        unsigned long long v;
        bool done = false;
        if (try_fast && !failed_alloc) {
          v = atomicAdd(&q->sem.v, SemWord::sub(n));
          if (SemWord::count(v) >= static_cast<long long>(n)) {
            mode = kTake;
            arg = n;
            done = true;
          } else {
            atomicAdd(&q->sem.v, static_cast<unsigned long long>(n));
          }
        }
        if (!done) {
          v = ld_relaxed(&q->sem.v);
          for (uint32_t tries = 0;; ++tries) {
            long long c = SemWord::count(v);
            uint32_t e = SemWord::exp_chunks(v);
            uint32_t r = SemWord::reserved(v);
            long long avail = c + static_cast<long long>(e) * ppc - r;
            unsigned long long nv;
            if (failed_alloc) {
              // out of chunks: take whatever is there, once
              uint32_t m = c <= 0 ? 0u : (c < n ? static_cast<uint32_t>(c) : n);
              nv = SemWord::make(c - m, e, r);
              mode = kTake;
              arg = m;
            } else if (avail < static_cast<long long>(n)) {
              // Size the growth on the count without the transient dips of
              // other groups' fast-path attempts (they add their pages back),
              // so that a burst does not allocate chunks for phantom demand.
              const long long settled = (c < 0 ? 0 : c) + static_cast<long long>(e) * ppc - r;
              const long long deficit = static_cast<long long>(n) - settled;
              uint32_t k = deficit <= 0 ? 1u : static_cast<uint32_t>((deficit + ppc - 1) / ppc);
              if (k > n) k = n;
              nv = SemWord::make(c, e + k, r);
              mode = kAlloc;
              arg = k;
            } else if (c >= static_cast<long long>(n)) {
              nv = SemWord::make(c - n, e, r);
              mode = kTake;
              arg = n;
            } else {
              nv = SemWord::make(c, e, r + n);
              mode = kReserve;
              arg = n;
            }
            unsigned long long seen = atomicCAS(&q->sem.v, v, nv);
            if (seen == v) break;
            if (tries > kSpinLimit) { note_timeout(h, kWaitSemCas); mode = kFail; break; }
            // contended: back off before re-reading, so that thousands of
            // arriving warps do not turn the word into a CAS storm
            __nanosleep(16u << (tries < 6u ? tries : 6u));
            v = ld_relaxed(&q->sem.v);
          }
          if (mode == kReserve) {
            // wait until the pages are there or our reservation is no longer covered
            uint32_t it = 0;
            for (;;) {
              unsigned long long w = ld_relaxed(&q->sem.v);
              long long c = SemWord::count(w);
              long long cover = c + static_cast<long long>(SemWord::exp_chunks(w)) * ppc;
              if (c >= static_cast<long long>(n) || static_cast<long long>(SemWord::reserved(w)) >= cover) break;
              if (it >= kSpinLimit) { note_timeout(h, kWaitSemReserve); break; }
              backoff(it);
            }
            atomicAdd(&q->sem.v, SemWord::sub(0) - (static_cast<unsigned long long>(n) << SemWord::kResShift));
          }
        }
      }
    }
    mode = bcast(g, mode);
    arg = bcast(g, arg);
    if (mode == kTake) return arg;
    if (mode == kFail) return 0u;
    if (mode == kAlloc) {
      uint32_t got = grow(arg);
      if (got < arg) failed_alloc = true;
      failed_alloc = bcast(g, static_cast<uint32_t>(failed_alloc)) != 0u;
    }
  }
}

}  // namespace ouro
