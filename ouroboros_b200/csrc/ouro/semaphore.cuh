// semaphore.cuh -- the per-class page semaphore.
//
// It plays the role of the reference's BulkSemaphore (BulkSemaphore_impl.cuh:
// 116-232): it counts a class's free pages, hands them to requesting groups
// and decides when chunks are added.  Its protocol is this build's own: a
// group never loops on a CAS of the hot word.
//
//   word = count (bits 0..37, biased by 2^37) | supply (bits 38..63, pages
//          ever added, mod 2^26; topmost, so that its carry leaves the word)
//
// * A group of n lanes takes n pages with ONE fetch-add of -n.  If the count
//   before it was >= n the pages are there: done (the warm path).
// * Otherwise the group keeps its demand: the count goes below zero and the
//   group owns the slice [max(-c0, 0), n - c0) of the class's deficit.  Every
//   multiple of pages-per-chunk inside its slice is a chunk that this group
//   adds itself.  Chunks being added always cover the deficit from 0 up to a
//   multiple of pages-per-chunk, so the chunks a burst needs are created once
//   each, in parallel, by the groups whose demand crossed them.  A lone thread
//   therefore adds a chunk exactly when the count is 0, which is the
//   reference's decision, so sequential replays stay bit-exact with it.
// * Adding pages (new chunks, frees, pre-fill) adds to count and supply in one
//   fetch-add.  The pages of a group that went into deficit exist once supply
//   has advanced by its slice end since its fetch-add, or once the count is
//   seen at or above zero; it waits for that (bounded) before it takes queue
//   entries.
// * Out of chunks: an addition that gets fewer chunks than it claimed adds the
//   pages it got and records the missing ones as holes of the class.  While
//   holes remain, waiting groups hand their demand back (paying holes down by
//   as much) and take what is there with fetch-adds (take_upto), retrying
//   while pages remain, so exactly the available pages are served and the
//   rest get nullptr.  The unbacked part of the deficit never exceeds the
//   holes, so a waiting group either sees its supply or sees holes.
// * Every wait is bounded and reports a timeout instead of hanging.
#pragma once

#include "heap.cuh"

namespace ouro {

struct SemWord {
  static constexpr uint32_t kCntBits = 38u;
  static constexpr unsigned long long kCntMask = (1ull << kCntBits) - 1u;
  static constexpr unsigned long long kBias = 1ull << (kCntBits - 1u);
  static constexpr uint32_t kSupShift = kCntBits;
  static constexpr uint32_t kSupBits = 64u - kSupShift;
  static constexpr unsigned long long kSupMask = (1ull << kSupBits) - 1u;
  static constexpr unsigned long long kInit = kBias;

  __host__ __device__ static long long count(unsigned long long v) {
    return static_cast<long long>(v & kCntMask) - static_cast<long long>(kBias);
  }
  __host__ __device__ static uint32_t supply(unsigned long long v) {
    return static_cast<uint32_t>((v >> kSupShift) & kSupMask);
  }
  // pages the supply field advanced from a to b (modular)
  __host__ __device__ static uint32_t supply_since(unsigned long long a, unsigned long long b) {
    return (supply(b) - supply(a)) & static_cast<uint32_t>(kSupMask);
  }
  // fetch-add operands: count -= n; count += n (a hand-back, not supply);
  // count += n and supply += n
  __host__ __device__ static unsigned long long take(uint32_t n) { return 0ull - static_cast<unsigned long long>(n); }
  __host__ __device__ static unsigned long long give(uint32_t n) { return static_cast<unsigned long long>(n); }
  __host__ __device__ static unsigned long long add(uint32_t n) {
    return static_cast<unsigned long long>(n) + (static_cast<unsigned long long>(n) << kSupShift);
  }
};

// Pages arrived (new chunks, a free, pre-fill): count += pages, supply += pages.
__device__ __forceinline__ void sem_signal(ClassState* q, uint32_t pages) {
  if (pages) atomicAdd(&q->sem.v, SemWord::add(pages));
}

// An addition of chunks got `missing` pages fewer than it claimed.
__device__ __forceinline__ void sem_mark_short(ClassState* q, uint32_t missing) {
  if (missing) atomicAdd(&q->holes, static_cast<int32_t>(missing));
}

// A waiting group hands back its demand of n pages: holes go down by as much,
// but not below zero.  One subtract, and the part that went below zero is
// added back; whatever the interleaving, the net effect of each hand-back is
// -max(holes it saw, 0) capped at n, so the count ends at max(holes - sum, 0)
// and only dips below zero in between (a waiter that reads the dip polls
// again).
__device__ __forceinline__ void sem_hand_back(ClassState* q, uint32_t n) {
  atomicAdd(&q->sem.v, SemWord::give(n));
  const int32_t old = atomicSub(&q->holes, static_cast<int32_t>(n));
  if (old < static_cast<int32_t>(n)) atomicAdd(&q->holes, static_cast<int32_t>(n) - (old > 0 ? old : 0));
}

// BulkSemaphore_impl.cuh:7-17 tryReduce: take n pages only if all of them are
// there.  Used by the standard chunk queue to hand a fully free chunk back to
// the pool; a CAS so that the count never dips for other groups (rare path).
__device__ __forceinline__ bool sem_try_reduce(ClassState* q, uint32_t n) {
  if (n == 0) return true;
  unsigned long long v = ld_relaxed(&q->sem.v);
  for (uint32_t tries = 0; tries < 64u; ++tries) {
    if (SemWord::count(v) < static_cast<long long>(n)) return false;
    const unsigned long long seen = atomicCAS(&q->sem.v, v, v + SemWord::take(n));
    if (seen == v) return true;
    v = seen;
  }
  return false;
}

// Take up to n pages that are there with fetch-adds only.  A group that took
// more than was there hands the excess back; if the count is positive after
// its hand-back (other groups' excess was in flight) and it still needs
// pages, it tries again after a short pause, so that many resolving groups do
// not keep the count oscillating.  Returns the pages taken.
__device__ inline uint32_t sem_take_upto(HeapCore* h, ClassState* q, uint32_t n) {
  uint32_t got = 0;
  for (uint32_t round = 0, it = 0; got < n && round < 4096u; ++round) {
    if (round) backoff(it);
    const uint32_t want = n - got;
    const unsigned long long old = atomicAdd(&q->sem.v, SemWord::take(want));
    const long long c0 = SemWord::count(old);
    const uint32_t t = c0 <= 0 ? 0u : (c0 < static_cast<long long>(want) ? static_cast<uint32_t>(c0) : want);
    got += t;
    if (t == want) break;
    const unsigned long long now = atomicAdd(&q->sem.v, SemWord::give(want - t)) + SemWord::give(want - t);
    if (SemWord::count(now) <= 0) break;
  }
  return got;
}

// Acquire g.size pages of class q for the group.  Collective over the group;
// the leader issues the atomics.  `grow(k)` is called collectively when the
// group has to add k chunks; it publishes the pages it got, adds them with
// sem_signal, and calls sem_mark_short with the pages it did not get.
// Returns the pages granted: g.size, or fewer when chunks ran out.
template <typename Grow>
__device__ inline uint32_t sem_acquire(HeapCore* h, ClassState* q, const Group& g, Grow&& grow) {
  const uint32_t n = static_cast<uint32_t>(g.size);
  const uint32_t ppc = q->ppc;
  uint32_t k = 0, b = 0;
  unsigned long long old = 0;
  if (g.is_leader()) {
    old = atomicAdd(&q->sem.v, SemWord::take(n));
    const long long c0 = SemWord::count(old);
    if (c0 < static_cast<long long>(n)) {
      const uint32_t a = c0 < 0 ? static_cast<uint32_t>(-c0) : 0u;
      b = static_cast<uint32_t>(static_cast<long long>(n) - c0);
      k = (b + ppc - 1u) / ppc - (a + ppc - 1u) / ppc;   // multiples of ppc in [a, b)
    }
  }
  k = bcast(g, k);
  if (k) grow(k);
  if (!bcast(g, b)) return n;
  // In deficit: wait until supply has covered the slice, or resolve against
  // what is there when an addition fell short.
  uint32_t granted = n;
  if (g.is_leader()) {
    uint32_t it = 0;
    for (;;) {
      // Covered once supply since the fetch-add reaches the slice end, or
      // once the count is back at or above zero: then every demand made so
      // far, this group's included, is backed by pages that are there (a
      // group ahead that handed its demand back moved the slice forward
      // without adding supply).
      const unsigned long long w = ld_relaxed(&q->sem.v);
      if (SemWord::supply_since(old, w) >= b || SemWord::count(w) >= 0) break;
      if (ld_relaxed(&q->holes) > 0) {
        sem_hand_back(q, n);
        granted = sem_take_upto(h, q, n);
        break;
      }
      if (it >= kSpinLimit) {
        note_timeout(h, kWaitSemReserve);
        atomicAdd(&q->sem.v, SemWord::give(n));
        granted = 0;
        break;
      }
      backoff(it);
    }
  }
  return bcast(g, granted);
}

}  // namespace ouro
