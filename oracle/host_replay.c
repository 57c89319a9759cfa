/*
 * host_replay.c -- host-allocator baseline, test and benchmark infrastructure only.
 *
 * The request pattern of one benchmark cell (n requests of one size, or a
 * size per request) replayed through the host's glibc malloc/free with T
 * threads: each thread takes a contiguous slice, mallocs every request, writes
 * and checks the same seeded uint32 pattern the GPU harness uses, then frees.
 * Reported beside the GPU numbers as the host-allocator baseline; it restates
 * no part of the reference.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <time.h>

typedef struct {
  uint32_t begin, end, size, seed;
  const uint32_t* sizes;
  void** ptrs;
  uint64_t bad, nulls;
  double alloc_s, free_s;
} slice_t;

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static uint32_t pattern(uint32_t i, uint32_t seed) {
  uint32_t x = (i ^ seed) | 1u;
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

static void* run(void* arg) {
  slice_t* s = (slice_t*)arg;
  double t0 = now();
  for (uint32_t i = s->begin; i < s->end; ++i) s->ptrs[i] = malloc(s->sizes ? s->sizes[i] : s->size);
  double t1 = now();
  for (uint32_t i = s->begin; i < s->end; ++i) {
    uint32_t* p = (uint32_t*)s->ptrs[i];
    if (!p) { s->nulls++; continue; }
    uint32_t words = (s->sizes ? s->sizes[i] : s->size) / 4u, v = pattern(i, s->seed);
    for (uint32_t w = 0; w < words; ++w) p[w] = v + w;
    for (uint32_t w = 0; w < words; ++w) s->bad += p[w] != v + w;
  }
  double t2 = now();
  for (uint32_t i = s->begin; i < s->end; ++i) free(s->ptrs[i]);
  double t3 = now();
  s->alloc_s = t1 - t0;
  s->free_s = t3 - t2;
  (void)t2;
  return NULL;
}

/* out[0] = alloc+free seconds (max over threads of each phase), out[1] = nulls,
 * out[2] = bad words.  Returns 0 on success. */
int host_replay(uint32_t n, uint32_t size, const uint32_t* sizes, uint32_t seed, int threads, double* out) {
  if (threads < 1 || threads > 1024 || !out) return 1;
  void** ptrs = (void**)calloc(n ? n : 1, sizeof(void*));
  slice_t* sl = (slice_t*)calloc((size_t)threads, sizeof(slice_t));
  pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
  if (!ptrs || !sl || !th) { free(ptrs); free(sl); free(th); return 2; }
  for (int t = 0; t < threads; ++t) {
    sl[t].begin = (uint32_t)((uint64_t)n * t / threads);
    sl[t].end = (uint32_t)((uint64_t)n * (t + 1) / threads);
    sl[t].size = size;
    sl[t].sizes = sizes;
    sl[t].seed = seed;
    sl[t].ptrs = ptrs;
    pthread_create(&th[t], NULL, run, &sl[t]);
  }
  double a = 0, f = 0;
  uint64_t bad = 0, nulls = 0;
  for (int t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    if (sl[t].alloc_s > a) a = sl[t].alloc_s;
    if (sl[t].free_s > f) f = sl[t].free_s;
    bad += sl[t].bad;
    nulls += sl[t].nulls;
  }
  out[0] = a + f;
  out[1] = (double)nulls;
  out[2] = (double)bad;
  free(ptrs);
  free(sl);
  free(th);
  return 0;
}
