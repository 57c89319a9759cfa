// A C++ client of the serving loop, through the C ABI only: a graph in a
// page-based virtualized-array heap, the device-resident loop started over it,
// 64 batches of disjoint vertices submitted from the host (no CUDA call per
// batch), completions polled, the loop stopped.  Every batch must finish
// without failed allocations; every vertex it grew must have doubled its
// degree (up to the 2048-edge cap) and hold the edges its recipe gives.
// Prints one JSON line; exit code 0 when all of that holds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <random>
#include <vector>

#include "ouroboros_b200.h"

#define CHECK(x)                                                            \
  do {                                                                      \
    int rc_ = (x);                                                          \
    if (rc_) {                                                              \
      printf("{\"ok\": false, \"call\": \"%s\", \"rc\": %d}\n", #x, rc_);   \
      return 1;                                                             \
    }                                                                       \
  } while (0)

int main() {
  const uint32_t nv = 1u << 16, batches = 64;
  ouro_heap* h = nullptr;
  CHECK(ouro_create(OURO_VAP, 2ull << 30, &h));
  void** vptr = nullptr;
  uint32_t *degree = nullptr, *scratch = nullptr, *verts = nullptr;
  unsigned long long* cnt = nullptr;
  CHECK(cudaMalloc(&vptr, nv * sizeof(void*)));
  CHECK(cudaMalloc(&degree, nv * sizeof(uint32_t)));
  CHECK(cudaMalloc(&scratch, nv * sizeof(uint32_t)));
  CHECK(cudaMalloc(&verts, nv * sizeof(uint32_t)));
  CHECK(cudaMalloc(&cnt, 4 * sizeof(unsigned long long)));
  CHECK(cudaMemset(cnt, 0, 4 * sizeof(unsigned long long)));
  CHECK(ouro_graph_init(h, vptr, degree, scratch, nv, 7, 2.1f, cnt, nullptr));
  CHECK(cudaDeviceSynchronize());
  std::vector<uint32_t> d0(nv);
  CHECK(cudaMemcpy(d0.data(), degree, nv * sizeof(uint32_t), cudaMemcpyDeviceToHost));

  // disjoint vertex sets, uneven batch sizes
  std::vector<uint32_t> perm(nv);
  std::iota(perm.begin(), perm.end(), 0u);
  std::mt19937 rng(11);
  std::shuffle(perm.begin(), perm.end(), rng);
  CHECK(cudaMemcpy(verts, perm.data(), nv * sizeof(uint32_t), cudaMemcpyHostToDevice));
  std::vector<uint32_t> off(batches + 1, 0);
  for (uint32_t b = 0; b < batches; ++b) off[b + 1] = off[b] + 200u + (b * 37u) % 800u;

  ouro_serve_config cfg{1024u, 16u, 0, 0.05, 10.0};
  ouro_server* s = nullptr;
  CHECK(ouro_serve_start(h, vptr, degree, nv, 7, &cfg, &s));
  for (uint32_t b = 0; b < batches; ++b) {
    uint64_t seq = 0;
    CHECK(ouro_serve_submit(s, verts + off[b], off[b + 1] - off[b], b % 8u, &seq));
  }
  std::vector<ouro_serve_result> res(batches);
  uint32_t have = 0;
  for (uint64_t it = 0; have < batches && it < 20000000ull; ++it) {
    uint32_t got = 0;
    CHECK(ouro_serve_poll(s, res.data() + have, batches - have, &got));
    have += got;
  }
  ouro_serve_stats st{};
  CHECK(ouro_serve_stop(s, &st));
  CHECK(ouro_serve_close(s));

  uint64_t failed = 0, giveups = 0;
  double lat_max = 0.0;
  for (uint32_t i = 0; i < have; ++i) {
    failed += res[i].failed_allocs;
    giveups += res[i].lock_giveups;
    lat_max = std::max(lat_max, (res[i].t_done_ns - res[i].t_seen_ns) * 1e-6);
  }
  std::vector<uint32_t> d1(nv);
  CHECK(cudaMemcpy(d1.data(), degree, nv * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  uint64_t wrong_degree = 0;
  for (uint32_t i = 0; i < off[batches]; ++i) {
    const uint32_t v = perm[i];
    wrong_degree += d1[v] != std::min(2u * d0[v], 2048u);
  }
  CHECK(ouro_graph_check(vptr, degree, verts, off[batches], nv, 7, cnt + 2, nullptr));
  unsigned long long chk[4] = {0, 0, 0, 0};
  CHECK(cudaMemcpy(chk, cnt, sizeof(chk), cudaMemcpyDeviceToHost));
  const bool ok = have == batches && failed == 0 && giveups == 0 && wrong_degree == 0 && chk[3] == 0 &&
                  st.batches_seen == batches && st.status == 0;
  printf("{\"ok\": %s, \"batches\": %u, \"failed_allocs\": %llu, \"lock_giveups\": %llu, \"wrong_degree\": %llu, "
         "\"bad_vertices\": %llu, \"max_latency_ms\": %.3f, \"status\": %u}\n",
         ok ? "true" : "false", have, (unsigned long long)failed, (unsigned long long)giveups,
         (unsigned long long)wrong_degree, chk[3], lat_max, st.status);
  cudaFree(vptr);
  cudaFree(degree);
  cudaFree(scratch);
  cudaFree(verts);
  cudaFree(cnt);
  ouro_destroy(h);
  return ok ? 0 : 1;
}
