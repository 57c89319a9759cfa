// Host check of the host-buffer calls' slice plan (ouroboros_b200/csrc/host_plan.h):
// for every batch size n below 20,000 and a set of large ones up to 2^32 - 1,
// and every wanted slice count 0..8, the plan must give 1..8 slices that each
// start below n, hold at least one request, and together hold exactly n.
// Prints "cases C bad B"; exit status 1 when B > 0.
#include <cstdint>
#include <cstdio>

#include "../../ouroboros_b200/csrc/host_plan.h"

int main() {
  using namespace ouro_host;
  long cases = 0, bad = 0;
  auto check = [&](uint32_t n, int wanted) {
    uint32_t k = 0, m = 0;
    host_slice_plan(n, wanted, &k, &m);
    ++cases;
    if (k < 1u || k > kHostSlicesMax || m == 0u) { ++bad; return; }
    uint64_t total = 0;
    for (uint32_t j = 0; j < k; ++j) {
      const uint64_t o = static_cast<uint64_t>(j) * m;
      if (o >= n) { ++bad; return; }
      const uint64_t c = n - o < m ? n - o : m;
      if (c == 0u) { ++bad; return; }
      total += c;
    }
    if (total != n) ++bad;
  };
  for (uint32_t n = 1; n < 20000u; ++n)
    for (int wanted = 0; wanted <= 8; ++wanted) check(n, wanted);
  const uint32_t large[] = {1u << 17, (1u << 18) + 5u, 1u << 20, 3000001u, 1u << 30, 0xFFFFFFF0u, 0xFFFFFFFFu};
  for (uint32_t n : large)
    for (int wanted = 0; wanted <= 8; ++wanted) check(n, wanted);
  // the defaults: 1 slice below 2^18 requests, 4 from 2^19 on
  uint32_t k = 0, m = 0;
  host_slice_plan(1u << 17, 0, &k, &m);
  bad += k != 1u;
  host_slice_plan(1u << 20, 0, &k, &m);
  bad += !(k == 4u && m == (1u << 18));
  std::printf("cases %ld bad %ld\n", cases, bad);
  return bad ? 1 : 0;
}
