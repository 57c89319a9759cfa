// host_plan.h -- how the host-buffer calls (ouro_alloc_host / ouro_free_host)
// cut a batch into slices.  Plain C++ with no CUDA types, so the plan is
// checked on the host by tests/host_plan/check_plan.cpp.
#pragma once

#include <cstdint>

namespace ouro_host {

constexpr uint32_t kHostSlicesMax = 8u;
constexpr uint32_t kHostSliceMin = 1u << 17;   // fewer requests per launch fill the GPU poorly

inline uint32_t host_slices(uint32_t n, int slices) {
  if (slices > 0) return n < static_cast<uint32_t>(slices) ? n : static_cast<uint32_t>(slices);
  const uint32_t k = n / kHostSliceMin;
  return k < 1u ? 1u : k > 4u ? 4u : k;
}

// k slices of m requests (the last one shorter): m = ceil(n / wanted), and
// k = ceil(n / m), so that every slice starts below n and holds at least one
// request (n = 10 in 8 wanted slices: 5 slices of 2).
inline void host_slice_plan(uint32_t n, int slices, uint32_t* k, uint32_t* m) {
  const uint64_t want = host_slices(n, slices);
  const uint64_t per = (n + want - 1u) / want;
  *m = static_cast<uint32_t>(per);
  *k = static_cast<uint32_t>((n + per - 1u) / per);
}

}  // namespace ouro_host
