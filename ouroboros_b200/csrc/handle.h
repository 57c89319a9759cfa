// handle.h -- the host-side heap handle and launch helpers shared by the
// library's translation units (capi.cu, batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "../../include/ouroboros_b200.h"
#include "host_plan.h"
#include "ouro/ouroboros.cuh"

struct ouro_heap {
  int variant;
  int device;
  unsigned long long heap_bytes;
  ouro::Layout L;
  ouro_config cfg;
  void* raw;
  ouro::HeapCore* dev;
  char* base;
  int batch_block;    // batched path: block size of the serving launch picked by ouro_autotune_batch (0: default)
  int batch_per_sm;   // kept for the C ABI's report; the serving launch is not persistent
  void* batch_scratch;              // batched path: sort counters and permutation (grown on demand)
  size_t batch_scratch_bytes;
  // host-buffer entry points (ouro_alloc_host / ouro_free_host): device
  // staging for request sizes and pointers, two copy streams and their
  // events, made on first use; calls on one heap take turns on the mutex
  void* host_stage;
  size_t host_stage_bytes;
  cudaStream_t host_in, host_out;
  cudaEvent_t host_entry, host_done, host_joined;
  cudaEvent_t host_slice_in[ouro_host::kHostSlicesMax], host_slice_run[ouro_host::kHostSlicesMax];
  bool host_ready;
  std::mutex host_mu;
};

namespace ouro {

inline int cuda_rc(cudaError_t e) { return e == cudaSuccess ? OURO_OK : OURO_ERR_CUDA; }

inline unsigned grid_for(uint32_t n, int block) { return (n + static_cast<unsigned>(block) - 1u) / block; }

// Run f with the instantiation index as a compile-time constant.
template <typename F>
int dispatch(int variant, F&& f) {
  switch (variant) {
    case 0: return f(std::integral_constant<int, 0>{});
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    default: return OURO_ERR_ARG;
  }
}

}  // namespace ouro
