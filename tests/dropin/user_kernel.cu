// A user program written against the drop-in header: its own kernel calls
// mm->malloc / mm->free directly, mixing sizes, writing and checking every
// allocation inside the same kernel, for several rounds.  Prints one JSON line.
#include <cstdio>
#include <cstdint>

#include "ouroboros_b200.cuh"

template <typename MM>
__global__ void churn(MM* mm, int rounds, unsigned long long* bad, unsigned long long* nulls) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  for (int r = 0; r < rounds; ++r) {
    uint32_t x = (tid * 2654435761u) ^ (r * 40503u);
    x ^= x >> 13;
    const uint32_t size = 16u + (x % 4000u);
    uint32_t* p = static_cast<uint32_t*>(mm->malloc(size));
    if (!p) { atomicAdd(nulls, 1ull); continue; }
    for (uint32_t w = 0; w < size / 4u; ++w) p[w] = tid + w;
    __syncwarp();
    uint32_t b = 0;
    for (uint32_t w = 0; w < size / 4u; ++w) b += p[w] != tid + w;
    if (b) atomicAdd(bad, static_cast<unsigned long long>(b));
    mm->free(p);
  }
}

template <typename Host>
int run(const char* name, int blocks, int rounds) {
  Host mm;
  mm.initialize(1ull << 30);
  unsigned long long* c = nullptr;
  cudaMalloc(&c, 2 * sizeof(unsigned long long));
  cudaMemset(c, 0, 2 * sizeof(unsigned long long));
  churn<<<blocks, 256>>>(mm.getDeviceMemoryManager(), rounds, c, c + 1);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long h[2] = {0, 0};
  cudaMemcpy(h, c, sizeof(h), cudaMemcpyDeviceToHost);
  ouro_heap_status st;
  ouro_get_status(mm.handle(), &st, 0);
  printf("{\"variant\": \"%s\", \"cuda\": %d, \"bad\": %llu, \"nulls\": %llu, \"flags\": %u}\n", name, (int)e, h[0], h[1],
         st.flags);
  cudaFree(c);
  return e == cudaSuccess && h[0] == 0 && h[1] == 0 && st.flags == 0 ? 0 : 1;
}

int main(int argc, char** argv) {
  int blocks = argc > 1 ? atoi(argv[1]) : 592;
  int rounds = argc > 2 ? atoi(argv[2]) : 8;
  int rc = 0;
  rc |= run<ouro::MultiOuroPQ>("P", blocks, rounds);
  rc |= run<ouro::MultiOuroCQ>("C", blocks, rounds);
  rc |= run<ouro::MultiOuroVAPQ>("VAP", blocks, rounds);
  rc |= run<ouro::MultiOuroVACQ>("VAC", blocks, rounds);
  rc |= run<ouro::MultiOuroVLPQ>("VLP", blocks, rounds);
  rc |= run<ouro::MultiOuroVLCQ>("VLC", blocks, rounds);
  return rc;
}
