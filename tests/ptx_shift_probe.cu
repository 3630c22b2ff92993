// Test helper: the PTX shift instructions the reference's over-wide shifts
// compile to on an NVIDIA GPU (shr.u32 / shl.b32 for the range masks of
// candidates.hpp:91-99, shl.b64 for the Bitset of utils.hpp:71-73), run with
// run-time shift counts.  Prints one line per count:
//     n shr.u32(0xFFFFFFFF, n) shl.b32(0xFFFFFFFF, n) shl.b64(1, n)
// Built and run by tests/test_gpu_reference.py.
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>

__global__ void probe(const uint32_t* n, uint32_t count, uint32_t* r32, uint64_t* r64) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t k = n[i];
  uint32_t a = 0, b = 0;
  uint64_t c = 0;
  asm volatile("shr.u32 %0, %1, %2;" : "=r"(a) : "r"(0xFFFFFFFFu), "r"(k));
  asm volatile("shl.b32 %0, %1, %2;" : "=r"(b) : "r"(0xFFFFFFFFu), "r"(k));
  asm volatile("shl.b64 %0, %1, %2;" : "=l"(c) : "l"(1ull), "r"(k));
  r32[2 * i] = a;
  r32[2 * i + 1] = b;
  r64[i] = c;
}

int main() {
  const uint32_t counts[] = {0, 1, 5, 31, 32, 33, 40, 63, 64, 65, 100, 255};
  const uint32_t m = sizeof(counts) / sizeof(counts[0]);
  uint32_t *dn = nullptr, *d32 = nullptr;
  uint64_t* d64 = nullptr;
  if (cudaMalloc(&dn, sizeof(counts)) != cudaSuccess || cudaMalloc(&d32, 8 * m) != cudaSuccess ||
      cudaMalloc(&d64, 8 * m) != cudaSuccess) {
    std::fprintf(stderr, "cudaMalloc failed\n");
    return 1;
  }
  cudaMemcpy(dn, counts, sizeof(counts), cudaMemcpyHostToDevice);
  probe<<<1, 32>>>(dn, m, d32, d64);
  uint32_t h32[2 * m];
  uint64_t h64[m];
  if (cudaMemcpy(h32, d32, 8 * m, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(h64, d64, 8 * m, cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "probe failed: %s\n", cudaGetErrorString(cudaGetLastError()));
    return 1;
  }
  for (uint32_t i = 0; i < m; ++i)
    std::printf("%u %u %u %llu\n", counts[i], h32[2 * i], h32[2 * i + 1], static_cast<unsigned long long>(h64[i]));
  cudaFree(dn);
  cudaFree(d32);
  cudaFree(d64);
  return 0;
}
