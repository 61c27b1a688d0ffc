// Latency probe: one thread follows a random cyclic permutation of 128-byte
// lines (all L2-resident after the warm-up), each access depending on the
// previous one, with plain L2 loads (ld.global.cg), strong relaxed GPU-scope
// loads and atomics.  Prints cycles and ns per access.  Build and run:
//   nvcc -O3 -gencode arch=compute_100a,code=sm_100a -o l2_latency l2_latency.cu && ./l2_latency
// Every index is an entry of the permutation, so every access is in bounds.
#include <cstdio>
#include <vector>
#include <random>
#include <algorithm>
#include <cuda_runtime.h>
__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p) { unsigned v; asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory"); return v; }
__device__ __forceinline__ unsigned ld_cg(const unsigned* p) { unsigned v; asm volatile("ld.global.cg.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory"); return v; }
template <int MODE>
__global__ void chase(unsigned* next, unsigned n, int steps, unsigned long long* out, unsigned* sink) {
  unsigned i = 0;
  for (int s = 0; s < 2000; ++s) i = MODE == 0 ? ld_cg(&next[i * 32]) : MODE == 1 ? ld_relaxed(&next[i * 32]) : atomicAdd(&next[i * 32], 0u);  // warm
  long long t0 = clock64();
  for (int s = 0; s < steps; ++s) i = MODE == 0 ? ld_cg(&next[i * 32]) : MODE == 1 ? ld_relaxed(&next[i * 32]) : atomicAdd(&next[i * 32], 0u);
  long long t1 = clock64();
  out[0] = (unsigned long long)(t1 - t0);
  sink[0] = i;
}
int main() {
  const char* names[3] = {"ld.cg (L2)", "ld.relaxed.gpu", "atomicAdd"};
  for (unsigned n : {64u, 4096u, 131072u}) {  // lines visited: 8 KB .. 16 MB of 128-byte lines
    std::vector<unsigned> perm(n);
    for (unsigned i = 0; i < n; ++i) perm[i] = i;
    std::mt19937 g(1);
    std::shuffle(perm.begin() + 1, perm.end(), g);
    std::vector<unsigned> next((size_t)n * 32, 0);
    for (unsigned i = 0; i < n; ++i) next[(size_t)perm[i] * 32] = perm[(i + 1) % n];  // one cycle through all lines
    unsigned *d, *sink; unsigned long long* o;
    cudaMalloc(&d, next.size() * 4); cudaMalloc(&o, 8); cudaMalloc(&sink, 4);
    cudaMemcpy(d, next.data(), next.size() * 4, cudaMemcpyHostToDevice);
    const int steps = 20000;
    for (int m = 0; m < 3; ++m) {
      unsigned long long cyc = 0;
      if (m == 0) chase<0><<<1, 1>>>(d, n, steps, o, sink);
      if (m == 1) chase<1><<<1, 1>>>(d, n, steps, o, sink);
      if (m == 2) chase<2><<<1, 1>>>(d, n, steps, o, sink);
      cudaError_t e = cudaDeviceSynchronize();
      cudaMemcpy(&cyc, o, 8, cudaMemcpyDeviceToHost);
      int clk = 0; cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, 0);
      printf("%-16s lines %7u (%6.1f MB)  %7.0f cycles  %6.0f ns/access (at %d MHz) %s\n", names[m], n, n * 128.0 / 1e6,
             (double)cyc / steps, (double)cyc / steps / (clk / 1e6), clk / 1000, cudaGetErrorString(e));
    }
    cudaFree(d); cudaFree(o); cudaFree(sink);
  }
  return 0;
}
