// Hop replay probe: one thread walks a 129x129 grid from neighbour to
// neighbour and at each step replays parts of a multiple-flow sweep hop's
// memory traffic (the node's 10-slot input row and 128-byte record line, one
// relaxed store into each of the 8 neighbours' slot rows, one atomic on each
// of the 8 neighbours' counters, the dependents' prefetches), each step
// depending on the previous one.  Prints cycles and ns per hop.  Build and run:
//   nvcc -O3 -gencode arch=compute_100a,code=sm_100a -o hop_replay hop_replay.cu && ./hop_replay
// Neighbour indices wrap inside the grid and counter offsets are reduced
// modulo the array size, so every access is in bounds.
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
__device__ __forceinline__ double ldr(const double* p) { double v; asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory"); return v; }
__device__ __forceinline__ double2 ldr2(const double* p) { double2 v; asm volatile("ld.relaxed.gpu.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p) : "memory"); return v; }
__device__ __forceinline__ void str(double* p, double v) { asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" :: "l"(p), "d"(v) : "memory"); }
// MODE bits: 1 loads (10 slots + 128-byte line), 2 stores to 8 neighbour rows, 4 atomics on 8 neighbour counters,
//            8 atomics on counters 64 KB apart instead of neighbours, 16 loads without the line, 32 one atomic only
template <int MODE>
__global__ void hop(double* slots, const int4* line, int* cnt, int nx, int ny, int steps, unsigned long long* out, double* sink) {
  int k = nx * (ny / 2) + nx / 2;
  double acc = 0.0;
  unsigned h = 12345u;
  long long t0 = 0;
  for (int s = -200; s < steps; ++s) {
    if (s == 0) t0 = clock64();
    const int i = k % nx, j = k / nx;
    int nb[8];
    int c = 0;
    for (int dj = -1; dj <= 1; ++dj)
      for (int di = -1; di <= 1; ++di)
        if (di || dj) nb[c++] = ((i + di + nx) % nx) + ((j + dj + ny) % ny) * nx;
    double v = 0.0;
    if (MODE & 1) {
      const double* in = slots + (size_t)k * 16;
      double a[10];
      if (MODE & 128) {
#pragma unroll
        for (int t = 0; t < 5; ++t) { const double2 w = ldr2(&in[2 * t]); a[2 * t] = w.x; a[2 * t + 1] = w.y; }
      } else {
#pragma unroll
        for (int t = 0; t < 10; ++t) a[t] = ldr(&in[t]);
      }
      if (!(MODE & 16)) {
        int4 L[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) L[t] = __ldg(line + (size_t)k * 8 + t);
#pragma unroll
        for (int t = 0; t < 8; ++t) v += (double)(L[t].x & 1);
      }
#pragma unroll
      for (int t = 0; t < 10; ++t) v += a[t];
    }
    v += acc;
    if (MODE & 64) {
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(line + (size_t)nb[t] * 8));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(slots + (size_t)nb[t] * 16));
      }
    }
    if (MODE & 2) {
#pragma unroll
      for (int t = 0; t < 8; ++t) str(&slots[(size_t)nb[t] * 16 + (t & 7)], v);
    }
    int o = 0;
    if (MODE & 4) {
      int old[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) old[t] = atomicAdd(&cnt[(MODE & 8) ? (nb[t] * 16 + t * 16384) % (nx * ny * 16) : nb[t]], 0);
#pragma unroll
      for (int t = 0; t < 8; ++t) o += old[t];
    }
    if (MODE & 32) o += atomicAdd(&cnt[nb[0]], 0);
    acc = v * 0.5;
    h = h * 1664525u + 1013904223u + (unsigned)o + (unsigned)(v != v);
    k = nb[(h >> 13) & 7];
  }
  out[0] = (unsigned long long)(clock64() - t0);
  sink[0] = acc;
}
template <int M>
void run(const char* name, double* slots, int4* line, int* cnt, int nx, int ny, unsigned long long* o, double* sink) {
  const int steps = 20000;
  hop<M><<<1, 1>>>(slots, line, cnt, nx, ny, steps, o, sink);
  cudaError_t e = cudaDeviceSynchronize();
  unsigned long long cyc = 0;
  cudaMemcpy(&cyc, o, 8, cudaMemcpyDeviceToHost);
  printf("%-44s %6.0f cycles  %5.0f ns/hop  %s\n", name, (double)cyc / steps, (double)cyc / steps / 1.965, cudaGetErrorString(e));
}
int main() {
  const int nx = 129, ny = 129, nn = nx * ny;
  double* slots; int4* line; int* cnt; unsigned long long* o; double* sink;
  cudaMalloc(&slots, (size_t)nn * 16 * 8); cudaMalloc(&line, (size_t)nn * 128); cudaMalloc(&cnt, (size_t)nn * 16 * 4);
  cudaMalloc(&o, 8); cudaMalloc(&sink, 8);
  cudaMemset(slots, 0, (size_t)nn * 16 * 8); cudaMemset(line, 0, (size_t)nn * 128); cudaMemset(cnt, 0, (size_t)nn * 16 * 4);
  run<0>("index arithmetic only", slots, line, cnt, nx, ny, o, sink);
  run<1>("loads: 10 slots + line", slots, line, cnt, nx, ny, o, sink);
  run<1 | 16>("loads: 10 slots only", slots, line, cnt, nx, ny, o, sink);
  run<1 | 16 | 128>("loads: 10 slots as 5 v2", slots, line, cnt, nx, ny, o, sink);
  run<32>("one atomic", slots, line, cnt, nx, ny, o, sink);
  run<4>("8 atomics, neighbour counters", slots, line, cnt, nx, ny, o, sink);
  run<4 | 8>("8 atomics, counters on distinct lines", slots, line, cnt, nx, ny, o, sink);
  run<2 | 4>("8 stores + 8 atomics", slots, line, cnt, nx, ny, o, sink);
  run<1 | 4>("loads + 8 atomics", slots, line, cnt, nx, ny, o, sink);
  run<1 | 2 | 4>("hop: loads + 8 stores + 8 atomics", slots, line, cnt, nx, ny, o, sink);
  run<1 | 2 | 4 | 8>("hop, counters on distinct lines", slots, line, cnt, nx, ny, o, sink);
  run<1 | 2 | 4 | 128>("hop, v2 slot loads", slots, line, cnt, nx, ny, o, sink);
  run<1 | 2 | 4 | 64>("hop + 16 prefetches", slots, line, cnt, nx, ny, o, sink);
  run<1 | 2 | 4 | 64 | 128>("hop + 16 prefetches, v2 slot loads", slots, line, cnt, nx, ny, o, sink);
  run<2 | 4 | 64>("stores + atomics + prefetches", slots, line, cnt, nx, ny, o, sink);
  return 0;
}
