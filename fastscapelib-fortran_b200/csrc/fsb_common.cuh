// Shared definitions of the B200 continental-step library.
//
// Node numbering is 0-based: ij = i + j*nx with i in [0,nx), j in [0,ny)
// (x fastest), i.e. the reference's ij = i + (j-1)*nx minus one.  Slot arrays
// (donors, multiple receivers) are node-major with 8 slots per node, which is
// the reference's column-major don(8,nn) / mrec(8,nn) layout.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

namespace fsb {

// Boundary description decoded from the reference's 4-digit code
// (src/FastScape_ctx.f90:565-593): digits are bottom, right, top, left.
struct Bounds {
  int nx, ny;
  int i1, i2, j1, j2;   // 0-based inclusive loop bounds of find_receiver
  int fix_bottom, fix_right, fix_top, fix_left;
  int xcyc, ycyc;
};

__host__ __device__ inline bool is_bc_node(const Bounds& b, int i, int j) {
  return (b.fix_left && i == 0) || (b.fix_right && i == b.nx - 1) || (b.fix_bottom && j == 0) ||
         (b.fix_top && j == b.ny - 1);
}

// Neighbour index with the reference's wrap-then-clamp rule
// (FlowRouting.f90:336-344).
__host__ __device__ inline int wrap_clamp(int v, int n, int cyc) {
  if (v < 0 && cyc) v += n;
  v = v < 0 ? 0 : v;
  if (v > n - 1 && cyc) v -= n;
  v = v > n - 1 ? n - 1 : v;
  return v;
}

// Error codes written by device code to the context's status word.
enum DeviceError : int {
  DEV_OK = 0,
  DEV_SPIN_LIMIT = 1,       // a bounded wait gave up
  DEV_STACK_ERROR = 2,      // a traversal did not cover every node
  DEV_TRIDAG_ZERO = 3,      // zero pivot in the tridiagonal solve
  DEV_OVERFLOW = 4,         // a data-dependent buffer bound was exceeded
  DEV_NOT_ADJACENT = 5,     // a receiver is not one of the node's 3x3 neighbours
  DEV_NEWTON_LIMIT = 6,     // a Newton solve of the stream power law did not converge
};

// Newton iterations a node may take before the stream power law reports
// DEV_NEWTON_LIMIT (the reference iterates until |h_new - h| <= 1e-3,
// StreamPowerLaw.f90:146-162 and :343-358; about 1.5 iterations are typical)
constexpr int kNewtonLimit = 10000;

constexpr int kSpinLimit = 1 << 21;  // polls (~1 s) before a bounded wait gives up

#ifdef __CUDACC__
// Acquire/release fence at GPU scope.  Hand-offs between threads use the
// pattern "write; fence; relaxed atomic or flag store" on the producer side
// and "relaxed atomic or flag load; fence; read" on the consumer side, which
// needs acquire-release ordering only -- not the sequentially consistent
// fence that __threadfence() issues.
__device__ __forceinline__ void fence_acq_rel() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

// loads with acquire semantics at GPU scope: later memory operations of the
// thread see everything released before the value read was written (cheaper
// than a load followed by fence_acq_rel)
__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// relaxed (strong, GPU scope) double load/store: never served from a stale L1 line
__device__ __forceinline__ double ld_relaxed_gpu(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_gpu(double* p, double v) {
  asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
#endif

}  // namespace fsb
