// One ADI hillslope-diffusion step for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: a real-time loop that must not stall
// on the allocator, code embedded in a framework that owns every device
// allocation through its own pool, or a host program that must not change
// the device's memory footprint after start-up.  fsb_diffusion_step_noalloc
// gives them the library's ADI diffusion step (the same kernels as the step
// driver) on arrays they already own.  Its scratch space -- kdint, the
// tridiagonal coefficients, the elimination factors and the x-pass result --
// lives in the file-scope device array below, sized for grids of at most
// kNoAllocMaxNodes nodes.  Every GPU that loads this library holds that
// array (about 3.7 MB) until the process exits.  All calls share it and it
// keeps the last call's contents, so calls that overlap on the GPU (two
// streams, two host threads) race; the error word is cleared on every call.
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <string>

#include "fsb_kernels.cuh"
#include "../../include/fastscape_b200.h"

namespace {

constexpr int kNoAllocMaxNodes = 1 << 16;  // nx*ny limit (e.g. 256 x 256)
constexpr int kScratchDoubles = 7 * kNoAllocMaxNodes + 32;  // 7 arrays + the error word

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

int noalloc_fail(const std::string& m) { return fsb::report_error(m); }

}  // namespace

extern "C" {

int fsb_diffusion_step_noalloc(int nx, int ny, double xl, double yl, double dt, int bc, double kdsed,
                               const double* kd, double* h, double* b, double* etot, double* erate,
                               void* stream) {
  if (nx < 3 || ny < 3) return noalloc_fail("fsb_diffusion_step_noalloc: nx and ny must be >= 3");
  if ((long long)nx * ny > kNoAllocMaxNodes)
    return noalloc_fail("fsb_diffusion_step_noalloc: nx*ny = " + std::to_string((long long)nx * ny) +
                        " exceeds the static scratch limit of " + std::to_string(kNoAllocMaxNodes) + " nodes");
  if (!kd || !h || !b || !etot || !erate) return noalloc_fail("fsb_diffusion_step_noalloc: null array");
  // An error left pending by earlier work of the caller's thread stays the
  // caller's: this call neither reports it as its own nor clears it.
  const cudaError_t pending = cudaPeekAtLastError();
  if (pending != cudaSuccess)
    return noalloc_fail(std::string("fsb_diffusion_step_noalloc: an earlier CUDA error is pending: ") +
                        cudaGetErrorString(pending));
  // The host-side name of the array is not a device address.  The address is
  // looked up on every call, with the caller's device and context current: the
  // query allocates nothing and stays right after cudaDeviceReset or under
  // another context on the same device.
  void* sym = nullptr;
  const cudaError_t se = cudaGetSymbolAddress(&sym, g_noalloc_scratch);
  if (se != cudaSuccess)
    return noalloc_fail(std::string("fsb_diffusion_step_noalloc: cudaGetSymbolAddress failed: ") +
                        cudaGetErrorString(se));
  double* scratch = static_cast<double*>(sym);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* err = reinterpret_cast<int*>(scratch + 7 * (size_t)kNoAllocMaxNodes);
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess)
    return noalloc_fail("fsb_diffusion_step_noalloc: could not clear the error word");
  // SetBC digits (FastScape_ctx.f90:565-593)
  char cbc[16];
  if (bc > 9999 || bc < -999) std::strcpy(cbc, "****");
  else std::snprintf(cbc, sizeof cbc, "%4d", bc);
  fsb::Bounds bd{};
  bd.nx = nx;
  bd.ny = ny;
  bd.fix_bottom = cbc[0] == '1';
  bd.fix_right = cbc[1] == '1';
  bd.fix_top = cbc[2] == '1';
  bd.fix_left = cbc[3] == '1';
  bd.i1 = bd.fix_left ? 1 : 0;
  bd.i2 = bd.fix_right ? nx - 2 : nx - 1;
  bd.j1 = bd.fix_bottom ? 1 : 0;
  bd.j2 = bd.fix_top ? ny - 2 : ny - 1;
  bd.xcyc = !bd.fix_left && !bd.fix_right;
  bd.ycyc = !bd.fix_bottom && !bd.fix_top;
  fsb::diffusion_raw(bd, xl / (nx - 1), yl / (ny - 1), dt, kdsed, kd, h, b, etot, erate, scratch, err, st);
  // launch errors of this call only (nothing was pending at entry)
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return noalloc_fail(std::string("fsb_diffusion_step_noalloc: launch failed: ") + cudaGetErrorString(e));
  int herr = 0;
  e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_fail(std::string("fsb_diffusion_step_noalloc: ") + cudaGetErrorString(e));
  if (herr != 0) return noalloc_fail("fsb_diffusion_step_noalloc: tridag failed (zero pivot)");
  return 0;
}

}  // extern "C"
