// One ADI hillslope-diffusion step for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a host callback
// or a real-time loop, code embedded in a framework that owns every device
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
#include <mutex>
#include <string>

#include "fsb_kernels.cuh"
#include "../../include/fastscape_b200.h"

namespace {

constexpr int kNoAllocMaxNodes = 1 << 16;  // nx*ny limit (e.g. 256 x 256)
constexpr int kScratchDoubles = 7 * kNoAllocMaxNodes + 32;  // 7 arrays + the error word

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_dev[kMaxDevices] = {};  // device address of g_noalloc_scratch per device

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
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail("fsb_diffusion_step_noalloc: no usable current CUDA device");
  double* scratch = nullptr;
  {
    // once per device, with that device current: the host-side name of the
    // array is not a device address, so ask the runtime for the real one
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return noalloc_fail(std::string("fsb_diffusion_step_noalloc: cudaGetSymbolAddress failed: ") +
                            cudaGetErrorString(e));
      g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
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
  int herr = 0;
  cudaError_t e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(std::string("fsb_diffusion_step_noalloc: ") + cudaGetErrorString(e));
  if (herr != 0) return noalloc_fail("fsb_diffusion_step_noalloc: tridag failed (zero pivot)");
  return 0;
}

}  // extern "C"
