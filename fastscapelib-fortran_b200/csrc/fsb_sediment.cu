// The stream power law with the sediment term (g > 0): Gauss-Seidel
// iterations of erosion sum, deposition-corrected surface and implicit solve,
// then the lake-sediment fill.
//
// Reference (fastscapelib-fortran file:line):
//   StreamPowerLaw (multiple flow)      src/StreamPowerLaw.f90:3-206
//   StreamPowerLawSingleFlowDirection   src/StreamPowerLaw.f90:210-400
// One iteration:
//   hp = h;  dh = erosion ht-hp summed downstream (bottom-up sweep), with each
//   lake sill's upstream share kept as lake_sediment;
//   elev = ht + (dh - (ht-hp)) * g * dx * dy / a  (ht on fixed boundaries);
//   the implicit solve from the current iterate with elev as the surface
//   (top-down sweep), which also records each node's lake sill and, for a
//   flooded node, its share w_rcv - h of the sill's water volume;
//   err = sqrt(sum((h-hp)^2)/nn) against tol = 1e-4*(max|ht|+1), at most 99
//   iterations; err = 0 when max(g) < tiny.
// Then b = min(h, b), each node of a lake with water volume V and sediment S
// rises by max(0, min(S, V))/V * (water - h), and etot, erate, Sedflux follow.
// The first iteration is the g = 0 solve (dh = 0, elev = ht); the reference's
// single-flow variant reads lake_sill before writing it in that iteration, with
// no effect since dh = 0 there; here lake_sill starts as "none".
// Sums of floating-point values run in another order than the reference's
// stack loops (lake volumes, the multiple-flow erosion sum, err), so results
// agree to rounding, not bit for bit.
#include <cfloat>
#include <cmath>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

constexpr int kRedBlocks = 512, kRedThreads = 256;

// g = g1, or g2 where h - b > 1 (StreamPowerLaw.f90:227-230)
__global__ void k_gfield(int nn, double g1, double g2, const double* __restrict__ h, const double* __restrict__ b,
                         double* __restrict__ g) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    double v = g1;
    if (g2 > 0.0 && (h[k] - b[k]) > 1.0) v = g2;
    g[k] = v;
  }
}

// part[b*2+0] = max |h|, part[b*2+1] = max g over block b's nodes
__global__ void __launch_bounds__(kRedThreads) k_max_partials(int nn, const double* __restrict__ h,
                                                              const double* __restrict__ g, double* __restrict__ part) {
  __shared__ double sh[2][kRedThreads];
  double mh = 0.0, mg = -DBL_MAX;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    mh = fmax(mh, fabs(h[k]));
    mg = fmax(mg, g[k]);
  }
  sh[0][threadIdx.x] = mh;
  sh[1][threadIdx.x] = mg;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + w]);
      sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x < 2) part[blockIdx.x * 2 + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(kRedThreads) k_max_final(const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[2][kRedThreads];
  double mh = 0.0, mg = -DBL_MAX;
  for (int b = threadIdx.x; b < kRedBlocks; b += kRedThreads) {
    mh = fmax(mh, part[b * 2]);
    mg = fmax(mg, part[b * 2 + 1]);
  }
  sh[0][threadIdx.x] = mh;
  sh[1][threadIdx.x] = mg;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + w]);
      sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x < 2) out[threadIdx.x] = sh[threadIdx.x][0];
}

// sum of (x - y)^2 in a fixed order (per-thread strides, block trees, one final block)
__global__ void __launch_bounds__(kRedThreads) k_sq_partials(int nn, const double* __restrict__ x,
                                                             const double* __restrict__ y, double* __restrict__ part) {
  __shared__ double sh[kRedThreads];
  double s = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double d = x[k] - y[k];
    s += d * d;
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void __launch_bounds__(kRedThreads) k_sum_final(const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[kRedThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < kRedBlocks; b += kRedThreads) s += part[b];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// e = ht - hp: the base of the multiple-flow erosion sum
__global__ void k_erosion(int nn, const double* __restrict__ ht, const double* __restrict__ hp, double* __restrict__ e) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) e[k] = ht[k] - hp[k];
}

// elev = ht on fixed boundaries, else ht + (dh - (ht-hp))*g*dx*dy/a, left to right
__global__ void k_elev(Bounds bd, double dx, double dy, const double* __restrict__ ht, const double* __restrict__ hp,
                       const double* __restrict__ dh, const double* __restrict__ g, const double* __restrict__ a,
                       double* __restrict__ elev) {
  const int nn = bd.nx * bd.ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    if (is_bc_node(bd, k % bd.nx, k / bd.nx)) elev[k] = ht[k];
    else elev[k] = ht[k] + (dh[k] - (ht[k] - hp[k])) * g[k] * dx * dy / a[k];
  }
}

__global__ void k_unpack_hw(int nn, const double2* __restrict__ hw, double* __restrict__ h, double* __restrict__ water) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double2 v = hw[k];
    h[k] = v.x;
    water[k] = v.y;
  }
}

// b = min(h, b); lake fill; etot, erate, Sedflux (StreamPowerLaw.f90:380-393)
__global__ void k_gs_finish(int nn, double dt, const double* __restrict__ hcur, const double* __restrict__ water,
                            const int* __restrict__ sill, const double* __restrict__ lsed,
                            const double* __restrict__ vol, double* __restrict__ h, double* __restrict__ b,
                            double* __restrict__ etot, double* __restrict__ erate, double* __restrict__ sedflux) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double ht = h[k];
    double hk = hcur[k];
    b[k] = fmin(hk, b[k]);
    const int s = sill[k];
    if (s >= 0) {
      const double v = vol[s];
      if (v > 0.0) hk = hk + fmax(0.0, fmin(lsed[s], v)) / v * (water[k] - hk);
    }
    etot[k] = etot[k] + ht - hk;
    erate[k] = (ht - hk) / dt;
    sedflux[k] = ht - hk;
    h[k] = hk;
  }
}

}  // namespace

bool gs_active(const Ctx& c) { return c.g1 > 0.0 || c.g2 > 0.0 || (c.g1 < 0.0 && c.g_positive); }

int stream_power_gs(Ctx& c) {
  const int nn = c.nn;
  cudaStream_t st = c.stream;
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  if (c.g1 >= 0.0) {
    k_gfield<<<grid1d(nn), kBlock, 0, st>>>(nn, c.g1, c.g2, c.h, c.b, c.g);
    c.count_launch();
  }
  double* part = c.red;
  double* out = c.red + 3 * 512;
  k_max_partials<<<kRedBlocks, kRedThreads, 0, st>>>(nn, c.h, c.g, part);
  k_max_final<<<1, kRedThreads, 0, st>>>(part, out);
  c.count_launch(2);
  double mx[2];
  if (cudaMemcpyAsync(mx, out, sizeof mx, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return report_error("stream power (g > 0): reading the maxima failed");
  const double tol = 1.0e-4 * (mx[0] + 1.0);
  const bool g_zero = mx[1] < DBL_MIN;
  c.g_positive = !g_zero;

  // scratch of the iterations (the diffusion buffers are free until the diffusion stage)
  double* hcur = c.hnew;  // current iterate
  double* hp = c.dA;
  double* dh = c.dB;
  double* lsed = c.dC;
  double* elev = c.dF;
  double* contrib = c.dG;
  double* e = c.dK;
  int* sill = c.s_flag;
  cudaMemcpyAsync(hcur, c.h, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(lsed, 0, sizeof(double) * nn, st);
  cudaMemsetAsync(sill, 0xff, sizeof(int) * nn, st);  // -1: no sill yet

  double err = 2.0 * tol;
  c.ngs = 0;
  while (err > tol && c.ngs < 99) {
    c.ngs += 1;
    cudaMemcpyAsync(hp, hcur, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
    if (c.sfd) {
      gs_erosion_chains(c, hp, sill, lsed, dh);
    } else {
      k_erosion<<<grid1d(nn), kBlock, 0, st>>>(nn, c.h, hp, e);
      c.count_launch();
      gs_erosion_mfd(c, e, sill, lsed, dh);
    }
    k_elev<<<grid1d(nn), kBlock, 0, st>>>(c.bd, dx, dy, c.h, hp, dh, c.g, c.a, elev);
    c.count_launch();
    if (c.sfd) {
      spl_chains_gs(c, elev, hp, hcur, sill, contrib);
    } else {
      spl_mfd_gs(c, elev, hp, sill, contrib);
      k_unpack_hw<<<grid1d(nn), kBlock, 0, st>>>(nn, reinterpret_cast<const double2*>(c.hw), hcur, c.water);
      c.count_launch();
    }
    k_sq_partials<<<kRedBlocks, kRedThreads, 0, st>>>(nn, hcur, hp, part);
    k_sum_final<<<1, kRedThreads, 0, st>>>(part, out);
    c.count_launch(2);
    double s2 = 0.0;
    int derr = 0;
    if (cudaMemcpyAsync(&s2, out, sizeof s2, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&derr, c.d_err, sizeof derr, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return report_error("stream power (g > 0): reading the iteration error failed");
    if (derr) break;  // a sweep gave up; the step's device-error check reports it
    err = std::sqrt(s2 / nn);
    if (g_zero) err = 0.0;
  }
  double* vol = c.dZ;
  double* up = reinterpret_cast<double*>(c.ch_val);
  ensure_chains(c);
  lake_volume_chains(c, sill, contrib, vol, up);
  k_gs_finish<<<grid1d(nn), kBlock, 0, st>>>(nn, c.dt, hcur, c.water, sill, lsed, vol, c.h, c.b, c.etot, c.erate,
                                            c.sedflux);
  c.count_launch();
  return 0;
}

}  // namespace fsb
