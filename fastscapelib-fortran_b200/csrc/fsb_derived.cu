// Derived fields and diagnostics of the API: catchment labels, slope and
// curvature, the layer shift of SetAllLayers and the sums of compute_fluxes.
//
// Reference routines restated here (fastscapelib-fortran file:line):
//   find_stack's catch propagation  src/FlowRouting.f90:393-443 (catch(k) is
//                                   catch0 of k's root before LocalMinima)
//   slope, curvature                src/TerrainDerivatives.f90:3-74
//   SetAllLayers                    src/FastScape_ctx.f90:660-676
//   compute_fluxes (the sums)       src/FastScape_ctx.f90:843-886
// The chi and sediment-flux recurrences are tree/DAG sweeps and live with the
// other sweeps (fsb_chains.cu, fsb_flow.cu).
#include <cfloat>
#include <cmath>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

// catch(k) = catch0(root of k): basin b's root is roots[b-1] (basin ids are
// the order of the roots along the stack, roots ascending).
__global__ void k_catchment(int nn, const int* __restrict__ basins, const int* __restrict__ roots,
                            const double* __restrict__ catch0, double* __restrict__ catchv) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    catchv[k] = catch0[roots[basins[k] - 1]];
}

// slope in degrees on interior nodes, 0 on the edges (TerrainDerivatives.f90:3-35);
// the offsets are the reference's, 0-based.
__global__ void k_slope(int nx, int ny, double dx, double dy, double con, const double* __restrict__ h,
                        double* __restrict__ s) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    double v = 0.0;
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
      const int ia = k + nx - 1, ib = ia + 1, ic = ib + 1, id = k - 1, iff = k + 1;
      const int ig = k - nx - 1, ih = ig + 1, ii = ih + 1;
      const double dzdx = ((h[ic] + 2.0 * h[iff] + h[ii]) - (h[ia] + 2.0 * h[id] + h[ig])) / 8.0 / dx;
      const double dzdy = ((h[ig] + 2.0 * h[ih] + h[ii]) - (h[ia] + 2.0 * h[ib] + h[ic])) / 8.0 / dy;
      v = dzdx * dzdx + dzdy * dzdy;
      if (v > DBL_MIN) v = atan(sqrt(v)) * con;
    }
    s[k] = v;
  }
}

// curvature on interior nodes, 0 on the edges (TerrainDerivatives.f90:39-74)
__global__ void k_curvature(int nx, int ny, double dx, double dy, const double* __restrict__ h,
                            double* __restrict__ curv) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    double v = 0.0;
    if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
      const int i1 = k + nx - 1, i2 = i1 + 1, i3 = i2 + 1, i4 = k - 1, i5 = k, i6 = k + 1;
      const int i7 = k - nx - 1, i8 = i7 + 1, i9 = i8 + 1;
      const double a = (h[i1] + h[i3] + h[i4] + h[i6] + h[i7] + h[i9]) / dx / dx / 12.0 -
                       (h[i2] + h[i5] + h[i8]) / dx / dx / 6.0;
      const double b = (h[i1] + h[i2] + h[i3] + h[i7] + h[i8] + h[i9]) / dy / dy / 12.0 -
                       (h[i4] + h[i5] + h[i6]) / dy / dy / 6.0;
      const double c = (h[i3] + h[i7] - h[i1] - h[i9]) / dx / dy / 4.0;
      const double d = (h[i3] + h[i6] + h[i9] - h[i1] - h[i4] - h[i7]) / dx / 6.0;
      const double e = (h[i1] + h[i2] + h[i3] - h[i7] - h[i8] - h[i9]) / dy / 6.0;
      v = 1.0 + d * d + e * e;
      if (v > DBL_MIN) v = (a * (1.0 + e * e) + b * (1.0 + d * d) - c * d * e) / pow(v, 3.0 / 2.0);
    }
    curv[k] = v;
  }
}

__global__ void k_add_layers(int nn, const double* __restrict__ dh, double* __restrict__ h, double* __restrict__ b) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    h[k] = h[k] + dh[k];
    b[k] = b[k] + dh[k];
  }
}

// Sums of u, erate and the flux on fixed-boundary nodes, in a fixed order
// (per-thread strides, then a shared-memory tree per block, then one block
// over the block sums), so repeated calls give identical results.
constexpr int kSumBlocks = 512, kSumThreads = 256;

__global__ void __launch_bounds__(kSumThreads) k_flux_partials(Bounds bd, const double* __restrict__ u,
                                                               const double* __restrict__ erate,
                                                               const double* __restrict__ flux,
                                                               double* __restrict__ part) {
  __shared__ double sh[3][kSumThreads];
  const int nn = bd.nx * bd.ny;
  double su = 0.0, se = 0.0, sb = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    su += u[k];
    se += erate[k];
    if (is_bc_node(bd, k % bd.nx, k / bd.nx)) sb += flux[k];
  }
  sh[0][threadIdx.x] = su;
  sh[1][threadIdx.x] = se;
  sh[2][threadIdx.x] = sb;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) part[blockIdx.x * 3 + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void __launch_bounds__(kSumThreads) k_flux_final(const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[3][kSumThreads];
  for (int q = 0; q < 3; ++q) {
    double s = 0.0;
    for (int b = threadIdx.x; b < kSumBlocks; b += kSumThreads) s += part[b * 3 + q];
    sh[q][threadIdx.x] = s;
  }
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int q = 0; q < 3; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 3) out[threadIdx.x] = sh[threadIdx.x][0];
}

}  // namespace

void catchment(Ctx& c) {
  k_catchment<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, c.basins, c.s_roots, c.catch0, c.catchv);
  c.count_launch();
}

void slope_field(Ctx& c, double* out) {
  const double con = 45.0 / std::atan(1.0);
  k_slope<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, c.xl / (c.nx - 1), c.yl / (c.ny - 1), con, c.h, out);
  c.count_launch();
}

void curvature_field(Ctx& c, double* out) {
  k_curvature<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, c.xl / (c.nx - 1), c.yl / (c.ny - 1), c.h, out);
  c.count_launch();
}

void add_layers(Ctx& c, const double* dh) {
  k_add_layers<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, dh, c.h, c.b);
  c.count_launch();
}

// out3 (device): sum(u), sum(erate), sum of flux over fixed-boundary nodes;
// part: 3 * 512 doubles of scratch
void flux_sums(Ctx& c, const double* flux, double* part, double* out3) {
  k_flux_partials<<<kSumBlocks, kSumThreads, 0, c.stream>>>(c.bd, c.u, c.erate, flux, part);
  k_flux_final<<<1, kSumThreads, 0, c.stream>>>(part, out3);
  c.count_launch(2);
}

}  // namespace fsb
