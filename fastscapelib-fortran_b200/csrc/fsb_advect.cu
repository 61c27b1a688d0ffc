// Horizontal advection of h, basement and total erosion by the velocity field
// (vx, vy): implicit upwind ADI, an x-pass over every row then a y-pass over
// every column, each a tridiagonal solve per line for the three fields.
//
// Reference: Advect, src/Advect.f90:1-103 (run first in FastScape_Execute_Step,
// src/FastScape_api.f90:209-214; velocities from FastScape_Set_V, api:634 ->
// ctx:616-632).  Per element with v = vx (x-pass) or vy (y-pass):
//   v > 0: diag = 1 + v*dt/d, inf = -v*dt/d;  v < 0: diag = 1 - v*dt/d,
//   sup = v*dt/d;  otherwise diag = 1;  then sup(1) = 0, diag(1) = 1,
//   diag(n) = 1, inf(n) = 0;  solved with the same Thomas recurrence as
//   tridag (Diffusion.f90:164-202), here k_thomas.  Finally b = min(b, h).
//
// Layout: the y-pass systems are columns, element j of column i at j*nx + i,
// i.e. the fields' own layout with consecutive systems adjacent in memory, so
// they are solved in place.  The x-pass systems are rows; the coefficients are
// written transposed (element i of row j at i*ny + j) through a shared-memory
// tile and each field is transposed in and out around its solve.
#include "fsb_kernels.cuh"

namespace fsb {

namespace {

constexpr int kT = 32;  // transpose tile

// coefficients of one element; `first`/`last` are the line's ends
__device__ inline void adv_coef(double v, double dt, double d, bool first, bool last, double& inf, double& diag,
                                double& sup) {
  diag = 1.0;
  sup = 0.0;
  inf = 0.0;
  if (v > 0.0) {
    diag = 1.0 + v * dt / d;
    inf = -v * dt / d;
  } else if (v < 0.0) {
    diag = 1.0 - v * dt / d;
    sup = v * dt / d;
  }
  if (first) { sup = 0.0; diag = 1.0; }
  if (last) { diag = 1.0; inf = 0.0; }
}

// x-pass coefficients from vx (natural layout), written transposed:
// element i of row j at [i*ny + j]
__global__ void k_adv_xcoef(int nx, int ny, double dt, double dx, const double* __restrict__ vx,
                            double* __restrict__ A, double* __restrict__ B, double* __restrict__ C) {
  __shared__ double tv[kT][kT + 1];
  const int i0 = blockIdx.x * kT, j0 = blockIdx.y * kT;
  for (int r = threadIdx.y; r < kT; r += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + r;
    if (i < nx && j < ny) tv[r][threadIdx.x] = vx[(size_t)j * nx + i];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < kT; r += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + r;
    if (i < nx && j < ny) {
      double inf, diag, sup;
      adv_coef(tv[threadIdx.x][r], dt, dx, i == 0, i == nx - 1, inf, diag, sup);
      const size_t o = (size_t)i * ny + j;
      A[o] = inf;
      B[o] = diag;
      C[o] = sup;
    }
  }
}

// y-pass coefficients from vy, natural layout (element j of column i at j*nx + i)
__global__ void k_adv_ycoef(int nx, int ny, double dt, double dy, const double* __restrict__ vy,
                            double* __restrict__ A, double* __restrict__ B, double* __restrict__ C) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int j = k / nx;
    double inf, diag, sup;
    adv_coef(vy[k], dt, dy, j == 0, j == ny - 1, inf, diag, sup);
    A[k] = inf;
    B[k] = diag;
    C[k] = sup;
  }
}

// out[c*rows + r] = in[r*cols + c]
__global__ void k_transpose(int rows, int cols, const double* __restrict__ in, double* __restrict__ out) {
  __shared__ double t[kT][kT + 1];
  const int c0 = blockIdx.x * kT, r0 = blockIdx.y * kT;
  for (int y = threadIdx.y; y < kT; y += blockDim.y) {
    const int r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[y][threadIdx.x] = in[(size_t)r * cols + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < kT; y += blockDim.y) {
    const int c = c0 + y, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[(size_t)c * rows + r] = t[threadIdx.x][y];
  }
}

__global__ void k_min_b(int nn, const double* __restrict__ h, double* __restrict__ b) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) b[k] = fmin(b[k], h[k]);
}

}  // namespace

void advect(Ctx& c) {
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  cudaStream_t st = c.stream;
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  double *A = c.dA, *B = c.dB, *C = c.dC, *G = c.dG, *T = c.dK;
  double* fields[3] = {c.h, c.b, c.etot};
  const dim3 tb(kT, 8);
  // x-pass: one system per row j, element i at [i*ny + j]
  k_adv_xcoef<<<dim3((nx + kT - 1) / kT, (ny + kT - 1) / kT), tb, 0, st>>>(nx, ny, c.dt, dx, c.vx, A, B, C);
  c.count_launch();
  for (double* f : fields) {
    k_transpose<<<dim3((nx + kT - 1) / kT, (ny + kT - 1) / kT), tb, 0, st>>>(ny, nx, f, T);
    thomas_lines(c, nx, ny, 0, ny, A, B, C, T, G);
    k_transpose<<<dim3((ny + kT - 1) / kT, (nx + kT - 1) / kT), tb, 0, st>>>(nx, ny, T, f);
    c.count_launch(2);
  }
  // y-pass: one system per column i, element j at [j*nx + i], solved in place
  k_adv_ycoef<<<grid1d(nn), kBlock, 0, st>>>(nx, ny, c.dt, dy, c.vy, A, B, C);
  c.count_launch();
  for (double* f : fields) thomas_lines(c, ny, nx, 0, nx, A, B, C, f, G);
  k_min_b<<<grid1d(nn), kBlock, 0, st>>>(nn, c.h, c.b);
  c.count_launch();
}

}  // namespace fsb
