// Lake filling, multiple-flow receivers, drainage area, implicit stream power
// law and ADI hillslope diffusion.
//
// Reference routines restated here (fastscapelib-fortran file:line):
//   hwater fill + lake_depth              src/FlowRouting.f90:73-89 (SFD), :183-198 (MFD h0)
//   find_mult_rec                         src/FlowRouting.f90:147-298
//   FlowAccumulation(SingleFlowDirection) src/FlowRouting.f90:97-143
//   StreamPowerLaw(SingleFlowDirection)   src/StreamPowerLaw.f90:3-206, 210-400 (g == 0)
//   Diffusion + tridag                    src/Diffusion.f90:1-202
//
// Tree and DAG recurrences (fill, area, implicit erosion) run as wavefront
// sweeps over a topological order: warps claim windows of 32 consecutive
// positions through an atomic ticket, wait (bounded) for dependencies in
// earlier windows through per-node epoch flags, and resolve dependencies
// inside the window through a warp ballot and shared memory.  Every
// dependency sits at an earlier position, so a window only waits on windows
// claimed before it and the sweep cannot deadlock; each per-node formula
// keeps the reference's operation order, so single-flow results are
// bit-identical to the sequential loops.
#include <cuda/atomic>
#include <cfloat>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kWarps = 4;  // warps per block in the sweep kernels

__device__ inline unsigned long long ordered_key(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

__device__ inline bool flag_ready(const unsigned* done, int k, unsigned epoch) {
  cuda::atomic_ref<unsigned, cuda::thread_scope_device> f(*const_cast<unsigned*>(&done[k]));
  return f.load(cuda::memory_order_acquire) == epoch;
}

__device__ inline void flag_publish(unsigned* done, int k, unsigned epoch) {
  cuda::atomic_ref<unsigned, cuda::thread_scope_device> f(done[k]);
  f.store(epoch, cuda::memory_order_release);
}

// Order views: position -> node and node -> position.
struct Fwd {
  const int* ord;
  const int* pos;
  int n;
  __device__ int at(int p) const { return ord[p]; }
  __device__ int posof(int k) const { return pos[k]; }
};
struct Rev {
  const int* ord;
  const int* pos;
  int n;
  __device__ int at(int p) const { return ord[n - 1 - p]; }
  __device__ int posof(int k) const { return n - 1 - pos[k]; }
};

// Generic wavefront over an order.  Op provides
//   MAXDEP, Val, St,
//   int  init(k, St&, int* deps)                  node-local work, list of dependencies
//   Val  load(d)                                  dependency value from global memory
//   Val  compute(k, St&, nd, const int*, const Val*)
//   void store(k, const Val&)                     publish to global memory
template <class Op, class Order>
__global__ void __launch_bounds__(kWarps * 32) k_wavefront(Op op, Order od, unsigned* ticket, unsigned* done,
                                                           unsigned epoch, int* err) {
  using Val = typename Op::Val;
  __shared__ Val sval[kWarps][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(ticket, 1u);
    w = __shfl_sync(FULL, w, 0);
    const long long base = (long long)w * 32;
    if (base >= od.n) break;
    const int p = (int)base + lane;
    const int k = p < od.n ? od.at(p) : -1;
    typename Op::St st;
    int deps[Op::MAXDEP];
    Val dv[Op::MAXDEP];
    int dl[Op::MAXDEP];
    int nd = 0;
    unsigned intra = 0;  // bit s set: deps[s] sits in this window, at lane dl[s]
    if (k >= 0) {
      nd = op.init(k, st, deps);
      for (int s = 0; s < nd; ++s) {
        const int q = od.posof(deps[s]);
        if (q >= base + 32) {  // not a topological order: report, never wait
          atomicExch(err, DEV_STACK_ERROR);
        } else if (q >= base) {
          intra |= 1u << s;
          dl[s] = q - (int)base;
        } else {
          int spins = 0;
          while (!flag_ready(done, deps[s], epoch)) {
            if (++spins > kSpinLimit) { atomicExch(err, DEV_SPIN_LIMIT); break; }
            // once any wait has failed, stop waiting everywhere (results are void)
            if ((spins & 255) == 0 && *(volatile int*)err != 0) break;
            __nanosleep(20);
          }
          dv[s] = op.load(deps[s]);
        }
      }
    }
    bool mine = k < 0;
    // every pass completes at least the lowest unfinished lane: <= 32 passes
    for (int it = 0; it < 34; ++it) {
      const unsigned dmask = __ballot_sync(FULL, mine);
      if (dmask == FULL) break;
      if (!mine) {
        bool ready = true;
        for (int s = 0; s < nd; ++s)
          if ((intra >> s) & 1u) ready = ready && ((dmask >> dl[s]) & 1u);
        if (ready) {
          for (int s = 0; s < nd; ++s)
            if ((intra >> s) & 1u) dv[s] = sval[warp][dl[s]];
          const Val v = op.compute(k, st, nd, deps, dv);
          sval[warp][lane] = v;
          op.store(k, v);
          flag_publish(done, k, epoch);
          mine = true;
        }
      }
      __syncwarp();
    }
    if (!mine) atomicExch(err, DEV_SPIN_LIMIT);
    __syncwarp();
  }
}

// ---- hwater fill (FlowRouting.f90:73-89 / 183-198) --------------------------
struct FillOp {
  static constexpr int MAXDEP = 1;
  struct Val { double hw; };
  struct St { double hk; int r; };
  const int* rec;
  const double* h;
  double* hwater;
  double* lake_depth;
  __device__ int init(int k, St& s, int* deps) const {
    s.r = rec[k];
    s.hk = h[k];
    if (s.r == k) return 0;
    deps[0] = s.r;
    return 1;
  }
  __device__ Val load(int d) const { return Val{__ldcg(&hwater[d])}; }
  __device__ Val compute(int k, St& s, int, const int*, const Val* dv) const {
    if (s.r == k) return Val{s.hk};
    const double hr = dv[0].hw;
    return Val{hr > s.hk ? hr + 1.0e-8 : s.hk};
  }
  __device__ void store(int k, const Val& v) const {
    hwater[k] = v.hw;
    lake_depth[k] = v.hw - h[k];
  }
};

// ---- single-flow drainage area (FlowRouting.f90:123-143) --------------------
// The reverse-stack scatter a(rec)+=a(k) adds the donors of k in descending
// order: a(k) = dx*dy*precip(k) + a(d_m) + ... + a(d_1); a root also adds
// itself (a(rec(k)) with rec(k)==k), doubling its area.
struct AccumSfdOp {
  static constexpr int MAXDEP = 8;
  struct Val { double a; };
  struct St { double base; int root; };
  const int* rec;
  const int* ndon;
  const int* don;
  const double* precip;
  double dxdy;
  double* a;
  __device__ int init(int k, St& s, int* deps) const {
    s.base = dxdy * precip[k];
    s.root = rec[k] == k;
    const int nd = ndon[k];
    for (int i = 0; i < nd; ++i) deps[i] = don[(size_t)k * 8 + i];
    return nd;
  }
  __device__ Val load(int d) const { return Val{__ldcg(&a[d])}; }
  __device__ Val compute(int, St& s, int nd, const int*, const Val* dv) const {
    double acc = s.base;
    for (int i = nd - 1; i >= 0; --i) acc = acc + dv[i].a;
    if (s.root) acc = acc + acc;
    return Val{acc};
  }
  __device__ void store(int k, const Val& v) const { a[k] = v.a; }
};

// ---- multiple-flow drainage area (FlowRouting.f90:97-119) -------------------
// a(k) = dx*dy*precip(k) + sum over donors d and their slots s targeting k of
// a(d)*mwrec(s,d).  Donors come from the precomputed 3x3 donor mask.
struct AccumMfdOp {
  static constexpr int MAXDEP = 8;
  struct Val { double a; };
  struct St { double base; };
  Bounds bd;
  const int* mdmask;
  const int* mrec;
  const int* mnrec;
  const double* mwrec;
  const double* precip;
  double dxdy;
  double* a;
  __device__ int init(int k, St& s, int* deps) const {
    s.base = dxdy * precip[k];
    const int m = mdmask[k];
    const int i = k % bd.nx, j = k / bd.nx;
    int nd = 0;
    for (int t = 0; t < 9; ++t) {
      if (!((m >> t) & 1)) continue;
      int ii = i + (t % 3) - 1, jj = j + (t / 3) - 1;
      if (ii < 0) ii += bd.nx; else if (ii >= bd.nx) ii -= bd.nx;
      if (jj < 0) jj += bd.ny; else if (jj >= bd.ny) jj -= bd.ny;
      deps[nd++] = ii + jj * bd.nx;
    }
    return nd;
  }
  __device__ Val load(int d) const { return Val{__ldcg(&a[d])}; }
  __device__ Val compute(int k, St& s, int nd, const int* deps, const Val* dv) const {
    double acc = s.base;
    for (int q = 0; q < nd; ++q) {
      const int d = deps[q];
      const int nr = mnrec[d];
      for (int t = 0; t < nr; ++t)
        if (mrec[(size_t)d * 8 + t] == k) acc = acc + dv[q].a * mwrec[(size_t)d * 8 + t];
    }
    return Val{acc};
  }
  __device__ void store(int k, const Val& v) const { a[k] = v.a; }
};

// ---- implicit stream power law, g == 0 (StreamPowerLaw.f90) -----------------
// With g == 0 the Gauss-Seidel loop runs once with elev == ht; the sweep
// visits receivers before donors and writes the new elevation to hnew while
// h keeps ht (the elevation at the start of the step).
struct SplSfdOp {
  static constexpr int MAXDEP = 1;
  struct Val { double h, w; };
  struct St { double ht, fact, htr; int r; };
  const int* rec;
  const double* h;       // ht
  const double* b;
  const double* kf;
  const double* a;
  const double* length;
  double kfsed, kfdt, m, n, omega;
  bool n_is_one;
  double* hnew;
  double* water;
  __device__ int init(int k, St& s, int* deps) const {
    s.r = rec[k];
    s.ht = h[k];
    if (s.r == k) return 0;
    s.htr = h[s.r];
    // kfint = kf, or kfsed where h-b > 1 (StreamPowerLaw.f90:242-243)
    const double kfint = (kfsed > 0.0 && (s.ht - b[k]) > 1.0) ? kfsed : kf[k];
    if (n_is_one) s.fact = kfint * kfdt * pow(a[k], m) / length[k];
    else s.fact = kfint * kfdt * pow(a[k], m) / pow(length[k], n);
    deps[0] = s.r;
    return 1;
  }
  __device__ Val load(int d) const { return Val{__ldcg(&hnew[d]), __ldcg(&water[d])}; }
  __device__ Val compute(int k, St& s, int, const int*, const Val* dv) const {
    if (s.r == k) return Val{s.ht, s.ht};
    const double hr = dv[0].h, wr = dv[0].w;
    const double elev = s.ht;
    double hk = s.ht;
    if (elev > wr) {
      if (n_is_one) {
        double f = elev, df = 1.0;
        f = f + s.fact * hr;
        df = df + s.fact;
        hk = f / df;
      } else {
        const double tolp = 1.0e-3;
        double errp = 2.0 * tolp;
        const double h0 = elev;
        int guard = 0;
        while (errp > tolp && guard++ < 10000) {
          double f = hk - h0, df = 1.0;
          if (s.ht > s.htr) {
            const double x = fmax(0.0, hk - hr);
            f = f + s.fact * pow(x, n);
            df = df + s.fact * n * pow(x, n - 1.0);
          }
          const double hn = hk - f / df;
          errp = fabs(hn - hk);
          hk = hk * (1.0 - omega) + hn * omega;
        }
      }
      if (hk < wr) hk = wr;
    } else {
      hk = elev;
    }
    return Val{hk, fmax(wr, hk)};
  }
  __device__ void store(int k, const Val& v) const {
    hnew[k] = v.h;
    water[k] = v.w;
  }
};

struct SplMfdOp {
  static constexpr int MAXDEP = 9;
  struct Val { double h, w; };
  struct St { double ht; double fact[8]; int gate; int nr; int r; int rdep; };
  const int* rec;
  const int* mrec;
  const int* mnrec;
  const double* mwrec;
  const double* mlrec;
  const double* h;  // ht
  const double* b;
  const double* kf;
  const double* a;
  double kfsed, kfdt, m, n, omega;
  bool n_is_one;
  double* hnew;
  double* water;
  __device__ int init(int k, St& s, int* deps) const {
    s.r = rec[k];
    s.ht = h[k];
    s.gate = 0;
    s.rdep = -1;
    if (s.r == k) { s.nr = 0; return 0; }
    const int nr = mnrec[k];
    s.nr = nr;
    const double ak = a[k];
    // kfint = kf, or kfsed where h-b > 1 (StreamPowerLaw.f90:35-36)
    const double kk = ((kfsed > 0.0 && (s.ht - b[k]) > 1.0) ? kfsed : kf[k]) * kfdt;
    int nd = 0;
    for (int t = 0; t < nr; ++t) {
      const int q = mrec[(size_t)k * 8 + t];
      const double w = mwrec[(size_t)k * 8 + t], l = mlrec[(size_t)k * 8 + t];
      const double hq = h[q];
      const bool g = n_is_one ? (s.ht >= hq) : (s.ht > hq);
      if (g) s.gate |= 1 << t;
      s.fact[t] = n_is_one ? kk * pow(ak * w, m) / l : kk * pow(ak * w, m) / pow(l, n);
      deps[nd++] = q;
    }
    for (int t = 0; t < nd; ++t)
      if (deps[t] == s.r) s.rdep = t;
    if (s.rdep < 0) { s.rdep = nd; deps[nd++] = s.r; }
    return nd;
  }
  __device__ Val load(int d) const { return Val{__ldcg(&hnew[d]), __ldcg(&water[d])}; }
  __device__ Val compute(int k, St& s, int, const int*, const Val* dv) const {
    if (s.r == k) return Val{s.ht, s.ht};
    const double wr = dv[s.rdep].w;
    const double elev = s.ht;
    double hk = s.ht;
    if (elev > wr) {
      if (s.nr > 0) {
        if (n_is_one) {
          double f = elev, df = 1.0;
          for (int t = 0; t < s.nr; ++t)
            if ((s.gate >> t) & 1) {
              f = f + s.fact[t] * dv[t].h;
              df = df + s.fact[t];
            }
          hk = f / df;
        } else {
          const double tolp = 1.0e-3;
          double errp = 2.0 * tolp;
          const double h0 = elev;
          int guard = 0;
          while (errp > tolp && guard++ < 10000) {
            double f = hk - h0, df = 1.0;
            for (int t = 0; t < s.nr; ++t)
              if ((s.gate >> t) & 1) {
                const double x = fmax(0.0, hk - dv[t].h);
                f = f + s.fact[t] * pow(x, n);
                df = df + s.fact[t] * n * pow(x, n - 1.0);
              }
            const double hn = hk - f / df;
            errp = fabs(hn - hk);
            hk = hk * (1.0 - omega) + hn * omega;
          }
        }
      }
      if (hk < wr) hk = wr;
    } else {
      hk = elev;
    }
    return Val{hk, fmax(wr, hk)};
  }
  __device__ void store(int k, const Val& v) const {
    hnew[k] = v.h;
    water[k] = v.w;
  }
};

template <class Op, class Order>
void run_wavefront(Ctx& c, const Op& op, const Order& od) {
  c.epoch += 1;
  if (c.epoch == 0) {  // flags wrapped: clear them so no stale epoch matches
    cudaMemsetAsync(c.done, 0, sizeof(unsigned) * c.nn, c.stream);
    c.epoch = 1;
  }
  cudaMemsetAsync(c.ticket, 0, sizeof(unsigned), c.stream);
  int blocks = 148 * 8;
  k_wavefront<Op, Order><<<blocks, kWarps * 32, 0, c.stream>>>(op, od, c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

// ---- find_mult_rec (FlowRouting.f90:200-243) --------------------------------
__global__ void k_mfd_receivers(Bounds bd, double p, const double* __restrict__ h0, const double* __restrict__ ltab,
                                int* __restrict__ mrec, int* __restrict__ mnrec, double* __restrict__ mwrec,
                                double* __restrict__ mlrec) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int ij = blockIdx.x * blockDim.x + threadIdx.x; ij < nn; ij += gridDim.x * blockDim.x) {
    const int i = ij % nx, j = ij / nx;
    int nr = 0;
    double w[8];
    if (i >= bd.i1 && i <= bd.i2 && j >= bd.j1 && j <= bd.j2) {
      const double hij = h0[ij];
      for (int jj = -1; jj <= 1; ++jj) {
        const int jjj = wrap_clamp(j + jj, ny, bd.ycyc);
        for (int ii = -1; ii <= 1; ++ii) {
          const int iii = wrap_clamp(i + ii, nx, bd.xcyc);
          const int ijk = iii + jjj * nx;
          if (hij > h0[ijk]) {
            const double l = ltab[(jj + 1) * 3 + (ii + 1)];
            mrec[(size_t)ij * 8 + nr] = ijk;
            mlrec[(size_t)ij * 8 + nr] = l;
            w[nr] = (hij - h0[ijk]) / l;
            ++nr;
          }
        }
      }
    }
    double pe = p;
    if (p < 0.0) {
      double slope = 0.0;
      if (nr != 0) {
        double s = 0.0;
        for (int t = 0; t < nr; ++t) s = s + w[t];
        slope = (double)(float)(s / nr);
      }
      pe = (double)0.5f + (double)0.6f * slope;
    }
    for (int t = 0; t < nr; ++t) w[t] = pow(w[t], pe);
    double sumw = 0.0;
    for (int t = 0; t < nr; ++t) sumw = sumw + w[t];
    for (int t = 0; t < nr; ++t) mwrec[(size_t)ij * 8 + t] = w[t] / sumw;
    for (int t = nr; t < 8; ++t) { mrec[(size_t)ij * 8 + t] = -1; mwrec[(size_t)ij * 8 + t] = 0.0; mlrec[(size_t)ij * 8 + t] = 0.0; }
    mnrec[ij] = nr;
  }
}

// donor mask over the 3x3 block (bit (jj+1)*3+(ii+1)) for the pull-form accumulation
__global__ void k_mfd_donor_mask(Bounds bd, const int* __restrict__ mrec, const int* __restrict__ mnrec,
                                 int* __restrict__ mask) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    int m = 0;
    int seen[9];
    int ns = 0;
    for (int jj = -1; jj <= 1; ++jj) {
      int y = j + jj;
      if (y < 0) { if (!bd.ycyc) continue; y += ny; }
      if (y >= ny) { if (!bd.ycyc) continue; y -= ny; }
      for (int ii = -1; ii <= 1; ++ii) {
        int x = i + ii;
        if (x < 0) { if (!bd.xcyc) continue; x += nx; }
        if (x >= nx) { if (!bd.xcyc) continue; x -= nx; }
        const int d = x + y * nx;
        if (d == k) continue;
        bool dup = false;
        for (int t = 0; t < ns; ++t) dup |= seen[t] == d;
        if (dup) continue;
        seen[ns++] = d;
        const int nr = mnrec[d];
        for (int t = 0; t < nr; ++t)
          if (mrec[(size_t)d * 8 + t] == k) { m |= 1 << ((jj + 1) * 3 + (ii + 1)); break; }
      }
    }
    mask[k] = m;
  }
}

// topological order for the MFD sweeps: ascending h0, ties in stack order
__global__ void k_order_keys(int nn, const int* __restrict__ stack, const double* __restrict__ h0,
                             unsigned long long* __restrict__ keys, int* __restrict__ vals) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
    const int k = stack[p];
    keys[p] = ordered_key(h0[k]);
    vals[p] = k;
  }
}

__global__ void k_order_finish(int nn, const int* __restrict__ ord, int* __restrict__ pos, int* __restrict__ mstack) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
    const int k = ord[p];
    pos[k] = p;
    mstack[nn - 1 - p] = k;  // reference orientation: donors before receivers
  }
}

// SPL epilogue (StreamPowerLaw.f90:380-393 with g == 0): b=min(h,b),
// etot=etot+ht-h, erate=(ht-h)/dt, Sedflux=ht-h.
__global__ void k_spl_finish(int nn, double dt, const double* __restrict__ hnew, double* __restrict__ h,
                             double* __restrict__ b, double* __restrict__ etot, double* __restrict__ erate,
                             double* __restrict__ sedflux) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double ht = h[k], hn = hnew[k];
    b[k] = fmin(hn, b[k]);
    etot[k] = etot[k] + ht - hn;
    erate[k] = (ht - hn) / dt;
    sedflux[k] = ht - hn;
    h[k] = hn;
  }
}

// ---- ADI diffusion (Diffusion.f90) ------------------------------------------
__device__ inline double fcoef(double k1, double k2, double dt2, double d2) { return (k1 + k2) / 2.0 * dt2 / d2; }

__global__ void k_diff_kdint(int nn, double kdsed, const double* __restrict__ kd, const double* __restrict__ h,
                             const double* __restrict__ b, double* __restrict__ kdint) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    double v = kd[k];
    if (kdsed > 0.0 && (h[k] - b[k]) > 1.0e-6) v = kdsed;
    kdint[k] = v;
  }
}

// x pass coefficients for rows j=1..ny-2, stored transposed: element i of
// row j at [i*ny + j]
__global__ void k_diff_xcoef(Bounds bd, double dt2, double dx2, double dy2, const double* __restrict__ K,
                             const double* __restrict__ z, double* __restrict__ A, double* __restrict__ B,
                             double* __restrict__ C, double* __restrict__ F) {
  const int nx = bd.nx, ny = bd.ny;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y + 1;
  if (i >= nx || j > ny - 2) return;
  const size_t o = (size_t)i * ny + j;
  auto Kv = [&](int x, int y) { return K[x + (size_t)y * nx]; };
  auto Z = [&](int x, int y) { return z[x + (size_t)y * nx]; };
  double a = 0.0, bb, c = 0.0, f;
  if (i >= 1 && i <= nx - 2) {
    const double fxp = fcoef(Kv(i + 1, j), Kv(i, j), dt2, dx2);
    const double fxm = fcoef(Kv(i - 1, j), Kv(i, j), dt2, dx2);
    const double fyp = fcoef(Kv(i, j + 1), Kv(i, j), dt2, dy2);
    const double fym = fcoef(Kv(i, j - 1), Kv(i, j), dt2, dy2);
    bb = 1.0 + fxp + fxm;
    c = -fxp;
    a = -fxm;
    f = Z(i, j) + fyp * Z(i, j + 1) - (fyp + fym) * Z(i, j) + fym * Z(i, j - 1);
  } else if (i == 0) {
    if (bd.fix_left) {
      bb = 1.0; c = 0.0; f = Z(0, j);
    } else {
      const double fxp = fcoef(Kv(1, j), Kv(0, j), dt2, dx2);
      const double fyp = fcoef(Kv(0, j + 1), Kv(0, j), dt2, dy2);
      const double fym = fcoef(Kv(0, j - 1), Kv(0, j), dt2, dy2);
      bb = 1.0 + fxp;
      c = -fxp;
      f = Z(0, j) + fyp * Z(0, j + 1) - (fyp + fym) * Z(0, j) + fym * Z(0, j - 1);
    }
  } else {
    if (bd.fix_right) {
      bb = 1.0; a = 0.0; f = Z(nx - 1, j);
    } else {
      const double fxm = fcoef(Kv(nx - 2, j), Kv(nx - 1, j), dt2, dx2);
      const double fyp = fcoef(Kv(nx - 1, j + 1), Kv(nx - 1, j), dt2, dy2);
      const double fym = fcoef(Kv(nx - 1, j - 1), Kv(nx - 1, j), dt2, dy2);
      bb = 1.0 + fxm;
      a = -fxm;
      f = Z(nx - 1, j) + fyp * Z(nx - 1, j + 1) - (fyp + fym) * Z(nx - 1, j) + fym * Z(nx - 1, j - 1);
    }
  }
  A[o] = a; B[o] = bb; C[o] = c; F[o] = f;
}

// y pass coefficients for columns i=1..nx-2 (natural layout [j*nx + i])
__global__ void k_diff_ycoef(Bounds bd, double dt2, double dx2, double dy2, const double* __restrict__ K,
                             const double* __restrict__ z, double* __restrict__ A, double* __restrict__ B,
                             double* __restrict__ C, double* __restrict__ F) {
  const int nx = bd.nx, ny = bd.ny;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < 1 || i > nx - 2 || j >= ny) return;
  const size_t o = (size_t)j * nx + i;
  auto Kv = [&](int x, int y) { return K[x + (size_t)y * nx]; };
  auto Z = [&](int x, int y) { return z[x + (size_t)y * nx]; };
  double a = 0.0, bb, c = 0.0, f;
  if (j >= 1 && j <= ny - 2) {
    const double fxp = fcoef(Kv(i + 1, j), Kv(i, j), dt2, dx2);
    const double fxm = fcoef(Kv(i - 1, j), Kv(i, j), dt2, dx2);
    const double fyp = fcoef(Kv(i, j + 1), Kv(i, j), dt2, dy2);
    const double fym = fcoef(Kv(i, j - 1), Kv(i, j), dt2, dy2);
    bb = 1.0 + fyp + fym;
    c = -fyp;
    a = -fym;
    f = Z(i, j) + fxp * Z(i + 1, j) - (fxp + fxm) * Z(i, j) + fxm * Z(i - 1, j);
  } else if (j == 0) {
    if (bd.fix_bottom) {
      bb = 1.0; c = 0.0; f = Z(i, 0);
    } else {
      // the reference reads kdint(i,j) with j left at ny by the preceding loop
      const double fxp = fcoef(Kv(i + 1, 0), Kv(i, ny - 1), dt2, dx2);
      const double fxm = fcoef(Kv(i - 1, 0), Kv(i, 0), dt2, dx2);
      const double fyp = fcoef(Kv(i, 1), Kv(i, 0), dt2, dy2);
      bb = 1.0 + fyp;
      c = -fyp;
      f = Z(i, 0) + fxp * Z(i + 1, 0) - (fxp + fxm) * Z(i, 0) + fxm * Z(i - 1, 0);
    }
  } else {
    if (bd.fix_top) {
      bb = 1.0; a = 0.0; f = Z(i, ny - 1);
    } else {
      const double fxp = fcoef(Kv(i + 1, ny - 1), Kv(i, ny - 1), dt2, dx2);
      const double fxm = fcoef(Kv(i - 1, ny - 1), Kv(i, ny - 1), dt2, dx2);
      const double fym = fcoef(Kv(i, ny - 2), Kv(i, ny - 1), dt2, dy2);
      bb = 1.0 + fym;
      a = -fym;
      f = Z(i, ny - 1) + fxp * Z(i + 1, ny - 1) - (fxp + fxm) * Z(i, ny - 1) + fxm * Z(i - 1, ny - 1);
    }
  }
  A[o] = a; B[o] = bb; C[o] = c; F[o] = f;
}

// tridag (Diffusion.f90:164-202) for independent systems s in [s0, s1):
// element t of system s at [t*L + s]; the solution overwrites F.
__global__ void k_thomas(int N, int L, int s0, int s1, const double* __restrict__ A, const double* __restrict__ B,
                         const double* __restrict__ C, double* __restrict__ F, double* __restrict__ G,
                         int* __restrict__ err) {
  const int s = s0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= s1) return;
  double bet = B[s];
  if (bet == 0.0) { atomicExch(err, DEV_TRIDAG_ZERO); return; }
  double up = F[s] / bet;
  F[s] = up;
  for (int t = 1; t < N; ++t) {
    const size_t o = (size_t)t * L + s;
    const double g = C[o - L] / bet;
    G[o] = g;
    bet = B[o] - A[o] * g;
    if (bet == 0.0) { atomicExch(err, DEV_TRIDAG_ZERO); return; }
    up = (F[o] - A[o] * up) / bet;
    F[o] = up;
  }
  for (int t = N - 2; t >= 0; --t) {
    const size_t o = (size_t)t * L + s;
    up = F[o] - G[o + L] * up;
    F[o] = up;
  }
}

// zint = x-pass result on rows 1..ny-2, h elsewhere (natural layout)
__global__ void k_diff_xgather(Bounds bd, const double* __restrict__ Ux, const double* __restrict__ h,
                               double* __restrict__ zint) {
  __shared__ double tile[32][33];
  const int nx = bd.nx, ny = bd.ny;
  // tile over (i, j): read Ux[i*ny + j] coalesced along j, write zint coalesced along i
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + r, j = j0 + threadIdx.x;
    if (i < nx && j < ny) tile[r][threadIdx.x] = Ux[(size_t)i * ny + j];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + r, i = i0 + threadIdx.x;
    if (i < nx && j < ny) {
      const size_t o = (size_t)j * nx + i;
      zint[o] = (j >= 1 && j <= ny - 2) ? tile[threadIdx.x][r] : h[o];
    }
  }
}

// result: zintp = y-pass result on columns 1..nx-2, h elsewhere (Diffusion.f90:143-152)
__global__ void k_diff_finish(Bounds bd, double dt, const double* __restrict__ Uy, double* __restrict__ h,
                              double* __restrict__ b, double* __restrict__ etot, double* __restrict__ erate) {
  const int nx = bd.nx, nn = nx * bd.ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx;
    const double hk = h[k];
    const double zp = (i >= 1 && i <= nx - 2) ? Uy[k] : hk;
    etot[k] = etot[k] + hk - zp;
    erate[k] = erate[k] + (hk - zp) / dt;
    h[k] = zp;
    b[k] = fmin(zp, b[k]);
  }
}

}  // namespace

// ============================================================================

void fill_sweep(Ctx& c) {
  FillOp op{c.rec, c.h, c.hwater, c.lake_depth};
  run_wavefront(c, op, Fwd{c.stack, c.pos, c.nn});
}

void mfd_receivers(Ctx& c) {
  const int nn = c.nn;
  k_mfd_receivers<<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.p, c.hwater, c.ltab, c.mrec, c.mnrec, c.mwrec, c.mlrec);
  k_mfd_donor_mask<<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.mrec, c.mnrec, c.mdmask);
  k_order_keys<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.stack, c.hwater, c.o_keys, c.o_vals);
  c.count_launch(3);
  sort_pairs_u64(c, c.o_keys, c.o_keys2, c.o_vals, c.o_vals2, nn);
  k_order_finish<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.o_vals2, c.o_pos, c.mstack);
  c.count_launch();
}

void accumulate(Ctx& c) {
  const double dxdy = c.dx * c.dy;
  if (c.sfd) {
    AccumSfdOp op{c.rec, c.ndon, c.don, c.precip, dxdy, c.a};
    run_wavefront(c, op, Rev{c.stack, c.pos, c.nn});
  } else {
    AccumMfdOp op{c.bd, c.mdmask, c.mrec, c.mnrec, c.mwrec, c.precip, dxdy, c.a};
    run_wavefront(c, op, Rev{c.o_vals2, c.o_pos, c.nn});
  }
}

void stream_power(Ctx& c) {
  const bool n1 = fabs(c.n - 1.0) < DBL_MIN;
  const double omega = 0.875 / c.n;
  double* hnew = c.hnew;
  if (c.sfd) {
    SplSfdOp op{c.rec, c.h, c.b, c.kf, c.a, c.length, c.kfsed, c.dt, c.m, c.n, omega, n1, hnew, c.water};
    run_wavefront(c, op, Fwd{c.stack, c.pos, c.nn});
  } else {
    SplMfdOp op{c.rec, c.mrec, c.mnrec, c.mwrec, c.mlrec, c.h, c.b, c.kf, c.a, c.kfsed, c.dt, c.m, c.n, omega, n1,
                hnew, c.water};
    run_wavefront(c, op, Fwd{c.o_vals2, c.o_pos, c.nn});
  }
  k_spl_finish<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, c.dt, hnew, c.h, c.b, c.etot, c.erate, c.sedflux);
  c.count_launch();
}

void diffusion(Ctx& c) {
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  const double dt2 = c.dt / 2.0, dx2 = c.dx * c.dx, dy2 = c.dy * c.dy;
  double *K = c.dK, *A = c.dA, *B = c.dB, *C = c.dC, *F = c.dF, *G = c.dG;
  k_diff_kdint<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.kdsed, c.kd, c.h, c.b, K);
  c.count_launch();
  if (ny >= 3) {
    dim3 g((nx + 127) / 128, ny - 2);
    k_diff_xcoef<<<g, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, c.h, A, B, C, F);
    // systems are rows j=1..ny-2 with element i at [i*ny + j]
    k_thomas<<<(ny - 2 + 63) / 64, 64, 0, c.stream>>>(nx, ny, 1, ny - 1, A, B, C, F, G, c.d_err);
    c.count_launch(2);
  }
  double* Z = c.dZ;
  {
    dim3 g((nx + 31) / 32, (ny + 31) / 32);
    k_diff_xgather<<<g, dim3(32, 8), 0, c.stream>>>(c.bd, F, c.h, Z);
    c.count_launch();
  }
  if (nx >= 3) {
    dim3 g((nx + 127) / 128, ny);
    k_diff_ycoef<<<g, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, Z, A, B, C, F);
    k_thomas<<<(nx - 2 + 63) / 64, 64, 0, c.stream>>>(ny, nx, 1, nx - 1, A, B, C, F, G, c.d_err);
    c.count_launch(2);
  }
  k_diff_finish<<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.dt, F, c.h, c.b, c.etot, c.erate);
  c.count_launch();
}

}  // namespace fsb
