// Region-owned sweeps of the multiple-flow receiver DAG: drainage area and
// the implicit stream power law with g == 0.
//
// Reference loops restated (fastscapelib-fortran file:line):
//   FlowAccumulation (MFD)   src/FlowRouting.f90:97-119
//   StreamPowerLaw (MFD)     src/StreamPowerLaw.f90:89-177 (g == 0: one
//                            Gauss-Seidel pass, elev = ht)
//
// Both sweeps are recurrences along the receiver DAG whose critical path is
// about three grid sides long, so their time is the number of hops on that
// path times the latency of one hop.  Here the grid is cut into 2^a x 2^b
// tiles, one co-resident CTA per tile (cooperative launch), and nodes are
// numbered tile-major (a tile's nodes are contiguous).  A CTA keeps its
// tile's dependency counters (one byte per node, four to a word) and its
// ready queue in shared memory: a hop between two nodes of one tile is a
// shared-memory atomic and loads that the SM's L1 serves, not an L2 round
// trip.  Every node's value lands once in a tile-major value array, from
// which its dependents gather it, so no input slots need resetting.  A
// dependency that crosses a tile boundary goes through a global counter; its
// last producer posts the node into the owning CTA's inbox (release/acquire
// at GPU scope), which one lane of the CTA polls.  The arithmetic of a node,
// including the order of its sums, is that of the queue engine in
// fsb_flow.cu, so both engines give bit-identical results.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

// Co-resident sweep CTAs per SM the tile plan counts on.  The threads of a
// sweep CTA (warp 0 polls the inbox, the others compute nodes) are the op's
// kThreads: 512 where its registers allow two such CTAs per SM -- more
// worker warps per tile measured faster at 2049^2 (stream-power sweep 32 ->
// 16 ms against 256 threads).
constexpr int kRegionCtasPerSm = 2;
constexpr unsigned short kQEmpty = 0xFFFF;
constexpr unsigned long long kRegionTimeLimitNs = 4000000000ull;  // a sweep giving up: 4 s

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// weak load that the SM's L1 may serve (values written by this CTA)
__device__ __forceinline__ double ld_l1(const double* p) {
  double v;
  asm volatile("ld.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ double2 ld_l1(const double2* p) {
  double2 v;
  asm volatile("ld.global.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p) : "memory");
  return v;
}
// load from L2 (values written by other SMs, after an acquire)
__device__ __forceinline__ double ld_l2(const double* p) {
  double v;
  asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ double2 ld_l2(const double2* p) {
  double2 v;
  asm volatile("ld.global.cg.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_l1f(const float* p) {
  float v;
  asm volatile("ld.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_l2f(const float* p) {
  float v;
  asm volatile("ld.global.cg.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_globalf(float* p, float v) {
  asm volatile("st.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ void st_global(double* p, double v) {
  asm volatile("st.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_global(double2* p, double2 v) {
  asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(p), "d"(v.x), "d"(v.y) : "memory");
}
__device__ __forceinline__ void st_relaxed_gpu_int(int* p, int v) {
  asm volatile("st.relaxed.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

__device__ inline unsigned short prio16(int size) { return (unsigned short)(__float_as_uint((float)size) >> 16); }

// Inserts node v of priority p into dep[0..n) / pr[0..n) (n < 8), kept in
// decreasing priority with ties in insertion order (registers only).
__device__ inline void insert_by_priority(int (&dep)[8], unsigned (&pr)[8], int n, int v, unsigned p) {
  int pos = 0;
#pragma unroll
  for (int t = 0; t < 8; ++t) pos += (t < n && pr[t] >= p) ? 1 : 0;
#pragma unroll
  for (int t = 7; t > 0; --t)
    if (t > pos && t <= n) {
      dep[t] = dep[t - 1];
      pr[t] = pr[t - 1];
    }
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (t == pos) {
      dep[t] = v;
      pr[t] = p;
    }
}
template <class T>
__device__ inline void set_at(T (&a)[8], int n, T v) {
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (t == n) a[t] = v;
}
template <class T>
__device__ inline bool contains(const T (&a)[8], int n, T v) {
  bool f = false;
#pragma unroll
  for (int t = 0; t < 8; ++t) f |= t < n && a[t] == v;
  return f;
}

// Coordinates of q if it is one of the 3x3 neighbours of (i, j), rows and
// columns wrapping across the grid's edges; the row is found by range compares
// (q lies in row j-1, j or j+1, or in a wrapped edge row), so the common
// case needs no integer division.  False if q is not a neighbour.
__device__ inline bool nbr_of(int i, int j, int q, int nx, int ny, int& qi, int& qj) {
  const int r0 = j * nx;
  int y;
  if (q >= r0 && q < r0 + nx) y = j;
  else if (q < r0 && q >= r0 - nx) y = j - 1;
  else if (q >= r0 + nx && q < r0 + 2 * nx) y = j + 1;
  else if (q >= 0 && q < nx) y = 0;
  else if (q >= (ny - 1) * nx && q < ny * nx) y = ny - 1;
  else return false;
  const int x = q - y * nx;
  int di = x - i, dj = y - j;
  if (di > 1) di -= nx; else if (di < -1) di += nx;
  if (dj > 1) dj -= ny; else if (dj < -1) dj += ny;
  if (di < -1 || di > 1 || dj < -1 || dj > 1 || (di == 0 && dj == 0)) return false;
  qi = x;
  qj = y;
  return true;
}

// tile-major index of receiver q of (i, j), reporting a non-neighbour
__device__ inline int nbr_g(const TileMap& tm, int i, int j, int q, int nx, int ny, int* err) {
  int qi, qj;
  if (!nbr_of(i, j, q, nx, ny, qi, qj)) {
    atomicExch(err, DEV_NOT_ADJACENT);
    qi = q % nx;
    qj = q / nx;
  }
  return tm.g(qi, qj);
}

// The slots of d's receiver row that hold k, as bits (rows are padded with -1
// past mnrec, so all eight slots are compared: two 16-byte loads)
__device__ inline unsigned row_hits(const int* __restrict__ mrec, int d, int k) {
  const int4* r = reinterpret_cast<const int4*>(mrec + (size_t)d * 8);
  const int4 a = __ldg(r), b = __ldg(r + 1);
  return (unsigned)(a.x == k) | (unsigned)(a.y == k) << 1 | (unsigned)(a.z == k) << 2 | (unsigned)(a.w == k) << 3 |
         (unsigned)(b.x == k) << 4 | (unsigned)(b.y == k) << 5 | (unsigned)(b.z == k) << 6 | (unsigned)(b.w == k) << 7;
}

// One record line per node, tile-major: the inputs a node gathers, their
// coefficients, and its dependents (tile-major indices, -1 past the last;
// dependents largest priority first).
//   area:          c[t] = summed weight of input (donor) t's slots targeting k
//   stream power:  c[t] = kf*dt*(a*w)^m/l^n of gated receiver slot t
// The coefficients are double in the plain form and float in the mixed one.
template <class T>
struct __align__(128) RegionLineT {
  T c[8];
  int dep[8];
  int inp[8];
};
using RegionLine = RegionLineT<double>;
using RegionLineF = RegionLineT<float>;
static_assert(sizeof(RegionLine) == 128 && sizeof(RegionLineF) == 128, "one line per node");

// a line in registers: the words that hold data (128 bytes, or 96 with float
// coefficients), read through the read-only path
template <class T>
struct LineRegsT {
  static constexpr int kWords = (8 * (int)sizeof(T) + 64) / 16;
  static constexpr int kDep = 2 * (int)sizeof(T);  // int index of dep[0]
  union {
    int4 v[kWords];
    T c[8];
    int s[4 * kWords];
  };
  __device__ explicit LineRegsT(const RegionLineT<T>* p) {
#pragma unroll
    for (int t = 0; t < kWords; ++t) v[t] = __ldg(reinterpret_cast<const int4*>(p) + t);
  }
  __device__ int dep(int t) const { return s[kDep + t]; }
  __device__ int inp(int t) const { return s[kDep + 8 + t]; }
};
using LineRegs = LineRegsT<double>;

// stream-power node metadata kept in the value array's water word until the
// node is computed: rec (tile-major, or -1 for a root) and whether mnrec > 0
__device__ inline double pack_meta(int rec_g, bool has_mrec) {
  const long long v = (long long)(unsigned)rec_g | (has_mrec ? (1ll << 40) : 0ll);
  return __longlong_as_double(v);
}
__device__ inline void unpack_meta(double w, int& rec_g, bool& has_mrec) {
  const long long v = __double_as_longlong(w);
  rec_g = (int)(unsigned)(v & 0xffffffffll);
  has_mrec = (v >> 40) & 1;
}

// ---- line builders (natural node order in, tile-major out) ------------------

// Area: inputs are k's distinct donors among its 3x3 neighbours (jj outer, ii
// inner, as FlowRouting.f90's neighbour loops) with the summed weight of
// their slots targeting k; dependents are k's distinct receivers.  cnt0 gets
// the in-tile input count plus one if any input lies in another tile (that
// token is released by the inbox); xcnt the number of cross-tile inputs.
template <class T>
__global__ void k_acc_lines_t(Bounds bd, TileMap tm, double dxdy, const int* __restrict__ mrec,
                              const int* __restrict__ mnrec, const double* __restrict__ mwrec,
                              const double* __restrict__ precip, const int* __restrict__ prio,
                              RegionLineT<T>* __restrict__ line, T* __restrict__ val,
                              unsigned char* __restrict__ cnt0, int* __restrict__ xcnt, int* err) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    const int gk = tm.g(i, j);
    const int tile = gk >> tm.lr();
    const size_t o = (size_t)k * 8;
    const int nr = mnrec[k];
    int mr[8], dep[8];
    unsigned pr[8];
    {  // the row past mnrec holds -1
      const int4 ra = __ldg(reinterpret_cast<const int4*>(mrec + o)), rb = __ldg(reinterpret_cast<const int4*>(mrec + o) + 1);
      mr[0] = ra.x; mr[1] = ra.y; mr[2] = ra.z; mr[3] = ra.w;
      mr[4] = rb.x; mr[5] = rb.y; mr[6] = rb.z; mr[7] = rb.w;
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      dep[t] = -1;
      pr[t] = 0u;
    }
    int rn = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t >= nr) break;
      const int q = mr[t];
      if (contains(mr, t, q)) continue;
      insert_by_priority(dep, pr, rn++, nbr_g(tm, i, j, q, nx, ny, err), prio16(prio[q]));
    }
    int inp[8], seen[8];
    double aw[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      aw[t] = 0.0;
      inp[t] = -1;
    }
    int an = 0, ns = 0, nin = 0, nx_in = 0;
#pragma unroll
    for (int jj = -1; jj <= 1; ++jj) {
      int y = j + jj;
      if (y < 0) { if (!bd.ycyc) continue; y += ny; }
      if (y >= ny) { if (!bd.ycyc) continue; y -= ny; }
#pragma unroll
      for (int ii = -1; ii <= 1; ++ii) {
        int x = i + ii;
        if (x < 0) { if (!bd.xcyc) continue; x += nx; }
        if (x >= nx) { if (!bd.xcyc) continue; x -= nx; }
        const int d = x + y * nx;
        if (d == k || contains(seen, ns, d)) continue;
        set_at(seen, ns++, d);
        const unsigned hm = row_hits(mrec, d, k);
        double wsum = 0.0;
        int hits = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (hm >> t & 1u) {
            const double w = mwrec[(size_t)d * 8 + t];
            wsum = hits ? wsum + w : w;
            ++hits;
          }
        if (hits && an < 8) {
          const int gd = tm.g(x, y);
          set_at(inp, an, gd);
          set_at(aw, an++, wsum);
          if ((gd >> tm.lr()) == tile) ++nin; else ++nx_in;
        }
      }
    }
    RegionLineT<T> L;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      L.c[t] = (T)aw[t];
      L.dep[t] = dep[t];
      L.inp[t] = inp[t];
    }
    line[gk] = L;
    val[gk] = (T)(dxdy * precip[k]);
    cnt0[gk] = (unsigned char)(nin + (nx_in > 0 ? 1 : 0));
    xcnt[gk] = nx_in;
  }
}

// Stream power: inputs are k's gated receiver slots (ht(k) >= ht(q) for n = 1,
// > otherwise: the terms StreamPowerLaw.f90:108-114 / 152-158 include), in
// mrec slot order, duplicates kept; the counter also waits for rec(k), whose
// water the node compares against.  Dependents are the donors that read
// k's new elevation (gated) or its water (rec == k).  The value array starts
// as (ht, metadata) and ends as (h, water).
template <class T>
__global__ void k_spl_lines_t(Bounds bd, TileMap tm, int n_is_one, double kfsed, double dt, double m, double n,
                              const int* __restrict__ rec, const int* __restrict__ mrec,
                              const int* __restrict__ mnrec, const double* __restrict__ mwrec,
                              const double* __restrict__ mlrec, const double* __restrict__ h,
                              const double* __restrict__ b, const double* __restrict__ kf,
                              const double* __restrict__ a, const int* __restrict__ prio,
                              const double* __restrict__ ltab, const T* __restrict__ lpow,
                              RegionLineT<T>* __restrict__ line, double2* __restrict__ hw,
                              unsigned char* __restrict__ cnt0, int* __restrict__ xcnt, int* err) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  const double l_diag = __ldg(&ltab[0]), l_dy = __ldg(&ltab[1]);
  const T lp_diag = __ldg(&lpow[0]), lp_dy = __ldg(&lpow[1]), lp_dx = __ldg(&lpow[3]);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    const int gk = tm.g(i, j);
    const int tile = gk >> tm.lr();
    const size_t o = (size_t)k * 8;
    const double htk = h[k];
    const int nr = mnrec[k];
    const int r = rec[k];
    const double kk = ((kfsed > 0.0 && (htk - b[k]) > 1.0) ? kfsed : kf[k]) * dt;
    const double ak = a[k];
    int qv[8], inp[8], dep[8];
    unsigned pr[8];
    T fact[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      qv[t] = -1;
      inp[t] = -1;
      dep[t] = -1;
      pr[t] = 0u;
      fact[t] = 0;
    }
    int nq = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t >= nr) break;
      const int q = mrec[o + t];
      if (n_is_one ? (htk >= h[q]) : (htk > h[q])) {
        const double w = mwrec[o + t], l = mlrec[o + t];
        // l^n from the table of the neighbour lengths: l is one of its three
        // values (diagonal at 0, dy at 1, dx at 3; equal values have equal powers)
        const T ln = l == l_diag ? lp_diag : l == l_dy ? lp_dy : lp_dx;
        if constexpr (sizeof(T) == sizeof(double)) {
          set_at(fact, nq, n_is_one ? kk * pow(ak * w, m) / l : kk * pow(ak * w, m) / ln);
        } else {  // mixed precision: the erosion factor in FP32
          const float kf32 = (float)kk, aw32 = (float)(ak * w), l32 = (float)l;
          set_at(fact, nq, n_is_one ? kf32 * powf(aw32, (float)m) / l32 : kf32 * powf(aw32, (float)m) / ln);
        }
        set_at(inp, nq, nbr_g(tm, i, j, q, nx, ny, err));
        set_at(qv, nq++, q);
      }
    }
    // distinct inputs: gated receivers and rec(k), split by tile
    int nin = 0, nx_in = 0;
    const int rg = r != k ? nbr_g(tm, i, j, r, nx, ny, err) : -1;
    if (r != k) {
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < nq && !contains(qv, t, qv[t])) {
          if ((inp[t] >> tm.lr()) == tile) ++nin; else ++nx_in;
        }
      if (!contains(qv, nq, r)) {
        if ((rg >> tm.lr()) == tile) ++nin; else ++nx_in;
      }
    }
    int dn = 0, ns = 0;
    int seen[8];
#pragma unroll
    for (int jj = -1; jj <= 1; ++jj) {
      int y = j + jj;
      if (y < 0) { if (!bd.ycyc) continue; y += ny; }
      if (y >= ny) { if (!bd.ycyc) continue; y -= ny; }
#pragma unroll
      for (int ii = -1; ii <= 1; ++ii) {
        int x = i + ii;
        if (x < 0) { if (!bd.xcyc) continue; x += nx; }
        if (x >= nx) { if (!bd.xcyc) continue; x -= nx; }
        const int d = x + y * nx;
        if (d == k || contains(seen, ns, d)) continue;
        set_at(seen, ns++, d);
        const int rd = rec[d];
        if (rd == d) continue;
        const bool hits = row_hits(mrec, d, k) != 0u;
        const bool gated = hits && (n_is_one ? (h[d] >= htk) : (h[d] > htk));
        if ((gated || rd == k) && dn < 8) insert_by_priority(dep, pr, dn++, tm.g(x, y), prio16(prio[d]));
      }
    }
    RegionLineT<T> L;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      L.c[t] = fact[t];
      L.dep[t] = dep[t];
      L.inp[t] = inp[t];
    }
    line[gk] = L;
    hw[gk] = make_double2(htk, pack_meta(rg, nr > 0));
    cnt0[gk] = (unsigned char)(nin + (nx_in > 0 ? 1 : 0));
    xcnt[gk] = nx_in;
  }
}

// l^n for the nine neighbour lengths of find_receiver / find_mult_rec, with
// the same pow the per-node expression used (so the factors are unchanged)
__global__ void k_length_pow(const double* __restrict__ ltab, double n, double* __restrict__ lpow,
                             float* __restrict__ lpowf) {
  const int e = threadIdx.x;
  if (e < 9) {
    lpow[e] = pow(ltab[e], n);
    lpowf[e] = powf((float)ltab[e], (float)n);
  }
}

// ---- node operations: a warp segment per node -------------------------------------
// A node is computed by a segment of W = 32 / NPW lanes of a warp (NPW nodes
// per warp).  Lane t < 8 of the segment holds slot t of the node's line
// (coefficient, input, dependent), loads input t and forms term t; the
// node's sums then run over the present slots in slot order -- the order of
// the queue engine in fsb_flow.cu -- with every lane of the segment doing the
// same scalar arithmetic on shuffled terms.  The area sums issue all eight
// shuffles and mask absent slots in the adds (an early exit serialised the
// shuffles and measured slower); the one-node Newton loop of the stream power
// law stops at the last present slot (measured faster: it runs once per
// iteration).  All segments of a warp execute
// the same instruction stream: a segment without a node, or whose node needs
// fewer Newton iterations, runs along without effect, so warp-collective
// shuffles and ballots stay convergent.  Lane 0 of a segment stores the
// node's value.  run() returns the dependent in this lane's slot (-1 for
// none).
constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ float ld_l1(const float* p) { return ld_l1f(p); }
__device__ __forceinline__ float ld_l2(const float* p) { return ld_l2f(p); }

// An input's value: this tile's nodes through L1, other tiles' (which arrive
// through the inbox, after an acquire at GPU scope) from L2.  Measured on
// B200: a shared-memory cache of produced values in front of these loads
// was slower (its fences and the L1 capacity it took cost more than the
// round trips it saved).
struct TileLoc {
  int tile, lr;
  template <class V>
  __device__ V load(const V* arr, int q) const {
    return (q >> lr) == tile ? ld_l1(arr + q) : ld_l2(arr + q);
  }
};

// A lane's segment: its lane within the segment and the segment's first lane.
struct Seg {
  int sl, base;
  __device__ double shfl(double v, int s) const { return __shfl_sync(FULL, v, base + s); }
  __device__ float shfl(float v, int s) const { return __shfl_sync(FULL, v, base + s); }
  // bit t: predicate of lane t (< 8) of this segment
  __device__ unsigned slots(bool p) const { return (__ballot_sync(FULL, p) >> base) & 0xffu; }
};

// The slot fields of a node's line for this lane (nothing for an idle segment).
template <class T>
struct Slot {
  T c = 0;
  int d = -1, q = -1;
  bool owner = false;  // lane < 8 of the segment: the slot is this lane's
  __device__ Slot(const RegionLineT<T>* line, int g, const Seg& sg) {
    if (g >= 0) {  // lanes 8.. of a wide segment read the same slots (one line, coalesced)
      const RegionLineT<T>* L = line + g;
      const int t = sg.sl & 7;
      c = __ldg(&L->c[t]);
      d = __ldg(&L->dep[t]);
      q = __ldg(&L->inp[t]);
      owner = sg.sl < 8;
    }
  }
  // the dependent's line (lanes 0-7) and its own entry (lanes 8-15, or the
  // same lanes in 8-lane segments) into L1
  template <class E>
  __device__ void prefetch(const void* lines, const E* entries, const Seg& sg, int w) const {
    if (d < 0) return;
    if (sg.sl < 8) prefetch_l1(reinterpret_cast<const RegionLineT<T>*>(lines) + d);
    if (w > 8 ? (sg.sl >= 8 && sg.sl < 16) : true) prefetch_l1(entries + d);
  }
};

// a(k) = dx*dy*precip(k) + sum over donors of a(d)*w(d->k) (FlowRouting.f90:109-115)
template <class T, int NPW>
struct AccRegionOpT {
  using Value = T;
  static constexpr int kThreads = 512, kNpw = NPW, kId = sizeof(T) == sizeof(double) ? 0 : 3;
  const RegionLineT<T>* line;
  T* val;
  __device__ int run(int g, const Seg& sg, const TileLoc& vc) const {
    const Slot<T> sl(line, g, sg);
    const bool mine = sl.owner && sl.q >= 0;
    T x = 0;
    if (mine) x = vc.load(val, sl.q);
    sl.prefetch(line, val, sg, 32 / NPW);
    const T term = x * sl.c;
    const unsigned present = sg.slots(mine);
    const int npres = __popc(present);  // slots fill from 0: the present ones are 0..npres-1
    T acc = g >= 0 ? ld_l1(val + g) : T(0);  // dx*dy*precip(k), stored by the line builder
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      const T v = sg.shfl(term, s);
      if (s < npres) acc = acc + v;
    }
    if (g >= 0 && sg.sl == 0) {
      if constexpr (sizeof(T) == sizeof(double)) st_global(val + g, acc);
      else st_globalf(val + g, acc);
    }
    return sl.owner ? sl.d : -1;
  }
};
template <int NPW> using AccRegionOpN = AccRegionOpT<double, NPW>;
template <int NPW> using AccRegionOpFN = AccRegionOpT<float, NPW>;

// x^n and x^(n-1) for the Newton update (as NewtonPow in fsb_flow.cu): for
// n = 1.5 as x*sqrt(x) and sqrt(x); otherwise x*x^(n-1) with one pow for x > 0.
struct RegionPow {
  double n;
  int half3;
  __device__ void eval(double x, double& pn, double& pn1) const {
    if (half3) {
      const double r = sqrt(x);
      pn = x * r;
      pn1 = r;
    } else if (x > 0.0) {
      pn1 = pow(x, n - 1.0);
      pn = x * pn1;
    } else {
      pn = pow(x, n);
      pn1 = pow(x, n - 1.0);
    }
  }
};

// implicit stream power law over the multiple receivers with g == 0
// (StreamPowerLaw.f90:92-177): hw[g] = (new h, water).  For n = 1.5 each
// Newton iteration evaluates the receivers' x*sqrt(x) in parallel, one per
// lane; for other n lane 0 of the segment iterates with pow (a shuffle in a
// loop with pow does not compile).
template <bool HALF3, int NPW>
struct SplRegionOpN {
  using Value = double2;
  static constexpr int kThreads = HALF3 ? 512 : 256, kNpw = NPW, kId = HALF3 ? 1 : 2;
  const RegionLine* line;
  double2* hw;
  RegionPow np;
  double omega;
  int n_is_one;
  int* err;
  __device__ int run(int g, const Seg& sg, const TileLoc& vc) const {
    const Slot<double> sl(line, g, sg);
    int rg = -1;
    bool has_mrec = false;
    double ht = 0.0;
    if (g >= 0) {
      const double2 self = ld_l1(hw + g);
      unpack_meta(self.y, rg, has_mrec);
      ht = self.x;
    }
    const bool mine = sl.owner && sl.q >= 0;
    const unsigned present = sg.slots(mine);
    const int npres = __popc(present);
    double hq = 0.0, w = 0.0;
    if (rg >= 0) {
      if (mine) hq = vc.load(hw, sl.q).x;
      if (sg.sl == 0) w = vc.load(hw, rg).y;
    }
    const double wr = sg.shfl(w, 0);
    sl.prefetch(line, hw, sg, 32 / NPW);  // the dependent's line and own entry (ht, rec)
    const double elev = ht;
    const bool solve = rg >= 0 && elev > wr && has_mrec;
    double hk = ht;
    if (n_is_one) {
      const double tf = sl.c * hq;
      double f = elev, df = 1.0;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const double a = sg.shfl(tf, s), b = sg.shfl(sl.c, s);
        if (s < npres) {
          f = f + a;
          df = df + b;
        }
      }
      if (solve) hk = f / df;
    } else if constexpr (HALF3 && NPW == 1) {
      // one node per warp: solve and npres are warp-uniform, so the loop is
      // the reference's and the sums stop at the last present slot
      if (solve) {
        const double tolp = 1.0e-3;
        double errp = 2.0 * tolp;
        int guard = 0;
        while (errp > tolp) {
          if (++guard > kNewtonLimit) {
            if (sg.sl == 0) atomicExch(err, DEV_NEWTON_LIMIT);
            break;
          }
          const double x = fmax(0.0, hk - hq);
          const double r = sqrt(x);
          const double tf = sl.c * (x * r), tdf = sl.c * np.n * r;
          double f = hk - elev, df = 1.0;
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            if (s >= npres) break;
            const double a = sg.shfl(tf, s), b = sg.shfl(tdf, s);
            f = f + a;
            df = df + b;
          }
          const double hn = hk - f / df;
          errp = fabs(hn - hk);
          hk = hk * (1.0 - omega) + hn * omega;
        }
      }
    } else if constexpr (HALF3) {
      const double tolp = 1.0e-3;
      bool go = solve;
      int guard = 0;
      while (__any_sync(FULL, go)) {
        if (go && ++guard > kNewtonLimit) {
          if (sg.sl == 0) atomicExch(err, DEV_NEWTON_LIMIT);
          go = false;
        }
        const double x = fmax(0.0, hk - hq);
        const double r = sqrt(x);
        const double tf = sl.c * (x * r), tdf = sl.c * np.n * r;
        double f = hk - elev, df = 1.0;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          const double a = sg.shfl(tf, s), b = sg.shfl(tdf, s);
          if (s < npres) {
            f = f + a;
            df = df + b;
          }
        }
        if (go) {
          const double hn = hk - f / df;
          const double errp = fabs(hn - hk);
          hk = hk * (1.0 - omega) + hn * omega;
          go = errp > tolp;
        }
      }
    } else {
      double fs[8], qs[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        fs[s] = sg.shfl(sl.c, s);
        qs[s] = sg.shfl(hq, s);
      }
      if (sg.sl == 0 && solve) {
        const double tolp = 1.0e-3;
        double errp = 2.0 * tolp;
        int guard = 0;
        while (errp > tolp) {
          if (++guard > kNewtonLimit) {
            atomicExch(err, DEV_NEWTON_LIMIT);
            break;
          }
          double f = hk - elev, df = 1.0;
#pragma unroll
          for (int s = 0; s < 8; ++s)
            if (s < npres) {
              const double x = fmax(0.0, hk - qs[s]);
              double pn, pn1;
              np.eval(x, pn, pn1);
              f = f + fs[s] * pn;
              df = df + fs[s] * np.n * pn1;
            }
          const double hn = hk - f / df;
          errp = fabs(hn - hk);
          hk = hk * (1.0 - omega) + hn * omega;
        }
      }
      hk = sg.shfl(hk, 0);
    }
    double wk = ht;
    if (rg >= 0) {
      if (elev > wr) {
        if (hk < wr) hk = wr;
      } else {
        hk = elev;
      }
      wk = fmax(wr, hk);
    }
    if (g >= 0 && sg.sl == 0) st_global(hw + g, make_double2(hk, wk));
    return sl.owner ? sl.d : -1;
  }
};

// Mixed precision: the stream-power solve for the increment d = h - ht in FP32.
// Elevations, water levels and the h update stay FP64; the distances to the
// receivers' new elevations, ht(k) - h(q), are taken in FP64 and rounded once.
// n = 1: d = -sum f*(ht - hq) / (1 + sum f), the closed form of
// StreamPowerLaw.f90:108-118 rewritten for the increment; otherwise Newton on
// d (x = max(0, ht - hq + d), :146-162) with the reference's tolerance and
// relaxation.
template <bool HALF3, int NPW>
struct SplRegionOpMN {
  using Value = double2;
  static constexpr int kThreads = HALF3 ? 512 : 256, kNpw = NPW, kId = HALF3 ? 4 : 5;
  const RegionLineF* line;
  double2* hw;
  float n;
  int half3;
  float omega;
  int n_is_one;
  int* err;
  __device__ int run(int g, const Seg& sg, const TileLoc& vc) const {
    const Slot<float> sl(line, g, sg);
    int rg = -1;
    bool has_mrec = false;
    double ht = 0.0;
    if (g >= 0) {
      const double2 self = ld_l1(hw + g);
      unpack_meta(self.y, rg, has_mrec);
      ht = self.x;
    }
    const bool mine = sl.owner && sl.q >= 0;
    const unsigned present = sg.slots(mine);
    const int npres = __popc(present);
    double hq = 0.0, w = 0.0;
    if (rg >= 0) {
      if (mine) hq = vc.load(hw, sl.q).x;
      if (sg.sl == 0) w = vc.load(hw, rg).y;
    }
    const double wr = sg.shfl(w, 0);
    sl.prefetch(line, hw, sg, 32 / NPW);
    const bool solve = rg >= 0 && ht > wr && has_mrec;
    const float dist = mine ? (float)(ht - hq) : 0.0f;
    float d = 0.0f;
    if (n_is_one) {
      const float tf = sl.c * dist;
      float num = 0.0f, den = 1.0f;
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const float a = sg.shfl(tf, s), b = sg.shfl(sl.c, s);
        if (s < npres) {
          num = num + a;
          den = den + b;
        }
      }
      d = -num / den;
    } else if constexpr (HALF3 && NPW == 1) {  // warp-uniform, as in SplRegionOpN
      if (solve) {
        const float tolp = 1.0e-3f;
        float errp = 2.0f * tolp;
        int guard = 0;
        while (errp > tolp) {
          if (++guard > kNewtonLimit) {
            if (sg.sl == 0) atomicExch(err, DEV_NEWTON_LIMIT);
            break;
          }
          const float x = fmaxf(0.0f, dist + d);
          const float r = sqrtf(x);
          const float tf = sl.c * (x * r), tdf = sl.c * n * r;
          float f = d, df = 1.0f;
#pragma unroll
          for (int s = 0; s < 8; ++s) {
            if (s >= npres) break;
            const float a = sg.shfl(tf, s), b = sg.shfl(tdf, s);
            f = f + a;
            df = df + b;
          }
          const float dn = d - f / df;
          errp = fabsf(dn - d);
          d = d * (1.0f - omega) + dn * omega;
        }
      }
    } else if constexpr (HALF3) {
      const float tolp = 1.0e-3f;
      bool go = solve;
      int guard = 0;
      while (__any_sync(FULL, go)) {
        if (go && ++guard > kNewtonLimit) {
          if (sg.sl == 0) atomicExch(err, DEV_NEWTON_LIMIT);
          go = false;
        }
        const float x = fmaxf(0.0f, dist + d);
        const float r = sqrtf(x);
        const float tf = sl.c * (x * r), tdf = sl.c * n * r;
        float f = d, df = 1.0f;
#pragma unroll
        for (int s = 0; s < 8; ++s) {
          const float a = sg.shfl(tf, s), b = sg.shfl(tdf, s);
          if (s < npres) {
            f = f + a;
            df = df + b;
          }
        }
        if (go) {
          const float dn = d - f / df;
          const float errp = fabsf(dn - d);
          d = d * (1.0f - omega) + dn * omega;
          go = errp > tolp;
        }
      }
    } else {
      float fs[8], ds[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        fs[s] = sg.shfl(sl.c, s);
        ds[s] = sg.shfl(dist, s);
      }
      if (sg.sl == 0 && solve) {
        const float tolp = 1.0e-3f;
        float errp = 2.0f * tolp;
        int guard = 0;
        while (errp > tolp) {
          if (++guard > kNewtonLimit) {
            atomicExch(err, DEV_NEWTON_LIMIT);
            break;
          }
          float f = d, df = 1.0f;
#pragma unroll
          for (int s = 0; s < 8; ++s)
            if (s < npres) {
              const float x = fmaxf(0.0f, ds[s] + d);
              float pn, pn1;
              if (x > 0.0f) {
                pn1 = powf(x, n - 1.0f);
                pn = x * pn1;
              } else {
                pn = powf(x, n);
                pn1 = powf(x, n - 1.0f);
              }
              f = f + fs[s] * pn;
              df = df + fs[s] * n * pn1;
            }
          const float dn = d - f / df;
          errp = fabsf(dn - d);
          d = d * (1.0f - omega) + dn * omega;
        }
      }
      d = sg.shfl(d, 0);
    }
    double hk = ht, wk = ht;
    if (rg >= 0) {
      if (ht > wr) {
        if (has_mrec) hk = ht + (double)d;
        if (hk < wr) hk = wr;
      } else {
        hk = ht;
      }
      wk = fmax(wr, hk);
    }
    if (g >= 0 && sg.sl == 0) st_global(hw + g, make_double2(hk, wk));
    return sl.owner ? sl.d : -1;
  }
};

// Nodes per warp: each sweep runs as two kernels, one node per warp (the
// shortest latency per node, best where the critical path dominates) and four
// per warp (8-lane segments, more nodes in flight, best on large grids); the
// tuner below picks one per grid size class.  Single-node ops (n != 1.5 SPL)
// have one form.
constexpr int kNpwWide = 4;

// ---- the sweep kernel ------------------------------------------------------------
// One CTA per tile.  Shared memory: the tile's counters (bytes, four per word)
// and its ready queue (local indices, filled once each, never wrapped).
// Warp 0's lane 0 polls the tile's inbox; every other warp computes up to
// NPW nodes at a time, one per segment: after a node, its lanes release the
// node's dependents (one per lane), the segment continues with the first one
// made ready (they come largest priority first) and queues the others.  A
// segment without a node claims the next queue slot and waits for it to be
// filled.  A CTA ends when all nodes of its tile are done; every wait is
// bounded by a 4 s limit, after which the sweep reports DEV_SPIN_LIMIT.
template <class Op>
__global__ void __launch_bounds__(Op::kThreads, kRegionCtasPerSm)
    k_region_sweep(Op op, TileMap tm, const unsigned char* __restrict__ cnt0, int* xcnt, int* inbox, int icap,
                   unsigned* itail, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lr = tm.lr();
  const int R = 1 << lr;
  unsigned* cnt = reinterpret_cast<unsigned*>(smem);                  // R bytes
  unsigned short* q = reinterpret_cast<unsigned short*>(smem + R);    // R entries
  __shared__ int qhead, qtail, ndone, stop;
  const int tile = blockIdx.x;
  const int gbase = tile << lr;
  const int tx = tile % tm.ntx, ty = tile / tm.ntx;
  const int count = min(1 << tm.ltx, tm.nx - (tx << tm.ltx)) * min(1 << tm.lty, tm.ny - (ty << tm.lty));
  const unsigned long long t0 = global_ns();

  if (threadIdx.x == 0) {
    qhead = 0;
    qtail = 0;
    ndone = 0;
    stop = 0;
  }
  for (int w = threadIdx.x; w < R / 4; w += blockDim.x)
    cnt[w] = reinterpret_cast<const unsigned*>(cnt0 + gbase)[w];
  for (int l = threadIdx.x; l < R; l += blockDim.x) q[l] = kQEmpty;
  __syncthreads();
  const TileLoc vc{tile, lr};
  for (int l = threadIdx.x; l < R; l += blockDim.x)
    if (cnt0[gbase + l] == 0) q[atomicAdd(&qtail, 1)] = (unsigned short)l;
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto push = [&](int l) {
    __threadfence_block();
    const int p = atomicAdd(&qtail, 1);
    if (p < R) *(volatile unsigned short*)&q[p] = (unsigned short)l;
    else atomicExch(err, DEV_OVERFLOW);
  };
  // decrements node l's counter; true when l became ready
  auto release = [&](int l) {
    const unsigned sh = 8u * (unsigned)(l & 3);
    const unsigned old = atomicSub(&cnt[l >> 2], 1u << sh);
    return ((old >> sh) & 0xffu) == 1u;
  };
  // periodic checks of the time limit and of failures elsewhere (one lane)
  auto should_stop = [&](int& ticks) {
    if (*(volatile int*)&stop) return true;
    if (++ticks < 256) return false;
    ticks = 0;
    if (*(volatile int*)err != 0) {
      *(volatile int*)&stop = 1;
      return true;
    }
    if (global_ns() - t0 > kRegionTimeLimitNs) {
      atomicExch(err, DEV_SPIN_LIMIT);
      *(volatile int*)&stop = 1;
      return true;
    }
    return false;
  };

  if (warp == 0) {
    if (lane != 0) return;
    int ih = 0, ticks = 0;
    int* box = inbox + (size_t)tile * icap;
    for (;;) {
      if (ih < icap) {
        const int d = ld_relaxed_gpu(&box[ih]);
        if (d >= 0) {
          ++ih;
          __threadfence();  // acquire: the cross-tile producers' values
          if (release(d - gbase)) push(d - gbase);
          continue;
        }
      }
      if (*(volatile int*)&ndone >= count) return;
      if (should_stop(ticks)) return;
      __nanosleep(64);
    }
  }
  constexpr int W = 32 / Op::kNpw;  // lanes per node
  const Seg sg{lane % W, lane - lane % W};
  const unsigned segmask = (W == 32 ? 0xffffffffu : ((1u << W) - 1u)) << sg.base;
  int cur = -1, slot = -1, ticks = 0, back = 32;
  for (;;) {
    // segments without a node try their queue slot (the segment's lane 0);
    // a one-segment warp that continues with a dependent skips the poll
    if (W < 32 || cur < 0) {
      int got = -1;
      if (cur < 0 && sg.sl == 0) {
        if (slot < 0) slot = atomicAdd(&qhead, 1);
        if (slot < R) {
          const unsigned short v = *(volatile unsigned short*)&q[slot];
          if (v != kQEmpty) {
            got = v;
            slot = -1;
          }
        }
      }
      got = __shfl_sync(FULL, got, sg.base);
      if (cur < 0) cur = got;
      if (!__any_sync(FULL, cur >= 0)) {
        int quit = 0;
        if (lane == 0) quit = *(volatile int*)&ndone >= count || should_stop(ticks);
        if (__shfl_sync(FULL, quit, 0)) return;
        // idle warps back off (32 ns doubling to 512 ns): polling warps take
        // issue slots from the busy ones (stream-power sweep at 2049^2:
        // 15.9 -> 15.3 ms against a constant 32 ns)
        __nanosleep(back);
        if (back < 512) back <<= 1;
        continue;
      }
      back = 32;
      __threadfence_block();  // acquire: the producers' values
    }
    const int d = op.run(cur >= 0 ? gbase + cur : -1, sg, vc);
    __syncwarp();
    __threadfence_block();  // release: the node's value before its dependents' counters
    bool ready = false;
    if (d >= 0) {
      if ((d >> lr) == tile) {
        ready = release(d - gbase);
      } else {
        __threadfence();  // release at GPU scope before a cross-tile counter
        if (atomicSub(&xcnt[d], 1) == 1) {
          __threadfence();
          const int owner = d >> lr;
          const unsigned p = atomicAdd(&itail[owner], 1u);
          if (p < (unsigned)icap) st_relaxed_gpu_int(&inbox[(size_t)owner * icap + p], d);
          else atomicExch(err, DEV_OVERFLOW);
        }
      }
    }
    const unsigned rm = __ballot_sync(FULL, ready) & segmask;
    const int first = rm ? __ffs(rm) - 1 : lane;
    const int nxt_l = __shfl_sync(FULL, d - gbase, first);
    if (ready && lane != first) push(d - gbase);
    if (rm) __threadfence_block();  // acquire for the continuation
    if (sg.sl == 0 && cur >= 0) atomicAdd(&ndone, 1);
    cur = rm ? nxt_l : -1;
  }
}

// natural-order copies of the sweeps' results
template <class T>
__global__ void k_untile_area(int nx, int ny, TileMap tm, const T* __restrict__ val, double* __restrict__ a) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    a[k] = (double)val[tm.g(k % nx, k / nx)];
}

// StreamPowerLaw.f90:380-393 with g == 0: b=min(h,b), etot=etot+ht-h,
// erate=(ht-h)/dt, Sedflux=ht-h, from the tile-major (h, water) pairs
__global__ void k_spl_finish_t(int nx, int ny, TileMap tm, double dt, const double2* __restrict__ hw,
                               double* __restrict__ h, double* __restrict__ b, double* __restrict__ etot,
                               double* __restrict__ erate, double* __restrict__ sedflux) {
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double ht = h[k], hn = hw[tm.g(k % nx, k / nx)].x;
    b[k] = fmin(hn, b[k]);
    etot[k] = etot[k] + ht - hn;
    erate[k] = (ht - hn) / dt;
    sedflux[k] = ht - hn;
    h[k] = hn;
  }
}


template <class Op>
size_t region_smem(const TileMap& tm) {
  return (size_t)3 << tm.lr();
}

// whether every tile's CTA of this sweep kernel can be co-resident
template <class Op>
bool region_fits(const TileMap& tm) {
  const size_t smem = region_smem<Op>(tm);
  auto kern = k_region_sweep<Op>;
  // the permitted maximum covers every plan (3 bytes per node, 32768 nodes per
  // tile), so instances with different plans never undo each other's setting
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * 32768) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Op::kThreads, smem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return per_sm * sms >= tm.tiles();
}

// whether the sweep of op Op can run on one of the instance's tile plans
// (checked once per instance and op)
template <class Op>
bool region_usable(Ctx& c) {
  if (!c.region_enabled || c.ntplans == 0) return false;
  signed char& st = c.region_ok[Op::kId];
  if (st == 0) {
    st = -1;
    for (int i = 0; i < c.ntplans; ++i)
      if (region_fits<Op>(c.tplans[i])) st = 1;
  }
  return st > 0;
}

template <class Op>
bool launch_region(Ctx& c, Op op, const TileMap& tm) {
  const int tiles = tm.tiles();
  const size_t smem = region_smem<Op>(tm);
  auto kern = k_region_sweep<Op>;
  cudaMemsetAsync(c.rl_inbox, 0xff, sizeof(int) * (size_t)tiles * c.rl_icap, c.stream);
  cudaMemsetAsync(c.rl_itail, 0, sizeof(unsigned) * (size_t)tiles, c.stream);
  const unsigned char* cnt0 = c.rl_cnt0;
  int* xcnt = c.rl_xcnt;
  int* inbox = c.rl_inbox;
  int icap = c.rl_icap;
  unsigned* itail = c.rl_itail;
  int* err = c.d_err;
  TileMap tmv = tm;
  void* args[] = {&op, &tmv, &cnt0, &xcnt, &inbox, &icap, &itail, &err};
  const int timer = Op::kId == 0 || Op::kId == 3 ? KT_AREA_SWEEP : KT_SPL_SWEEP;
  stage_begin(c, timer);
  const cudaError_t e =
      cudaLaunchCooperativeKernel((const void*)kern, dim3(tiles), dim3(Op::kThreads), args, smem, c.stream);
  stage_end(c, timer);
  c.count_launch();
  if (e != cudaSuccess) {  // e.g. the GPU is shared and the tiles no longer fit
    cudaGetLastError();
    return false;
  }
  return true;
}

// ---- the tile-plan tuner ------------------------------------------------------
// The tile shape decides how a sweep's work is split between co-resident CTAs
// and how often its critical path crosses a tile boundary, and the nodes per
// warp trade latency per node for nodes in flight; which pair is fastest
// depends on the grid.  The first sweep of an op on an instance whose grid
// size class has not been seen by the process runs twice on each candidate
// (every candidate plan -- the smallest tiles that fit the co-resident CTAs
// and up to two coarser ones -- with each form of the kernel), timed with
// CUDA events, and keeps the fastest, also for every later instance of that
// size class.  Every run is a complete, correct sweep: a node's arithmetic
// depends neither on the plan nor on the form, so each run gives the same
// values and the last one's output is used.  A cached choice applies to a
// later grid of the same size class when its candidate list holds that tile
// shape.
std::mutex g_tune_mu;
// (size class, aspect class, op) -> (ltx, lty, form); a size class spans a
// factor sqrt(2) in nodes, so a stream of requests of many sizes (the served
// form) tunes once per class, not once per size
std::map<std::tuple<int, int, int>, std::tuple<int, int, int>> g_tuned;
std::tuple<int, int, int> tune_key(const Ctx& c, int op) {
  const int size_class = (int)std::floor(2.0 * std::log2((double)c.nx * (double)c.ny));
  const int aspect_class = (int)std::lround(std::log2((double)c.nx / (double)c.ny));
  return std::make_tuple(size_class * 64 + aspect_class, 0, op);
}

// Runs run(plan, form) on op id's tuned plan and form (0 <= form < nforms),
// tuning first where needed; fits(plan, form) says whether the form's CTAs
// are co-resident on the plan.  Returns the plan of the last complete run, or
// nullptr when no plan could run.
template <class Fits, class Run>
const TileMap* run_tuned(Ctx& c, int id, int nforms, Fits fits, Run run) {
  TileMap& chosen = c.tplan_of[id];
  int& form = c.tform_of[id];
  if (chosen.ntx == 0) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(tune_key(c, id));
    if (it != g_tuned.end() && std::get<2>(it->second) < nforms)
      for (int i = 0; i < c.ntplans; ++i)
        if (c.tplans[i].ltx == std::get<0>(it->second) && c.tplans[i].lty == std::get<1>(it->second)) {
          chosen = c.tplans[i];
          form = std::get<2>(it->second);
        }
  }
  if (chosen.ntx != 0) {
    if (fits(chosen, form) && run(chosen, form)) return &chosen;
    c.region_ok[id] = -1;  // the queue engine runs from now on
    return nullptr;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const TileMap* last = nullptr;
  float best_ms = 0.f;
  int best = -1, best_form = 0;
  for (int i = 0; i < c.ntplans; ++i)
    for (int f = 0; f < nforms; ++f) {
      if (!fits(c.tplans[i], f)) continue;
      float cand_ms = -1.f;  // the better of two runs of each candidate
      for (int rep = 0; rep < 2; ++rep) {
        cudaEventRecord(e0, c.stream);
        const bool ok = run(c.tplans[i], f);
        cudaEventRecord(e1, c.stream);
        float ms = 0.f;
        if (!ok || cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
          cudaGetLastError();
          cand_ms = -1.f;
          break;
        }
        last = &c.tplans[i];
        if (cand_ms < 0.f || ms < cand_ms) cand_ms = ms;
      }
      if (cand_ms >= 0.f && (best < 0 || cand_ms < best_ms)) {
        best = i;
        best_form = f;
        best_ms = cand_ms;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (best < 0) c.region_ok[id] = -1;  // no plan ran: the queue engine from now on
  if (best >= 0) {
    chosen = c.tplans[best];
    form = best_form;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[tune_key(c, id)] = std::make_tuple(chosen.ltx, chosen.lty, form);
  }
  return last;
}

// area sweep of value type T on plan p with NPW nodes per warp
template <class T, int NPW>
bool acc_run(Ctx& c, const TileMap& p) {
  using Op = AccRegionOpT<T, NPW>;
  RegionLineT<T>* line = static_cast<RegionLineT<T>*>(c.rl_line);
  T* val = reinterpret_cast<T*>(c.rl_val);
  cudaMemsetAsync(c.rl_cnt0, 0xff, (size_t)p.padded(), c.stream);  // padding slots never run
  k_acc_lines_t<T><<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, p, c.dx * c.dy, c.mrec, c.mnrec, c.mwrec, c.precip,
                                                          c.size, line, val, c.rl_cnt0, c.rl_xcnt, c.d_err);
  c.count_launch();
  return launch_region<Op>(c, Op{line, val}, p);
}

template <class T>
bool region_accumulate_t(Ctx& c) {
  using Op1 = AccRegionOpT<T, 1>;
  using OpW = AccRegionOpT<T, kNpwWide>;
  if (!region_usable<Op1>(c)) return false;
  const TileMap* tm = run_tuned(
      c, Op1::kId, 2, [&](const TileMap& p, int f) { return f ? region_fits<OpW>(p) : region_fits<Op1>(p); },
      [&](const TileMap& p, int f) { return f ? acc_run<T, kNpwWide>(c, p) : acc_run<T, 1>(c, p); });
  if (!tm) return false;
  k_untile_area<T><<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, *tm, reinterpret_cast<T*>(c.rl_val), c.a);
  c.count_launch();
  return true;
}

// stream-power sweep: op1 (one node per warp) and opw (its wide form, the
// same type where the op has one form only: nforms = 1)
template <class Op1, class OpW, class T>
const TileMap* spl_sweep(Ctx& c, const Op1& op1, const OpW& opw, int nforms, RegionLineT<T>* line,
                         const T* lpow) {
  const int n1 = fabs(c.n - 1.0) < DBL_MIN;
  double2* hw = reinterpret_cast<double2*>(c.rl_val);
  return run_tuned(
      c, Op1::kId, nforms, [&](const TileMap& p, int f) { return f ? region_fits<OpW>(p) : region_fits<Op1>(p); },
      [&](const TileMap& p, int f) {
        cudaMemsetAsync(c.rl_cnt0, 0xff, (size_t)p.padded(), c.stream);
        k_spl_lines_t<T><<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, p, n1, c.kfsed, c.dt, c.m, c.n, c.rec, c.mrec,
                                                                c.mnrec, c.mwrec, c.mlrec, c.h, c.b, c.kf, c.a,
                                                                c.size, c.ltab, lpow, line, hw, c.rl_cnt0,
                                                                c.rl_xcnt, c.d_err);
        c.count_launch();
        return f ? launch_region<OpW>(c, opw, p) : launch_region<Op1>(c, op1, p);
      });
}

}  // namespace

// Tile plans: tiles of 2^a x 2^b nodes (32 x 32 at least, 32768 nodes at
// most, width >= height) whose count fits the co-resident CTAs
// (kRegionCtasPerSm per SM) -- the smallest such tiles and up to two coarser
// ones, for the tuner.  None fits -> the queue engine runs.
int plan_tiles(int nx, int ny, int sms, TileMap* out, int max_plans) {
  const int max_ctas = kRegionCtasPerSm * std::max(1, sms);
  static const int cand[][2] = {{5, 5}, {6, 5}, {6, 6}, {7, 6}, {7, 7}, {8, 7}};
  int n = 0;
  for (const auto& cd : cand) {
    const int ntx = (nx + (1 << cd[0]) - 1) >> cd[0], nty = (ny + (1 << cd[1]) - 1) >> cd[1];
    if (ntx * nty <= max_ctas && n < max_plans) {
      TileMap& tm = out[n++];
      tm.nx = nx;
      tm.ny = ny;
      tm.ltx = cd[0];
      tm.lty = cd[1];
      tm.ntx = ntx;
      tm.nty = nty;
    }
  }
  return n;
}

bool region_accumulate(Ctx& c) {
  return c.mixed ? region_accumulate_t<float>(c) : region_accumulate_t<double>(c);
}

bool region_stream_power(Ctx& c) {
  const bool h3 = c.n == 1.5;
  const bool ok = c.mixed ? (h3 ? region_usable<SplRegionOpMN<true, 1>>(c) : region_usable<SplRegionOpMN<false, 1>>(c))
                          : (h3 ? region_usable<SplRegionOpN<true, 1>>(c) : region_usable<SplRegionOpN<false, 1>>(c));
  if (!ok) return false;
  const int n1 = fabs(c.n - 1.0) < DBL_MIN;
  double2* hw = reinterpret_cast<double2*>(c.rl_val);
  double* lpow = c.ltab + 16;
  float* lpowf = reinterpret_cast<float*>(c.ltab + 32);
  k_length_pow<<<1, 32, 0, c.stream>>>(c.ltab, c.n, lpow, lpowf);
  c.count_launch();
  const TileMap* tm;
  const double omega = 0.875 / c.n;
  if (c.mixed) {
    RegionLineF* line = static_cast<RegionLineF*>(c.rl_line);
    const float nf = (float)c.n, of = (float)omega;
    if (h3)
      tm = spl_sweep(c, SplRegionOpMN<true, 1>{line, hw, nf, 1, of, n1, c.d_err},
                     SplRegionOpMN<true, kNpwWide>{line, hw, nf, 1, of, n1, c.d_err}, 2, line, lpowf);
    else
      tm = spl_sweep(c, SplRegionOpMN<false, 1>{line, hw, nf, 0, of, n1, c.d_err},
                     SplRegionOpMN<false, 1>{line, hw, nf, 0, of, n1, c.d_err}, 1, line, lpowf);
  } else {
    RegionLine* line = static_cast<RegionLine*>(c.rl_line);
    if (h3)
      tm = spl_sweep(c, SplRegionOpN<true, 1>{line, hw, RegionPow{c.n, 1}, omega, n1, c.d_err},
                     SplRegionOpN<true, kNpwWide>{line, hw, RegionPow{c.n, 1}, omega, n1, c.d_err}, 2, line, lpow);
    else
      tm = spl_sweep(c, SplRegionOpN<false, 1>{line, hw, RegionPow{c.n, 0}, omega, n1, c.d_err},
                     SplRegionOpN<false, 1>{line, hw, RegionPow{c.n, 0}, omega, n1, c.d_err}, 1, line, lpow);
  }
  if (!tm) return false;
  k_spl_finish_t<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, *tm, c.dt, hw, c.h, c.b, c.etot, c.erate,
                                                        c.sedflux);
  c.count_launch();
  return true;
}

}  // namespace fsb
