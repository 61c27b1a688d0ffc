// Depression routing (Cordonnier et al. 2019 as implemented in the reference's
// src/LocalMinima.f90:1-132, continuous_flow_v2 branch).
//
//   compute_basins        LocalMinima.f90:136-169  -> k_basins (scan over the stack)
//   connect_basins        LocalMinima.f90:173-329  -> k_conn_pass / k_conn_compact / sort
//   loc_min_3_indexx      LocalMinima.f90:947-1046 -> exact segmented emulation (nr_*)
//   mst_kruskal+UnionFind LocalMinima.f90:333-385,766-832 -> Boruvka on the sort ranks
//   order_tree            LocalMinima.f90:389-533  -> Euler tour of the tree + ranking
//   correct_receivers_v2  LocalMinima.f90:601-662  -> k_correct (one thread per edge)
//
// Exactness argument.  Kruskal accepts edges in the order of the NR index
// sort; the accepted set is the unique minimum spanning tree under the total
// order "position in that sorted permutation", which Boruvka computes in
// parallel.  The sorted permutation itself is reproduced exactly: quicksort
// segments are independent once created, and one Hoare partition of a
// segment is determined by the positions of the left-scan stoppers
// (arr >= pivot) and right-scan stoppers (arr <= pivot) of the segment, which
// prefix sums give in parallel (see k_nr_cross for the crossing rule).  The
// conn list is built in the reference's discovery order: edge (b,nb) sits at
// the first (stack position, neighbour slot) where it is met and keeps the
// earliest minimum-weight pass.  Receiver corrections touch disjoint child
// basins, so they run in parallel in any order.
#include <cfloat>
#include <climits>

#include <cooperative_groups.h>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

enum {
  C_NBASINS = 0, C_NLOCMIN = 1, C_BASIN0 = 2, C_NEDGE = 3, C_NSEG = 4, C_NSMALL = 5,
  C_CHANGED = 6, C_NTREE = 7, C_NLOCMIN_AFTER = 8, C_OVERFLOW = 9, C_NSEG2 = 11,
  C_NRIDX = 12, C_NRLEVELS = 13, C_NMED = 14,
  C_MST_CHANGED = 24, C_MST_FLAT = 25,  // 25..27: the cooperative MST's rotating flags
  C_MST_DONE = 28                        // host-driven MST: a round changed nothing
};
constexpr int kNrCounters = 15;  // counters the NR sort reads back

// Segments of 8..kNrMedium elements leave the level-synchronous partition and
// are finished each by one warp in shared memory (k_nr_medium): the last
// levels of the sort, which hold only such segments, would otherwise each
// cost a round of grid-wide barriers.
constexpr int kNrMedium = 512;

// Level bound of the emulation: every level shrinks every segment by at least
// its pivot, so n + 8 levels always suffice.  A fixed bound would not do: the
// reference's median of three (LocalMinima.f90:985-1006) degenerates on
// descending keys, to a quicksort tree about n/6 levels deep, which the
// reference runs sequentially (slowly) and this emulation level by level.
inline int nr_max_levels(int n) { return n + 8; }

__constant__ int c_ii[8] = {-1, 1, 0, 0, -1, 1, -1, 1};
__constant__ int c_jj[8] = {0, 0, -1, 1, -1, -1, 1, 1};

__device__ inline unsigned long long ordered_u64(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

__device__ inline unsigned long long mix64(unsigned long long x) {
  x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
  return x;
}

// ---- basins --------------------------------------------------------------
__global__ void k_pos_root_flags(int nn, const int* __restrict__ stack, const int* __restrict__ rec,
                                 int* __restrict__ flag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
    const int k = stack[p];
    flag[p] = rec[k] == k ? 1 : 0;
  }
}

__global__ void k_basins(int nn, const int* __restrict__ stack, const int* __restrict__ incl,
                         int* __restrict__ basins) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x)
    basins[stack[p]] = incl[p];
}

// active roots (local minima) and basin0 = first basin whose root is on a fixed boundary
// the root count comes from cnt[C_NBASINS] (set on the device), so that one
// read-back brings the basins, the pits and basin0 together
__global__ void k_roots_scan(Bounds bd, const int* __restrict__ roots, int* cnt) {
  const int nroots = cnt[C_NBASINS];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nroots; r += gridDim.x * blockDim.x) {
    const int k = roots[r];
    if (is_bc_node(bd, k % bd.nx, k / bd.nx)) atomicMin(&cnt[C_BASIN0], r + 1);
    else atomicAdd(&cnt[C_NLOCMIN], 1);
  }
}

// ---- connect_basins ------------------------------------------------------
__device__ inline unsigned ht_insert(unsigned long long* keys, size_t cap, unsigned long long key) {
  size_t s = mix64(key) & (cap - 1);
  const size_t limit = cap < 4096 ? cap : 4096;  // load stays below 1/2: long probes mean overflow
  for (size_t probe = 0; probe < limit; ++probe) {
    const unsigned long long old = atomicCAS(&keys[s], ~0ull, key);
    if (old == ~0ull || old == key) return (unsigned)s;
    s = (s + 1) & (cap - 1);
  }
  return 0xffffffffu;
}

__device__ inline unsigned ht_find(const unsigned long long* keys, size_t cap, unsigned long long key) {
  size_t s = mix64(key) & (cap - 1);
  const size_t limit = cap < 4096 ? cap : 4096;
  for (size_t probe = 0; probe < limit; ++probe) {
    const unsigned long long k = keys[s];
    if (k == key) return (unsigned)s;
    if (k == ~0ull) return 0xffffffffu;
    s = (s + 1) & (cap - 1);
  }
  return 0xffffffffu;
}

// pass 0: insert pairs, min weight, first discovery; pass 1: earliest
// discovery among the minimum-weight candidates of each pair.
template <int PASS>
__global__ void k_conn_pass(Bounds bd, const int* __restrict__ basins, const int* __restrict__ roots,
                            const int* __restrict__ pos, const double* __restrict__ h,
                            unsigned long long* __restrict__ ht_key, unsigned long long* __restrict__ ht_wmin,
                            unsigned* __restrict__ ht_first, unsigned* __restrict__ ht_best, size_t cap,
                            int* __restrict__ cnt) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
    const int b = basins[p];
    const int outlet = roots[b - 1];
    if (is_bc_node(bd, outlet % nx, outlet / nx)) continue;  // inactive basin: not scanned
    const int i = p % nx, j = p / nx;
    const double hp = h[p];
    const unsigned disc0 = (unsigned)pos[p] * 8u;
    for (int k = 0; k < 8; ++k) {
      const int ki = i + c_ii[k], kj = j + c_jj[k];
      if (ki < 0 || ki >= nx || kj < 0 || kj >= ny) continue;
      const int q = ki + kj * nx;
      const int nb = basins[q];
      const int nbo = roots[nb - 1];
      if (b >= nb && !is_bc_node(bd, nbo % nx, nbo / nx)) continue;
      const double w = fmax(hp, h[q]);
      const unsigned long long key = ((unsigned long long)b << 32) | (unsigned)nb;
      const unsigned disc = disc0 + (unsigned)k;
      if (PASS == 0) {
        const unsigned s = ht_insert(ht_key, cap, key);
        if (s == 0xffffffffu) { atomicExch(&cnt[C_OVERFLOW], 1); continue; }
        atomicMin(&ht_wmin[s], ordered_u64(w));
        atomicMin(&ht_first[s], disc);
      } else {
        const unsigned s = ht_find(ht_key, cap, key);
        if (s == 0xffffffffu) continue;
        if (ordered_u64(w) == ht_wmin[s]) atomicMin(&ht_best[s], disc);
      }
    }
  }
}

__global__ void k_conn_compact(Bounds bd, size_t cap, const unsigned long long* __restrict__ ht_key,
                               const unsigned* __restrict__ ht_first, const unsigned* __restrict__ ht_best,
                               const int* __restrict__ stack, const double* __restrict__ h, size_t conn_cap,
                               unsigned* __restrict__ r_key, int* __restrict__ r_b1, int* __restrict__ r_b2,
                               int* __restrict__ r_n1, int* __restrict__ r_n2, double* __restrict__ r_w,
                               int* __restrict__ cnt) {
  const int nx = bd.nx;
  for (size_t s = blockIdx.x * (size_t)blockDim.x + threadIdx.x; s < cap; s += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long key = ht_key[s];
    if (key == ~0ull) continue;
    const int idx = atomicAdd(&cnt[C_NEDGE], 1);
    if ((size_t)idx >= conn_cap) { atomicExch(&cnt[C_OVERFLOW], 1); continue; }
    const unsigned best = ht_best[s];
    if (best == 0xffffffffu) { atomicExch(&cnt[C_OVERFLOW], 1); continue; }
    const int p = stack[best >> 3];
    const int k = best & 7;
    const int q = (p % nx + c_ii[k]) + (p / nx + c_jj[k]) * nx;
    r_key[idx] = ht_first[s];
    r_b1[idx] = (int)(key >> 32);
    r_b2[idx] = (int)(key & 0xffffffffu);
    r_n1[idx] = p;
    r_n2[idx] = q;
    r_w[idx] = fmax(h[p], h[q]);
  }
}

// virtual edges basin0 <-> every other open basin, keyed at the open root's stack position
__global__ void k_conn_virtual(Bounds bd, int nroots, const int* __restrict__ roots, const int* __restrict__ pos,
                               size_t conn_cap, unsigned* __restrict__ r_key, int* __restrict__ r_b1,
                               int* __restrict__ r_b2, int* __restrict__ r_n1, int* __restrict__ r_n2,
                               double* __restrict__ r_w, int* __restrict__ cnt) {
  const int basin0 = cnt[C_BASIN0];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nroots; r += gridDim.x * blockDim.x) {
    const int k = roots[r];
    if (!is_bc_node(bd, k % bd.nx, k / bd.nx) || r + 1 == basin0) continue;
    const int idx = atomicAdd(&cnt[C_NEDGE], 1);
    if ((size_t)idx >= conn_cap) { atomicExch(&cnt[C_OVERFLOW], 1); continue; }
    r_key[idx] = (unsigned)pos[k] * 8u;
    r_b1[idx] = basin0;
    r_b2[idx] = r + 1;
    r_n1[idx] = -1;
    r_n2[idx] = -1;
    r_w[idx] = -1.0e10;
  }
}

__global__ void k_iota(int n, int* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

__global__ void k_conn_gather(int n, const int* __restrict__ perm, const int* __restrict__ r_b1,
                              const int* __restrict__ r_b2, const int* __restrict__ r_n1,
                              const int* __restrict__ r_n2, const double* __restrict__ r_w,
                              int* __restrict__ b1, int* __restrict__ b2, int* __restrict__ n1,
                              int* __restrict__ n2, double* __restrict__ w) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int e = perm[t];
    b1[t] = r_b1[e]; b2[t] = r_b2[e]; n1[t] = r_n1[e]; n2[t] = r_n2[e]; w[t] = r_w[e];
  }
}

// ---- loc_min_3_indexx emulation (1-based positions l..ir) -----------------
// idx[1..n] holds 1-based edge ids, arr[1..n] the weights (arr = w - 1).
__global__ void k_nr_init(int n, int* __restrict__ idx, int* __restrict__ segof, int* __restrict__ seg,
                          int* __restrict__ small, int* __restrict__ med, int* __restrict__ cnt) {
  const bool level = n > kNrMedium;  // else the whole array is one medium or small segment
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n + 1; q += gridDim.x * blockDim.x) {
    if (q >= 1 && q <= n) idx[q] = q;
    segof[q] = (q >= 1 && q <= n && level) ? 0 : -1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cnt[C_NSEG] = 0;
    cnt[C_NMED] = 0;
    if (level) { seg[0] = 1; seg[1] = n; cnt[C_NSEG] = 1; }
    else if (n - 1 >= 7) { med[0] = 1; med[1] = n; cnt[C_NMED] = 1; }
    else if (n >= 2) { small[0] = 1; small[1] = n; cnt[C_NSMALL] = 1; }
  }
}

__device__ inline void iswap(int* v, int a, int b) { const int t = v[a]; v[a] = v[b]; v[b] = t; }

// ---- one NR level, per segment s / per position q (shared by the level
// kernels below and the cooperative kernel k_nr_levels) ----------------------
// No pointer here is __restrict__ but the weights: in k_nr_levels the same
// arrays are written in one phase and read in the next, so their loads must
// not take the non-coherent read-only path.

// median of three (LocalMinima.f90:985-1006)
__device__ inline void nr_median_one(int s, const int* seg, const double* __restrict__ arr,
                                     int* idx, double* piv, int* meta) {
  const int l = seg[2 * s], ir = seg[2 * s + 1];
  const int k = (l + ir) / 2;
  iswap(idx, k, l + 1);
  if (arr[idx[l + 1]] > arr[idx[ir]]) iswap(idx, l + 1, ir);
  if (arr[idx[l]] > arr[idx[ir]]) iswap(idx, l, ir);
  if (arr[idx[l + 1]] > arr[idx[l]]) iswap(idx, l + 1, l);
  piv[s] = arr[idx[l]];
  meta[4 * s] = idx[l];
}

// stopper flags of position q: the left scan stops where arr >= a (positions
// l+2..ir), the right scan where arr <= a (positions l+1..ir-1)
__device__ inline void nr_flags_one(int q, const int* segof, const int* seg,
                                    const double* piv, const double* __restrict__ arr,
                                    const int* idx, int& a, int& b) {
  a = 0;
  b = 0;
  const int s = segof[q];
  if (s >= 0) {
    const int l = seg[2 * s], ir = seg[2 * s + 1];
    const double pv = piv[s];
    const double v = arr[idx[q]];
    a = (q >= l + 2 && q <= ir && v >= pv) ? 1 : 0;
    b = (q >= l + 1 && q <= ir - 1 && v <= pv) ? 1 : 0;
  }
}

// Crossing of the Hoare scans.  With L_t the t-th left stopper (ascending)
// and R_t the t-th right stopper (descending) of the unmodified segment, the
// partition swaps (L_t, R_t) for every t < T, T = min{t : L_t >= R_t}.  If
// L_T == R_T = P the scans stop at i=P+1, j=P-1; otherwise at
// i = min(L_T, R_{T-1}), j = max(R_T, L_{T-1}) (R_0 = +inf, L_0 = -inf).
__device__ inline void nr_cross_one(int s, const int* seg, const int* ls,
                                    const int* rs, const int* lpos,
                                    const int* rpos, int* meta) {
  const int l = seg[2 * s], ir = seg[2 * s + 1];
  const int lb = ls[l + 2], nL = ls[ir + 1] - ls[l + 2];
  const int rtop = rs[ir], nR = rs[ir] - rs[l + 1];
  auto L = [&](int t) { return lpos[lb + t - 1]; };
  auto R = [&](int t) { return rpos[rtop - t]; };
  int lo = 1, hi = min(nL, nR);
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (L(mid) >= R(mid)) hi = mid; else lo = mid + 1;
  }
  const int T = lo;
  int i, j;
  if (L(T) == R(T)) {
    i = L(T) + 1;
    j = L(T) - 1;
  } else {
    i = (T == 1) ? L(1) : min(L(T), R(T - 1));
    j = (T == 1) ? R(1) : max(R(T), L(T - 1));
  }
  meta[4 * s + 1] = i;
  meta[4 * s + 2] = j;
  meta[4 * s + 3] = T;
}

__device__ inline int nr_newval(int x, int l, int ir, int T, const int* idx, const int* lf,
                                const int* rf, const int* ls, const int* rs, const int* lpos,
                                const int* rpos) {
  if (lf[x]) {
    const int t = ls[x] - ls[l + 2] + 1;
    if (t < T) return idx[rpos[rs[ir] - t]];
  }
  if (rf[x]) {
    const int t = rs[ir] - rs[x];
    if (t < T) return idx[lpos[ls[l + 2] + t - 1]];
  }
  return idx[x];
}

// the partitioned permutation at position q (1..n)
__device__ inline int nr_apply_one(int q, const int* segof, const int* seg,
                                   const int* meta, const int* idx,
                                   const int* lf, const int* rf, const int* ls,
                                   const int* rs, const int* lpos,
                                   const int* rpos) {
  const int s = segof[q];
  if (s < 0) return idx[q];
  const int l = seg[2 * s], ir = seg[2 * s + 1];
  const int pv = meta[4 * s], j = meta[4 * s + 2], T = meta[4 * s + 3];
  if (q == l) return nr_newval(j, l, ir, T, idx, lf, rf, ls, rs, lpos, rpos);
  if (q == j) return pv;
  return nr_newval(q, l, ir, T, idx, lf, rf, ls, rs, lpos, rpos);
}

// children segments [l, j-1] and [i, ir]: partitioned at the next level when
// they hold more than kNrMedium elements (counted in cnt[out_slot]), finished
// in shared memory when they hold 8..kNrMedium (cnt[C_NMED]), insertion-sorted
// when fewer (M = 7)
// The children's ids go to child[4s..4s+3] (i, left id, right id, j); child
// may be meta itself (i and j are read before anything is written).
__device__ inline void nr_newsegs_one(int s, int out_slot, const int* seg, const int* meta, int* child,
                                      int* seg2, int* small, int* med, int* cnt,
                                      int small_cap, int med_cap) {
  const int l = seg[2 * s], ir = seg[2 * s + 1];
  const int i = meta[4 * s + 1], j = meta[4 * s + 2];
  int ids[2] = {-1, -1};
  const int lo[2] = {l, i}, hi[2] = {j - 1, ir};
  for (int c = 0; c < 2; ++c) {
    if (hi[c] - lo[c] >= 7 && hi[c] - lo[c] < kNrMedium) {
      const int id = atomicAdd(&cnt[C_NMED], 1);
      if (id < med_cap) { med[2 * id] = lo[c]; med[2 * id + 1] = hi[c]; }
      else atomicExch(&cnt[C_OVERFLOW], 1);
    } else if (hi[c] - lo[c] >= 7) {
      const int id = atomicAdd(&cnt[out_slot], 1);
      seg2[2 * id] = lo[c];
      seg2[2 * id + 1] = hi[c];
      ids[c] = id;
    } else if (hi[c] - lo[c] >= 1) {
      const int id = atomicAdd(&cnt[C_NSMALL], 1);
      if (id < small_cap) { small[2 * id] = lo[c]; small[2 * id + 1] = hi[c]; }
      else atomicExch(&cnt[C_OVERFLOW], 1);
    }
  }
  child[4 * s + 1] = ids[0];
  child[4 * s + 2] = ids[1];
  child[4 * s + 3] = j;  // boundary of the left child
  child[4 * s] = i;      // start of the right child
}

__device__ inline void nr_segof_one(int q, const int* seg, const int* child,
                                    int* segof) {
  const int s = segof[q];
  if (s < 0) return;
  const int l = seg[2 * s], ir = seg[2 * s + 1];
  const int i = child[4 * s], j = child[4 * s + 3];
  int ns = -1;
  if (q >= l && q <= j - 1) ns = child[4 * s + 1];
  else if (q >= i && q <= ir) ns = child[4 * s + 2];
  segof[q] = ns;
}

// ---- one level per kernel -------------------------------------------------
__global__ void k_nr_median(const int* __restrict__ nsegp, const int* __restrict__ seg, const double* __restrict__ arr,
                            int* __restrict__ idx, double* __restrict__ piv, int* __restrict__ meta) {
  const int nseg = *nsegp;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
    nr_median_one(s, seg, arr, idx, piv, meta);
}

__global__ void k_nr_flags(int n, const int* __restrict__ segof, const int* __restrict__ seg,
                           const double* __restrict__ piv, const double* __restrict__ arr,
                           const int* __restrict__ idx, int* __restrict__ lf, int* __restrict__ rf) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n + 1; q += gridDim.x * blockDim.x) {
    int a, b;
    nr_flags_one(q, segof, seg, piv, arr, idx, a, b);
    lf[q] = a;
    rf[q] = b;
  }
}

__global__ void k_nr_scatter(int n, const int* __restrict__ lf, const int* __restrict__ rf,
                             const int* __restrict__ ls, const int* __restrict__ rs, int* __restrict__ lpos,
                             int* __restrict__ rpos) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n + 1; q += gridDim.x * blockDim.x) {
    if (lf[q]) lpos[ls[q]] = q;
    if (rf[q]) rpos[rs[q]] = q;
  }
}

__global__ void k_nr_cross(const int* __restrict__ nsegp, const int* __restrict__ seg, const int* __restrict__ ls,
                           const int* __restrict__ rs, const int* __restrict__ lpos,
                           const int* __restrict__ rpos, int* __restrict__ meta) {
  const int nseg = *nsegp;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
    nr_cross_one(s, seg, ls, rs, lpos, rpos, meta);
}

__global__ void k_nr_apply(int n, const int* __restrict__ segof, const int* __restrict__ seg,
                           const int* __restrict__ meta, const int* __restrict__ idx, const int* __restrict__ lf,
                           const int* __restrict__ rf, const int* __restrict__ ls, const int* __restrict__ rs,
                           const int* __restrict__ lpos, const int* __restrict__ rpos, int* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n; q += gridDim.x * blockDim.x)
    if (q > 0) out[q] = nr_apply_one(q, segof, seg, meta, idx, lf, rf, ls, rs, lpos, rpos);
}

// reads the level's segment count from cnt[in_slot] and counts the next
// level's segments in cnt[out_slot] (zeroed before the launch)
__global__ void k_nr_newsegs(int in_slot, int out_slot, const int* __restrict__ seg, int* __restrict__ meta,
                             int* __restrict__ seg2, int* __restrict__ small, int* __restrict__ med,
                             int* __restrict__ cnt, int small_cap, int med_cap) {
  const int nseg = cnt[in_slot];
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x)
    nr_newsegs_one(s, out_slot, seg, meta, meta, seg2, small, med, cnt, small_cap, med_cap);
}

__global__ void k_nr_segof(int n, const int* __restrict__ seg, const int* __restrict__ meta,
                           int* __restrict__ segof) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n + 1; q += gridDim.x * blockDim.x)
    nr_segof_one(q, seg, meta, segof);
}

// ---- all levels in one cooperative kernel ----------------------------------
// The phases of a level (stopper flags and their prefix sums with the stopper
// positions; crossings; the partitioned permutation with the next level's
// segments; segment ids with the next level's medians) are separated by
// grid-wide barriers, five per level, so the whole sort is one launch
// instead of about eleven per level.  The prefix
// sums run over contiguous chunks of positions, one chunk per block: block
// totals, then each block's offset, then a tiled scan of the chunk (the two
// flags packed into one int, 16 bits each, per 256-position tile).
struct NrCoop {
  int n;
  const double* arr;
  int *idx, *idx2, *seg, *seg2, *segof, *lf, *rf, *ls, *rs, *lpos, *rpos, *meta, *child, *small, *med, *cnt, *bsum;
  double* piv;
  int small_cap, med_cap;
  int max_levels;
};

constexpr int kCoopThreads = 256;

__device__ inline int block_sum(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int t = 0;
  if (threadIdx.x < kCoopThreads / 32) t = sh[threadIdx.x];
  if (w == 0)
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  __syncthreads();
  if (threadIdx.x == 0) sh[0] = t;
  __syncthreads();
  const int r = sh[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kCoopThreads) k_nr_levels(NrCoop A) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ int sh[kCoopThreads / 32];
  __shared__ int wsc[kCoopThreads / 32];
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  const int n = A.n, np = n + 2;  // positions 0..n+1
  const int chunk = (np + gridDim.x - 1) / gridDim.x;
  const int q0 = min(np, blockIdx.x * chunk), q1 = min(np, q0 + chunk);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int *idx = A.idx, *idx2 = A.idx2, *seg = A.seg, *seg2 = A.seg2;
  int in = C_NSEG, out = C_NSEG2;
  int level = 0;
  {  // the first level's medians; later levels' run with the previous level's segment ids
    const int nseg0 = __ldcg(&A.cnt[in]);
    for (int s = tid; s < nseg0; s += nthreads) nr_median_one(s, seg, A.arr, idx, A.piv, A.meta);
  }
  grid.sync();
  for (; level < A.max_levels; ++level) {
    const int nseg = __ldcg(&A.cnt[in]);
    if (nseg == 0) break;
    if (tid == 0) A.cnt[out] = 0;
    // stopper flags and the block's totals
    int tl = 0, tr = 0;
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
      int a, b;
      nr_flags_one(q, A.segof, seg, A.piv, A.arr, idx, a, b);
      A.lf[q] = a;
      A.rf[q] = b;
      tl += a;
      tr += b;
    }
    tl = block_sum(tl, sh);
    tr = block_sum(tr, sh);
    if (threadIdx.x == 0) { A.bsum[2 * blockIdx.x] = tl; A.bsum[2 * blockIdx.x + 1] = tr; }
    grid.sync();
    // this block's offsets, then the tiled exclusive scan of its chunk
    int ol = 0, orr = 0;
    for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) {
      ol += __ldcg(&A.bsum[2 * b]);
      orr += __ldcg(&A.bsum[2 * b + 1]);
    }
    ol = block_sum(ol, sh);
    orr = block_sum(orr, sh);
    for (int base = q0; base < q1; base += blockDim.x) {
      const int q = base + threadIdx.x;
      const int a = q < q1 ? A.lf[q] : 0, b = q < q1 ? A.rf[q] : 0;
      const int v = a | (b << 16);
      int x = v;  // inclusive warp scan of the packed pair
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsc[wid] = x;
      __syncthreads();
      if (wid == 0) {
        int w = lane < kCoopThreads / 32 ? wsc[lane] : 0;
        for (int o = 1; o < kCoopThreads / 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, w, o);
          if (lane >= o) w += y;
        }
        if (lane < kCoopThreads / 32) wsc[lane] = w;  // inclusive warp totals
      }
      __syncthreads();
      const int excl = x - v + (wid > 0 ? wsc[wid - 1] : 0);
      const int tot = wsc[kCoopThreads / 32 - 1];
      if (q < q1) {
        const int L = ol + (excl & 0xffff), R = orr + (excl >> 16);
        A.ls[q] = L;
        A.rs[q] = R;
        if (a) A.lpos[L] = q;
        if (b) A.rpos[R] = q;
      }
      ol += tot & 0xffff;
      orr += tot >> 16;
      __syncthreads();
    }
    grid.sync();
    for (int s = tid; s < nseg; s += nthreads) nr_cross_one(s, seg, A.ls, A.rs, A.lpos, A.rpos, A.meta);
    grid.sync();
    // the partitioned permutation and the children (apply reads meta, the
    // children go to child: one phase)
    for (int q = tid + 1; q <= n; q += nthreads)
      idx2[q] = nr_apply_one(q, A.segof, seg, A.meta, idx, A.lf, A.rf, A.ls, A.rs, A.lpos, A.rpos);
    for (int s = tid; s < nseg; s += nthreads)
      nr_newsegs_one(s, out, seg, A.meta, A.child, seg2, A.small, A.med, A.cnt, A.small_cap, A.med_cap);
    grid.sync();
    // segment ids from the children, and the next level's medians on the
    // partitioned permutation (they touch neither segof nor child: one phase)
    for (int q = tid; q <= n + 1; q += nthreads) nr_segof_one(q, seg, A.child, A.segof);
    {
      const int nnext = __ldcg(&A.cnt[out]);
      for (int s = tid; s < nnext; s += nthreads) nr_median_one(s, seg2, A.arr, idx2, A.piv, A.meta);
    }
    grid.sync();
    int* t = idx; idx = idx2; idx2 = t;
    t = seg; seg = seg2; seg2 = t;
    const int ti = in; in = out; out = ti;
  }
  if (tid == 0) {
    A.cnt[C_NRIDX] = idx == A.idx ? 0 : 1;
    A.cnt[C_NRLEVELS] = level;
  }
}

// straight insertion of a small segment (LocalMinima.f90:967-976); the
// reference's inner loop runs down to 1 but stops at position l-1 at the
// latest because everything left of a segment is <= everything in it.
__global__ void k_nr_insertion(int nsmall, const int* __restrict__ small, const double* __restrict__ arr,
                               int* __restrict__ idx) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsmall; s += gridDim.x * blockDim.x) {
    const int l = small[2 * s], ir = small[2 * s + 1];
    for (int j = l + 1; j <= ir; ++j) {
      const int indxt = idx[j];
      const double a = arr[indxt];
      int i = j - 1;
      for (; i >= l; --i) {
        if (arr[idx[i]] <= a) break;
        idx[i + 1] = idx[i];
      }
      idx[i + 1] = indxt;
    }
  }
}

// The whole NR quicksort of one segment of 8..kNrMedium elements, as the
// reference runs it (LocalMinima.f90:953-1044: median of three, Hoare scans,
// larger part stacked, straight insertion below M = 7), by one thread on the
// segment's keys and ids in shared memory; positions are relative to the
// segment (the median index (l+ir)/2 keeps its value relative to l).
// Segments are independent, so the order they are finished in does not
// matter, and the insertion stops at the segment's start as k_nr_insertion's does.
__device__ bool nr_sort_local(double* key, int* id, int n) {
  int stk[32];
  int js = 0, l = 0, ir = n - 1;
  for (int it = 0; it < 4 * kNrMedium; ++it) {
    if (ir - l < 7) {
      for (int j = l + 1; j <= ir; ++j) {
        const double a = key[j];
        const int v = id[j];
        int i = j - 1;
        for (; i >= l; --i) {
          if (key[i] <= a) break;
          key[i + 1] = key[i];
          id[i + 1] = id[i];
        }
        key[i + 1] = a;
        id[i + 1] = v;
      }
      if (js == 0) return true;
      ir = stk[--js];
      l = stk[--js];
    } else {
      auto swap = [&](int x, int y) {
        const double t = key[x]; key[x] = key[y]; key[y] = t;
        const int u = id[x]; id[x] = id[y]; id[y] = u;
      };
      swap((l + ir) / 2, l + 1);
      if (key[l + 1] > key[ir]) swap(l + 1, ir);
      if (key[l] > key[ir]) swap(l, ir);
      if (key[l + 1] > key[l]) swap(l + 1, l);
      int i = l + 1, j = ir;
      const double a = key[l];
      const int v = id[l];
      for (;;) {  // the median of three leaves stoppers at l+1 and ir
        do ++i; while (key[i] < a);
        do --j; while (key[j] > a);
        if (j < i) break;
        swap(i, j);
      }
      key[l] = key[j];
      id[l] = id[j];
      key[j] = a;
      id[j] = v;
      if (js + 2 > 32) return false;  // depth <= 2*log2(kNrMedium) = 18
      if (ir - i + 1 >= j - l) {
        stk[js++] = i;
        stk[js++] = ir;
        ir = j - 1;
      } else {
        stk[js++] = l;
        stk[js++] = j - 1;
        l = i;
      }
    }
  }
  return false;
}

constexpr int kNrMedWarps = 4;
__global__ void __launch_bounds__(32 * kNrMedWarps) k_nr_medium(int nmed, const int* __restrict__ med,
                                                               const double* __restrict__ arr, int* __restrict__ idx,
                                                               int* __restrict__ cnt) {
  __shared__ double key[kNrMedWarps][kNrMedium];
  __shared__ int id[kNrMedWarps][kNrMedium];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int s = blockIdx.x * kNrMedWarps + w; s < nmed; s += gridDim.x * kNrMedWarps) {
    const int l = med[2 * s], n = med[2 * s + 1] - l + 1;
    if (n < 8 || n > kNrMedium) {  // never: nr_newsegs_one routes only such segments here
      if (lane == 0) atomicExch(&cnt[C_OVERFLOW], 1);
      continue;
    }
    for (int p = lane; p < n; p += 32) {
      const int v = idx[l + p];
      id[w][p] = v;
      key[w][p] = arr[v];
    }
    __syncwarp();
    if (lane == 0 && !nr_sort_local(key[w], id[w], n)) atomicExch(&cnt[C_OVERFLOW], 1);
    __syncwarp();
    for (int p = lane; p < n; p += 32) idx[l + p] = id[w][p];
    __syncwarp();
  }
}

__global__ void k_rank_from_perm(int n, const int* __restrict__ idx1, int* __restrict__ rank) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    rank[idx1[t + 1] - 1] = t;
}

// ---- Boruvka under the rank order ------------------------------------------
__global__ void k_mst_init(int nb, int* __restrict__ comp) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) comp[b] = b;
}

// Host-driven Borůvka rounds (graphs above kMstCoopMax edges).  Rounds are
// launched in batches without a read-back in between: once a round's hooking
// changes nothing, k_mst_check sets C_MST_DONE and every later kernel of the
// batch returns at once.
__global__ void k_mst_reset(int nb, int* __restrict__ mn, const int* __restrict__ done) {
  if (*done) return;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) mn[b] = INT_MAX;
}

__global__ void k_mst_minedge(int ne, const int* __restrict__ b1, const int* __restrict__ b2,
                              const int* __restrict__ rank, const int* __restrict__ comp, int* __restrict__ mn,
                              const int* __restrict__ done) {
  if (*done) return;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const int cu = comp[b1[e] - 1], cv = comp[b2[e] - 1];
    if (cu == cv) continue;
    atomicMin(&mn[cu], rank[e]);
    atomicMin(&mn[cv], rank[e]);
  }
}

__global__ void k_mst_hook(int nb, const int* __restrict__ idx1, const int* __restrict__ b1,
                           const int* __restrict__ b2, const int* __restrict__ comp, const int* __restrict__ mn,
                           int* __restrict__ next, int* __restrict__ inmst, int* __restrict__ cnt) {
  if (cnt[C_MST_DONE]) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nb; c += gridDim.x * blockDim.x) {
    next[c] = comp[c];
    if (comp[c] != c) continue;
    const int r = mn[c];
    if (r == INT_MAX) continue;
    const int e = idx1[r + 1] - 1;
    const int cu = comp[b1[e] - 1], cv = comp[b2[e] - 1];
    const int other = cu == c ? cv : cu;
    inmst[e] = 1;
    if (mn[other] == r && c < other) continue;  // mutual choice: the smaller id stays a root
    next[c] = other;
    cnt[C_CHANGED] = 1;
  }
}

// one thread: a round whose hooking changed nothing ends the MST
__global__ void k_mst_check(int* cnt) {
  if (cnt[C_MST_DONE]) return;
  if (!cnt[C_CHANGED]) cnt[C_MST_DONE] = 1;
  cnt[C_CHANGED] = 0;
}

__global__ void k_mst_apply(int nb, const int* __restrict__ next, int* __restrict__ comp,
                            const int* __restrict__ done) {
  if (*done) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nb; c += gridDim.x * blockDim.x) comp[c] = next[c];
}

// Flattens the hook forest in one launch: each thread moves its pointer to
// its grandparent until it reaches a root.  Other threads' updates only move
// pointers towards the roots (which never change here), so every thread ends
// at its root; the loop is bounded by the number of components.
__global__ void k_mst_flatten(int nb, int* comp, int* cnt) {
  if (*(volatile int*)&cnt[C_MST_DONE]) return;
  volatile int* vc = comp;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nb; c += gridDim.x * blockDim.x) {
    int it = 0;
    for (;; ++it) {
      const int r = vc[c];
      const int rr = vc[r];
      if (rr == r) break;
      if (it > nb) {  // not a forest
        atomicExch(&cnt[C_OVERFLOW], 1);
        break;
      }
      vc[c] = rr;
    }
  }
}

// All Borůvka rounds in one cooperative launch (the kernels above, as phases
// separated by grid-wide barriers), so that no round waits for the host.
// Flattening jumps in place: comp[c] <- comp[comp[c]] only ever moves a
// pointer towards its root, so concurrent updates leave the same roots.  A
// pass's "not flat" flag is one of three slots used in turn: the slot a pass
// sets was cleared two barriers earlier, after every thread had read it.
// Rounds and passes are bounded (64 each, as the host loop); a flatten that
// does not end sets the overflow counter.
struct MstCoop {
  int nb, ne;
  const int *idx1, *b1, *b2, *rank;
  int *comp, *mn, *next, *inmst, *cnt;
};

__global__ void __launch_bounds__(kCoopThreads) k_mst_coop(MstCoop A) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int nthreads = gridDim.x * blockDim.x;
  volatile int* comp = A.comp;
  for (int c = tid; c < A.nb; c += nthreads) comp[c] = c;
  for (int round = 0; round < 64; ++round) {
    for (int c = tid; c < A.nb; c += nthreads) A.mn[c] = INT_MAX;
    if (tid == 0) {
      A.cnt[C_MST_CHANGED] = 0;
      A.cnt[C_MST_FLAT] = 0;
    }
    grid.sync();
    for (int e = tid; e < A.ne; e += nthreads) {
      const int cu = comp[A.b1[e] - 1], cv = comp[A.b2[e] - 1];
      if (cu == cv) continue;
      atomicMin(&A.mn[cu], A.rank[e]);
      atomicMin(&A.mn[cv], A.rank[e]);
    }
    grid.sync();
    for (int c = tid; c < A.nb; c += nthreads) {
      A.next[c] = comp[c];
      if (comp[c] != c) continue;
      const int r = __ldcg(&A.mn[c]);
      if (r == INT_MAX) continue;
      const int e = A.idx1[r + 1] - 1;
      const int cu = comp[A.b1[e] - 1], cv = comp[A.b2[e] - 1];
      const int other = cu == c ? cv : cu;
      A.inmst[e] = 1;
      if (__ldcg(&A.mn[other]) == r && c < other) continue;  // mutual choice: the smaller id stays a root
      A.next[c] = other;
      A.cnt[C_MST_CHANGED] = 1;
    }
    grid.sync();
    if (__ldcg(&A.cnt[C_MST_CHANGED]) == 0) break;  // read by every thread after the barrier
    for (int c = tid; c < A.nb; c += nthreads) comp[c] = __ldcg(&A.next[c]);
    grid.sync();
    bool flat = false;
    for (int pass = 0; pass < 64; ++pass) {
      volatile int* fl = A.cnt + C_MST_FLAT + pass % 3;
      if (tid == 0) A.cnt[C_MST_FLAT + (pass + 1) % 3] = 0;
      for (int c = tid; c < A.nb; c += nthreads) {
        const int r = comp[c];
        const int rr = comp[r];
        if (rr != r) {
          comp[c] = rr;
          *fl = 1;
        }
      }
      grid.sync();
      if (*fl == 0) {
        flat = true;
        break;
      }
    }
    if (!flat) {
      if (tid == 0) A.cnt[C_OVERFLOW] = 1;
      break;
    }
  }
}

// tree = accepted edges in rank order (Kruskal acceptance order)
__global__ void k_tree_flags(int ne, const int* __restrict__ idx1, const int* __restrict__ inmst,
                             int* __restrict__ flag) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= ne; t += gridDim.x * blockDim.x)
    flag[t] = t < ne ? inmst[idx1[t + 1] - 1] : 0;
}

__global__ void k_tree_list(int ne, const int* __restrict__ idx1, const int* __restrict__ flag,
                            const int* __restrict__ scan, int* __restrict__ tree) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ne; t += gridDim.x * blockDim.x)
    if (flag[t]) tree[scan[t]] = idx1[t + 1] - 1;
}

// ---- order_tree: Euler tour over the tree arcs -------------------------------
__global__ void k_arc_degree(int ntree, const int* __restrict__ tree, const int* __restrict__ b1,
                             const int* __restrict__ b2, int* __restrict__ deg) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ntree; x += gridDim.x * blockDim.x) {
    const int e = tree[x];
    atomicAdd(&deg[b1[e] - 1], 1);
    atomicAdd(&deg[b2[e] - 1], 1);
  }
}

__global__ void k_arc_fill(int ntree, const int* __restrict__ tree, const int* __restrict__ b1,
                           const int* __restrict__ b2, const int* __restrict__ start, int* __restrict__ fill,
                           int* __restrict__ adj, int* __restrict__ slot) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ntree; x += gridDim.x * blockDim.x) {
    const int e = tree[x];
    const int u = b1[e] - 1, v = b2[e] - 1;
    const int su = atomicAdd(&fill[u], 1);
    adj[start[u] + su] = 2 * x;       // arc u -> v
    slot[2 * x] = su;
    const int sv = atomicAdd(&fill[v], 1);
    adj[start[v] + sv] = 2 * x + 1;   // arc v -> u
    slot[2 * x + 1] = sv;
  }
}

__global__ void k_arc_tour(int ntree, int root, const int* __restrict__ tree, const int* __restrict__ b1,
                           const int* __restrict__ b2, const int* __restrict__ start,
                           const int* __restrict__ deg, const int* __restrict__ adj,
                           const int* __restrict__ slot, unsigned long long* __restrict__ lst) {
  const unsigned END = 0xffffffffu;
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < 2 * ntree; a += gridDim.x * blockDim.x) {
    const int e = tree[a >> 1];
    const int y = (a & 1) ? b1[e] - 1 : b2[e] - 1;  // head of arc a
    const int tw = a ^ 1;                           // twin arc y -> x
    const int ns = (slot[tw] + 1) % deg[y];
    unsigned succ = (unsigned)adj[start[y] + ns];
    if (y == root && ns == 0) succ = END;
    lst[a] = ((unsigned long long)succ << 32) | 1ull;
  }
}

__global__ void k_copy_edges(int ne, const int* __restrict__ b1, const int* __restrict__ b2,
                             const int* __restrict__ n1, const int* __restrict__ n2, int* __restrict__ ob1,
                             int* __restrict__ ob2, int* __restrict__ on1, int* __restrict__ on2) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    ob1[e] = b1[e]; ob2[e] = b2[e]; on1[e] = n1[e]; on2[e] = n2[e];
  }
}

__global__ void k_orient_tree(int ntree, const int* __restrict__ tree, const unsigned long long* __restrict__ rk,
                              const int* __restrict__ b1, const int* __restrict__ b2, const int* __restrict__ n1,
                              const int* __restrict__ n2, int* __restrict__ ob1, int* __restrict__ ob2,
                              int* __restrict__ on1, int* __restrict__ on2) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ntree; x += gridDim.x * blockDim.x) {
    const int e = tree[x];
    const unsigned r_uv = (unsigned)rk[2 * x], r_vu = (unsigned)rk[2 * x + 1];
    // the arc met first in the tour (larger distance to the end) leaves the parent
    if (r_uv < r_vu) {
      ob1[e] = b2[e]; ob2[e] = b1[e]; on1[e] = n2[e]; on2[e] = n1[e];
    }
  }
}

// correct_receivers_v2: redirect node_from to node_to and reverse the
// receiver path from node_from down to the child basin's outlet
__global__ void k_correct(int ntree, int nx, double dx, double dy, int nn, const int* __restrict__ tree,
                          const int* __restrict__ ob2, const int* __restrict__ on1, const int* __restrict__ on2,
                          const int* __restrict__ roots, int* rec, double* length, int* __restrict__ err) {
  for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < ntree; x += gridDim.x * blockDim.x) {
    const int e = tree[x];
    const int node_to = on1[e], node_from = on2[e];
    if (node_from == -1) continue;
    const int outlet_from = roots[ob2[e] - 1];
    int next_node = rec[node_from];
    int cur = node_from;
    double prev = length[node_from];
    rec[node_from] = node_to;
    const double ddx = dx * (double)((node_from % nx) - (node_to % nx));
    const double ddy = dy * (double)((node_from / nx) - (node_to / nx));
    length[node_from] = sqrt(ddx * ddx + ddy * ddy);
    int guard = 0;
    while (cur != outlet_from) {
      if (++guard > nn) { atomicExch(err, DEV_STACK_ERROR); break; }
      const int rcv_next = rec[next_node];
      rec[next_node] = cur;
      const double tmp = prev;
      prev = length[next_node];
      length[next_node] = tmp;
      cur = next_node;
      next_node = rcv_next;
    }
  }
}

__global__ void k_count_active_roots(Bounds bd, const int* __restrict__ rec, int* __restrict__ cnt) {
  const int nn = bd.nx * bd.ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    if (rec[k] == k && !is_bc_node(bd, k % bd.nx, k / bd.nx)) atomicAdd(&cnt[C_NLOCMIN_AFTER], 1);
}

__global__ void k_copy_nroots(const int* src, int* cnt) {
  cnt[C_NBASINS] = *src;
  cnt[C_NLOCMIN] = 0;
  cnt[C_BASIN0] = INT_MAX;
  for (int i = C_NEDGE; i <= C_OVERFLOW; ++i) cnt[i] = 0;
}

}  // namespace

// Runs the exact NR index sort on w[0..n-1]; result: c.nr_idx[1..n] holds the
// 1-based ids in sorted order.  Returns false on buffer overflow.
// All levels in one cooperative launch; false when the device cannot run it
// (the caller then runs one launch per level).  Reads the counters back.
static int nr_med_cap(const Ctx& c) { return (int)(c.conn_cap / 8 + 8); }

static bool nr_levels_coop(Ctx& c, int n, const double* arr, int small_cap) {
  int dev = 0, coop = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nr_levels, kCoopThreads, 0) != cudaSuccess ||
      per_sm < 1)
    return false;
  // about 2048 positions per block, at most what is resident at once
  const int want = (n + 2 + 2047) / 2048;
  const int blocks = std::max(1, std::min(want, std::min(sms * per_sm, c.nr_bsum_cap / 2)));
  NrCoop A{n,         arr,       c.nr_idx,  c.nr_idx2, c.nr_seg,     c.nr_seg2,  c.nr_segof,
           c.nr_lf,   c.nr_rf,   c.nr_ls,   c.nr_rs,   c.nr_lpos,    c.nr_rpos,  c.nr_segmeta, c.nr_child,
           c.nr_small, c.nr_med, c.d_cnt,   c.nr_bsum, c.nr_piv,     small_cap,  nr_med_cap(c),
           nr_max_levels(n)};
  void* args[] = {&A};
  if (cudaLaunchCooperativeKernel((const void*)k_nr_levels, dim3(blocks), dim3(kCoopThreads), args, 0, c.stream) !=
      cudaSuccess) {
    cudaGetLastError();  // clear the launch error; the per-level path runs instead
    return false;
  }
  c.count_launch();
  fetch_counters(c, kNrCounters);
  return true;
}

static bool nr_indexx(Ctx& c, int n, const double* w) {
  const double* arr = w - 1;  // 1-based
  int* idx = c.nr_idx;
  int* idx2 = c.nr_idx2;
  int* seg = c.nr_seg;
  int* seg2 = c.nr_seg2;
  const int small_cap = (int)(c.conn_cap / 2 + 8);
  k_nr_init<<<grid1d(n + 2), kBlock, 0, c.stream>>>(n, idx, c.nr_segof, seg, c.nr_small, c.nr_med, c.d_cnt);
  c.count_launch();
  int nseg = 1;  // k_nr_init makes one segment of the whole array when n > kNrMedium
  if (n <= kNrMedium) {
    fetch_counters(c, kNrCounters);
    nseg = c.h_cnt[C_NSEG];
  }
  if (nseg > 0 && nr_levels_coop(c, n, arr, small_cap)) {
    if (c.h_cnt[C_OVERFLOW]) { c.err = "NR sort emulation: small-segment buffer overflow"; return false; }
    if (c.h_cnt[C_NRLEVELS] >= nr_max_levels(n)) { c.err = "NR sort emulation: too many levels"; return false; }
    if (c.h_cnt[C_NRIDX]) std::swap(idx, idx2);
    nseg = 0;  // all levels done
  }
  // Levels run with the segment count on the device (slot `in` of d_cnt), a
  // few levels per read-back: a level with no segment left changes nothing.
  // Every segment holds at least 8 elements, so a level has at most n/8.
  const unsigned gseg = grid1d((size_t)n / 8 + 1);
  int in = C_NSEG, out = C_NSEG2;
  int levels = 0;
  while (nseg > 0) {
    for (int b = 0; b < 4; ++b) {
      if (++levels > nr_max_levels(n)) { c.err = "NR sort emulation: too many levels"; return false; }
      const int* nsegp = c.d_cnt + in;
      k_nr_median<<<gseg, kBlock, 0, c.stream>>>(nsegp, seg, arr, idx, c.nr_piv, c.nr_segmeta);
      k_nr_flags<<<grid1d(n + 2), kBlock, 0, c.stream>>>(n, c.nr_segof, seg, c.nr_piv, arr, idx, c.nr_lf, c.nr_rf);
      exclusive_scan_int(c, c.nr_lf, c.nr_ls, n + 2);
      exclusive_scan_int(c, c.nr_rf, c.nr_rs, n + 2);
      k_nr_scatter<<<grid1d(n + 2), kBlock, 0, c.stream>>>(n, c.nr_lf, c.nr_rf, c.nr_ls, c.nr_rs, c.nr_lpos,
                                                            c.nr_rpos);
      k_nr_cross<<<gseg, kBlock, 0, c.stream>>>(nsegp, seg, c.nr_ls, c.nr_rs, c.nr_lpos, c.nr_rpos, c.nr_segmeta);
      k_nr_apply<<<grid1d(n + 1), kBlock, 0, c.stream>>>(n, c.nr_segof, seg, c.nr_segmeta, idx, c.nr_lf, c.nr_rf,
                                                          c.nr_ls, c.nr_rs, c.nr_lpos, c.nr_rpos, idx2);
      std::swap(idx, idx2);
      cudaMemsetAsync(c.d_cnt + out, 0, sizeof(int), c.stream);
      k_nr_newsegs<<<gseg, kBlock, 0, c.stream>>>(in, out, seg, c.nr_segmeta, seg2, c.nr_small, c.nr_med, c.d_cnt,
                                                  small_cap, nr_med_cap(c));
      k_nr_segof<<<grid1d(n + 2), kBlock, 0, c.stream>>>(n, seg, c.nr_segmeta, c.nr_segof);
      c.count_launch(7);
      std::swap(seg, seg2);
      std::swap(in, out);
    }
    fetch_counters(c, kNrCounters);
    nseg = c.h_cnt[in];
    if (c.h_cnt[C_OVERFLOW]) { c.err = "NR sort emulation: small-segment buffer overflow"; return false; }
  }
  const int nmed = c.h_cnt[C_NMED];
  if (nmed > 0) {
    const int blocks = std::min((nmed + kNrMedWarps - 1) / kNrMedWarps, 148 * 16);
    k_nr_medium<<<blocks, 32 * kNrMedWarps, 0, c.stream>>>(nmed, c.nr_med, arr, idx, c.d_cnt);
    c.count_launch();
  }
  const int nsmall = c.h_cnt[C_NSMALL];
  if (nsmall > 0) {
    k_nr_insertion<<<grid1d(nsmall), kBlock, 0, c.stream>>>(nsmall, c.nr_small, arr, idx);
    c.count_launch();
  }
  if (nmed > 0) {  // the medium kernel reports an impossible segment through the overflow flag
    fetch_counters(c, kNrCounters);
    if (c.h_cnt[C_OVERFLOW]) { c.err = "NR sort emulation: medium segment out of range"; return false; }
  }
  if (idx != c.nr_idx)
    cudaMemcpyAsync(c.nr_idx, idx, sizeof(int) * (n + 2), cudaMemcpyDeviceToDevice, c.stream);
  return true;
}

// Borůvka in one cooperative launch; false when the device refuses it or the
// graph is large (the host-driven rounds run instead).  Measured on B200: the
// cooperative form saves the rounds' read-backs (1025^2 grid, 3.7e5 edges:
// LocalMinima 3.12 -> 2.71 ms), but its grid-wide barriers over many blocks
// cost more than they save on large graphs (2049^2, 1.5e6 edges: 5.08 ->
// 5.74 ms), hence the size limit.
constexpr int kMstCoopMax = 1 << 20;

static bool mst_coop(Ctx& c, int nroots, int ne) {
  if (std::max(ne, nroots) > kMstCoopMax) return false;
  int dev = 0, coop = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mst_coop, kCoopThreads, 0) != cudaSuccess ||
      per_sm < 1) {
    cudaGetLastError();
    return false;
  }
  // about 2048 edges per block, at most what is resident at once
  const int want = (std::max(ne, nroots) + 2047) / 2048;
  const int blocks = std::max(1, std::min(want, sms * per_sm));
  MstCoop A{nroots, ne, c.nr_idx, c.e_b1, c.e_b2, c.e_rank, c.mst_comp, c.mst_min, c.mst_next, c.e_inmst, c.d_cnt};
  void* args[] = {&A};
  if (cudaLaunchCooperativeKernel((const void*)k_mst_coop, dim3(blocks), dim3(kCoopThreads), args, 0, c.stream) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  c.count_launch();
  return true;
}

bool local_minima(Ctx& c) {
  const int nn = c.nn;
  cudaStream_t st = c.stream;
  if (c.capture) {
    cudaMemcpyAsync(c.rec_pre, c.rec, sizeof(int) * nn, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(c.stack_pre, c.stack, sizeof(int) * nn, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(c.length_pre, c.length, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
  }
  // ---- compute_basins: basin id = number of roots met so far along the stack
  k_copy_nroots<<<1, 1, 0, st>>>(c.s_scan + nn, c.d_cnt);
  k_pos_root_flags<<<grid1d(nn), kBlock, 0, st>>>(nn, c.stack, c.rec, c.s_flag);
  c.count_launch(2);
  inclusive_scan_int(c, c.s_flag, c.s_scan2, nn);
  k_basins<<<grid1d(nn), kBlock, 0, st>>>(nn, c.stack, c.s_scan2, c.basins);
  c.count_launch();
  catchment(c);  // find_stack's catch: labels of the forest before re-routing
  k_roots_scan<<<grid1d(nn), kBlock, 0, st>>>(c.bd, c.s_roots, c.d_cnt);
  c.count_launch();
  fetch_counters(c, 10);
  const int nroots = c.h_cnt[C_NBASINS];
  c.nbasins = nroots;
  c.nlocmin_before = c.h_cnt[C_NLOCMIN];
  c.basin0 = c.h_cnt[C_BASIN0] == INT_MAX ? -1 : c.h_cnt[C_BASIN0];
  c.nconn = 0;
  c.tree_size = 0;
  c.nlocmin_after = c.nlocmin_before;
  if (c.nlocmin_before == 0 && !c.capture) return true;  // no pit: receivers unchanged
  if (c.basin0 < 1) {
    c.err = "LocalMinima: no basin drains to a fixed boundary (the reference indexes out of bounds here)";
    return false;
  }
  // ---- connect_basins
  size_t cap = 1024;
  while (cap < 16 * (size_t)nroots && cap < c.hash_cap) cap <<= 1;
  cudaMemsetAsync(c.ht_key, 0xff, sizeof(unsigned long long) * cap, st);
  cudaMemsetAsync(c.ht_wmin, 0xff, sizeof(unsigned long long) * cap, st);
  cudaMemsetAsync(c.ht_first, 0xff, sizeof(unsigned) * cap, st);
  cudaMemsetAsync(c.ht_best, 0xff, sizeof(unsigned) * cap, st);
  k_conn_pass<0><<<grid1d(nn), kBlock, 0, st>>>(c.bd, c.basins, c.s_roots, c.pos, c.h, c.ht_key, c.ht_wmin,
                                                 c.ht_first, c.ht_best, cap, c.d_cnt);
  k_conn_pass<1><<<grid1d(nn), kBlock, 0, st>>>(c.bd, c.basins, c.s_roots, c.pos, c.h, c.ht_key, c.ht_wmin,
                                                 c.ht_first, c.ht_best, cap, c.d_cnt);
  k_conn_compact<<<grid1d(cap), kBlock, 0, st>>>(c.bd, cap, c.ht_key, c.ht_first, c.ht_best, c.stack, c.h,
                                                  c.conn_cap, c.e_key, c.r_b1, c.r_b2, c.r_n1, c.r_n2,
                                                  c.r_w, c.d_cnt);
  k_conn_virtual<<<grid1d(nroots), kBlock, 0, st>>>(c.bd, nroots, c.s_roots, c.pos, c.conn_cap, c.e_key, c.r_b1,
                                                     c.r_b2, c.r_n1, c.r_n2, c.r_w, c.d_cnt);
  c.count_launch(4);
  fetch_counters(c, 10);
  if (c.h_cnt[C_OVERFLOW]) { c.err = "connect_basins: edge buffer overflow"; return false; }
  const int ne = c.h_cnt[C_NEDGE];
  c.nconn = ne;
  if (ne > 6 * nroots) {
    c.err = "connect_basins: nconn exceeds nconn_max=6*nbasins (the reference overflows here)";
    return false;
  }
  k_iota<<<grid1d(ne), kBlock, 0, st>>>(ne, c.e_idx);
  c.count_launch();
  int bits = 1;
  while (bits < 32 && (1ull << bits) < 8ull * (unsigned long long)nn) ++bits;
  sort_pairs_u32(c, c.e_key, c.e_key2, c.e_idx, c.e_idx2, ne, bits);
  k_conn_gather<<<grid1d(ne), kBlock, 0, st>>>(ne, c.e_idx2, c.r_b1, c.r_b2, c.r_n1, c.r_n2, c.r_w, c.e_b1,
                                                c.e_b2, c.e_n1, c.e_n2, c.e_w);
  c.count_launch();
  // ---- loc_min_3_indexx + Kruskal
  if (!nr_indexx(c, ne, c.e_w)) return false;
  k_rank_from_perm<<<grid1d(ne), kBlock, 0, st>>>(ne, c.nr_idx, c.e_rank);
  cudaMemsetAsync(c.e_inmst, 0, sizeof(int) * ne, st);
  k_mst_init<<<grid1d(nroots), kBlock, 0, st>>>(nroots, c.mst_comp);
  c.count_launch(2);
  if (!mst_coop(c, nroots, ne)) {
    // rounds in batches of four, one read-back per batch (Borůvka at least
    // halves the components per round, so the bound of 64 is never reached)
    constexpr int kMstBatch = 4;
    cudaMemsetAsync(c.d_cnt + C_CHANGED, 0, sizeof(int), st);
    cudaMemsetAsync(c.d_cnt + C_MST_DONE, 0, sizeof(int), st);
    const int* done = c.d_cnt + C_MST_DONE;
    for (int round = 0; round < 64; round += kMstBatch) {
      for (int r = 0; r < kMstBatch; ++r) {
        k_mst_reset<<<grid1d(nroots), kBlock, 0, st>>>(nroots, c.mst_min, done);
        k_mst_minedge<<<grid1d(ne), kBlock, 0, st>>>(ne, c.e_b1, c.e_b2, c.e_rank, c.mst_comp, c.mst_min, done);
        k_mst_hook<<<grid1d(nroots), kBlock, 0, st>>>(nroots, c.nr_idx, c.e_b1, c.e_b2, c.mst_comp, c.mst_min,
                                                       c.mst_next, c.e_inmst, c.d_cnt);
        k_mst_check<<<1, 1, 0, st>>>(c.d_cnt);
        k_mst_apply<<<grid1d(nroots), kBlock, 0, st>>>(nroots, c.mst_next, c.mst_comp, done);
        k_mst_flatten<<<grid1d(nroots), kBlock, 0, st>>>(nroots, c.mst_comp, c.d_cnt);
        c.count_launch(6);
      }
      fetch_counters(c, C_MST_DONE + 1);
      if (c.h_cnt[C_MST_DONE]) break;
    }
  }
  k_tree_flags<<<grid1d(ne + 1), kBlock, 0, st>>>(ne, c.nr_idx, c.e_inmst, c.nr_lf);
  c.count_launch();
  exclusive_scan_int(c, c.nr_lf, c.nr_ls, ne + 1);
  k_tree_list<<<grid1d(ne), kBlock, 0, st>>>(ne, c.nr_idx, c.nr_lf, c.nr_ls, c.tree);
  cudaMemcpyAsync(c.d_cnt + C_NTREE, c.nr_ls + ne, sizeof(int), cudaMemcpyDeviceToDevice, st);
  c.count_launch();
  fetch_counters(c, 10);
  const int ntree = c.h_cnt[C_NTREE];
  c.tree_size = ntree;
  if (c.h_cnt[C_OVERFLOW]) {
    c.err = "LocalMinima: the spanning tree's components did not flatten";
    return false;
  }
  if (ntree != nroots - 1) {
    c.err = "LocalMinima: the basin graph is not connected";
    return false;
  }
  // ---- order_tree
  k_copy_edges<<<grid1d(ne), kBlock, 0, st>>>(ne, c.e_b1, c.e_b2, c.e_n1, c.e_n2, c.o_b1, c.o_b2, c.o_n1,
                                              c.o_n2);
  c.count_launch();
  if (ntree > 0) {
    cudaMemsetAsync(c.arc_deg, 0, sizeof(int) * (nroots + 1), st);
    k_arc_degree<<<grid1d(ntree), kBlock, 0, st>>>(ntree, c.tree, c.e_b1, c.e_b2, c.arc_deg);
    c.count_launch();
    exclusive_scan_int(c, c.arc_deg, c.arc_start, nroots + 1);
    cudaMemsetAsync(c.mst_min, 0, sizeof(int) * nroots, st);
    k_arc_fill<<<grid1d(ntree), kBlock, 0, st>>>(ntree, c.tree, c.e_b1, c.e_b2, c.arc_start, c.mst_min,
                                                  c.arc_adj, c.arc_slot);
    k_arc_tour<<<grid1d(2 * ntree), kBlock, 0, st>>>(ntree, c.basin0 - 1, c.tree, c.e_b1, c.e_b2, c.arc_start,
                                                      c.arc_deg, c.arc_adj, c.arc_slot, c.s_list_a);
    c.count_launch(2);
    unsigned long long* rk = list_rank(c, 2 * (size_t)ntree, c.s_list_a, c.s_list_b);
    k_orient_tree<<<grid1d(ntree), kBlock, 0, st>>>(ntree, c.tree, rk, c.e_b1, c.e_b2, c.e_n1, c.e_n2, c.o_b1,
                                                     c.o_b2, c.o_n1, c.o_n2);
    // ---- correct_receivers_v2
    k_correct<<<grid1d(ntree, 128), 128, 0, st>>>(ntree, c.nx, c.dx, c.dy, nn, c.tree, c.o_b2, c.o_n1, c.o_n2,
                                                   c.s_roots, c.rec, c.length, c.d_err);
    c.count_launch(2);
  }
  if (c.capture) {
    k_count_active_roots<<<grid1d(nn), kBlock, 0, st>>>(c.bd, c.rec, c.d_cnt);
    c.count_launch();
    fetch_counters(c, 10);
    c.nlocmin_after = c.h_cnt[C_NLOCMIN_AFTER];
  }
  // loc_min_3_find_donors + loc_min_3_find_stack
  build_stack(c, c.rec, c.ndon, c.don, c.stack, c.pos, c.size);
  return true;
}

}  // namespace fsb
