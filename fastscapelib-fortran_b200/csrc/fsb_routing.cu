// Flow routing kernels: uplift, steepest-descent receivers, donor lists and the
// depth-first stack (DFS preorder) of the receiver forest.
//
// Reference routines restated here (file:line in fastscapelib-fortran):
//   Uplift                 src/Uplift.f90:9-10
//   find_receiver          src/FlowRouting.f90:302-362
//   find_donor             src/FlowRouting.f90:366-389 (= loc_min_3_find_donors,
//                          src/LocalMinima.f90:881-900)
//   find_stack(+recursion) src/FlowRouting.f90:393-443 (= loc_min_3_find_stack,
//                          src/LocalMinima.f90:904-923,1050-1067)
//
// The stack is the DFS preorder of the receiver forest with roots in ascending
// node order and children (donors) in ascending node order.  Instead of the
// reference's recursion it is built from the Euler tour of the forest: every
// node k contributes an enter event E(k)=2k and an exit event X(k)=2k+1, the
// tour successor of each event is local information (first donor, next
// sibling, parent, next root), and list ranking by pointer jumping counts the
// enter events from each event to the end of the tour.  That count gives the
// preorder position and the subtree size of every node exactly.
#include "fsb_kernels.cuh"

namespace fsb {

// ---------------------------------------------------------------------------
// Uplift: h += u*dt ; b += u*dt   (no FMA: the library is built --fmad=false)
__global__ void k_uplift(int nn, double dt, const double* __restrict__ u, double* __restrict__ h,
                         double* __restrict__ b) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double du = u[k] * dt;
    h[k] = h[k] + du;
    b[k] = b[k] + du;
  }
}

// find_receiver: one thread per node, 3x3 stencil, jj outer / ii inner, the
// first strictly steeper neighbour wins (smax starts at tiny(1d0)).  Lengths
// come from the 3x3 table `ltab` computed on the host exactly like the
// reference's sqrt((dx*ii)**2+(dy*jj)**2).
__global__ void k_find_receiver(Bounds bd, const double* __restrict__ h, const double* __restrict__ ltab,
                                int* __restrict__ rec, double* __restrict__ length) {
  const int nx = bd.nx, ny = bd.ny;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= nx || j >= ny) return;
  const int ij = i + j * nx;
  int r = ij;
  double len = 0.0;
  if (i >= bd.i1 && i <= bd.i2 && j >= bd.j1 && j <= bd.j2) {
    const double hij = h[ij];
    double smax = 2.2250738585072014e-308;
#pragma unroll
    for (int jj = -1; jj <= 1; ++jj) {
      const int jjj = wrap_clamp(j + jj, ny, bd.ycyc);
#pragma unroll
      for (int ii = -1; ii <= 1; ++ii) {
        const int iii = wrap_clamp(i + ii, nx, bd.xcyc);
        const int ijk = iii + jjj * nx;
        if (ijk != ij) {
          const double l = ltab[(jj + 1) * 3 + (ii + 1)];
          const double slope = (hij - h[ijk]) / l;
          if (slope > smax) {
            smax = slope;
            r = ijk;
            len = l;
          }
        }
      }
    }
  }
  rec[ij] = r;
  length[ij] = len;
}

// Donor lists by gathering: the receiver of any node is one of its 3x3
// (wrapped) neighbours, so node k's donors are the neighbours d with
// rec[d]==k and d!=k.  They are emitted in ascending node order, which is the
// order of the reference's scatter loop over ij=1..nn.
__global__ void k_find_donors(Bounds bd, const int* __restrict__ rec, int* __restrict__ ndon,
                              int* __restrict__ don) {
  const int nx = bd.nx, ny = bd.ny;
  const int nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    int cand[8];
    int nc = 0;
    // Distinct neighbours in the wrapped 3x3 block (rows/columns that fall off
    // a non-cyclic edge do not exist).
    int rows[3], nr = 0, cols[3], ncl = 0;
    for (int d = -1; d <= 1; ++d) {
      int jj = j + d;
      if (jj < 0) { if (!bd.ycyc) continue; jj += ny; }
      if (jj >= ny) { if (!bd.ycyc) continue; jj -= ny; }
      bool dup = false;
      for (int t = 0; t < nr; ++t) dup |= rows[t] == jj;
      if (!dup) rows[nr++] = jj;
    }
    for (int d = -1; d <= 1; ++d) {
      int ii = i + d;
      if (ii < 0) { if (!bd.xcyc) continue; ii += nx; }
      if (ii >= nx) { if (!bd.xcyc) continue; ii -= nx; }
      bool dup = false;
      for (int t = 0; t < ncl; ++t) dup |= cols[t] == ii;
      if (!dup) cols[ncl++] = ii;
    }
    for (int a = 0; a < nr; ++a)
      for (int c = 0; c < ncl; ++c) {
        const int q = cols[c] + rows[a] * nx;
        if (q != k && rec[q] == k && nc < 8) cand[nc++] = q;
      }
    // insertion sort (<= 8 entries)
    for (int x = 1; x < nc; ++x) {
      const int v = cand[x];
      int y = x - 1;
      while (y >= 0 && cand[y] > v) { cand[y + 1] = cand[y]; --y; }
      cand[y + 1] = v;
    }
    ndon[k] = nc;
    for (int x = 0; x < 8; ++x) don[(size_t)k * 8 + x] = x < nc ? cand[x] : -1;
  }
}

// root flags (rec==self) for the compaction of the ascending root list
__global__ void k_root_flags(int nn, const int* __restrict__ rec, int* __restrict__ flag) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    flag[k] = rec[k] == k ? 1 : 0;
}

// After an exclusive scan of the root flags: rank of each root and root list.
__global__ void k_root_list(int nn, const int* __restrict__ rec, const int* __restrict__ scan,
                            int* __restrict__ roots, int* __restrict__ root_rank) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x)
    if (rec[k] == k) {
      roots[scan[k]] = k;
      root_rank[k] = scan[k];
    }
}

// Euler tour successor, packed with the event weight for list ranking:
// entry = (succ << 32) | weight, succ = 0xffffffff at the end of the tour.
__global__ void k_euler_tour(int nn, const int* __restrict__ rec, const int* __restrict__ ndon,
                             const int* __restrict__ don, const int* __restrict__ roots,
                             const int* __restrict__ root_rank, const int* __restrict__ nroots,
                             unsigned long long* __restrict__ lst) {
  const unsigned END = 0xffffffffu;
  const int R = *nroots;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int nd = ndon[k];
    const unsigned se = nd > 0 ? 2u * (unsigned)don[(size_t)k * 8] : 2u * (unsigned)k + 1u;
    unsigned sx;
    const int r = rec[k];
    if (r != k) {
      int s = 0;
      const int pnd = ndon[r];
      while (s < pnd && don[(size_t)r * 8 + s] != k) ++s;
      sx = (s + 1 < pnd) ? 2u * (unsigned)don[(size_t)r * 8 + s + 1] : 2u * (unsigned)r + 1u;
    } else {
      const int rr = root_rank[k];
      sx = (rr + 1 < R) ? 2u * (unsigned)roots[rr + 1] : END;
    }
    lst[2 * (size_t)k] = ((unsigned long long)se << 32) | 1ull;
    lst[2 * (size_t)k + 1] = ((unsigned long long)sx << 32) | 0ull;
  }
}

// One Wyllie pointer-jumping round: value += value(succ); succ = succ(succ).
__global__ void k_list_rank_round(size_t n, const unsigned long long* __restrict__ in,
                                  unsigned long long* __restrict__ out) {
  const unsigned END = 0xffffffffu;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long cur = in[e];
    const unsigned nx = (unsigned)(cur >> 32);
    if (nx == END) {
      out[e] = cur;
    } else {
      const unsigned long long nb = in[nx];
      const unsigned v = (unsigned)cur + (unsigned)nb;
      out[e] = (nb & 0xffffffff00000000ull) | (unsigned long long)v;
    }
  }
}

// ---- list ranking by sublist walks (long lists) --------------------------------
// Entry e's result is the suffix sum of the weights from e to its list's end.
// Splitters: every kRankStride-th entry and every head (an entry that is no
// entry's successor).  Each splitter walks its sublist up to the next
// splitter, writing for every entry (splitter id << 32 | prefix), the prefix
// being the weights before the entry within the sublist, and records
// (next splitter id << 32 | sublist total).  Pointer jumping over the
// splitters then gives each its suffix sum V, and entry e's result is
// V(its splitter) - its prefix.  O(n) work against Wyllie's O(n log n).

// flags every entry that is some entry's successor; leaves the unused head
// slots of the splitter list inert (no successor, weight 0)
__global__ void k_rank_pred(size_t n, const unsigned long long* __restrict__ lst, unsigned char* __restrict__ pred,
                            unsigned long long* __restrict__ spl, size_t s0) {
  const unsigned END = 0xffffffffu;
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  for (size_t e = tid; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const unsigned nx = (unsigned)(lst[e] >> 32);
    if (nx != END && nx < n) pred[nx] = 1;
  }
  if (tid < (size_t)kRankMaxHeads) spl[s0 + tid] = (unsigned long long)END << 32;
}

// one sublist walk from splitter entry e with splitter id `id`; every step is
// one dependent load, and the walk ends within n steps
__device__ void rank_walk(size_t n, const unsigned long long* __restrict__ lst, unsigned long long* __restrict__ sub,
                          unsigned long long* __restrict__ spl, size_t e, unsigned id, int* err) {
  const unsigned END = 0xffffffffu;
  unsigned pre = 0, nid = END;
  size_t x = e;
  for (size_t steps = 0;; ++steps) {
    const unsigned long long cur = lst[x];
    sub[x] = ((unsigned long long)id << 32) | pre;
    pre += (unsigned)cur;
    const unsigned nx = (unsigned)(cur >> 32);
    if (nx == END) break;
    if (nx >= n || steps >= n) {  // not a list
      atomicExch(err, DEV_STACK_ERROR);
      break;
    }
    if (nx % kRankStride == 0) {
      nid = nx / kRankStride;
      break;
    }
    x = nx;
  }
  spl[id] = ((unsigned long long)nid << 32) | pre;
}

// thread t: the splitter at t*kRankStride, then any head among the next
// kRankStride - 1 entries (one 16-byte load of their flags)
__global__ void k_rank_walk(size_t n, size_t s0, const unsigned long long* __restrict__ lst,
                            const unsigned char* __restrict__ pred, unsigned long long* __restrict__ sub,
                            unsigned long long* __restrict__ spl, unsigned* nheads, int* err) {
  static_assert(kRankStride == 16, "one uint4 of flags per splitter");
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < s0; t += (size_t)gridDim.x * blockDim.x) {
    const size_t base = t * kRankStride;
    rank_walk(n, lst, sub, spl, base, (unsigned)t, err);
    const uint4 f4 = *reinterpret_cast<const uint4*>(pred + base);
    const unsigned f[4] = {f4.x, f4.y, f4.z, f4.w};
#pragma unroll
    for (int j = 1; j < kRankStride; ++j) {
      const size_t e = base + j;
      if (e >= n || ((f[j >> 2] >> (8 * (j & 3))) & 0xffu) != 0u) continue;
      const unsigned h = atomicAdd(nheads, 1u);
      if (h >= (unsigned)kRankMaxHeads) {
        atomicExch(err, DEV_OVERFLOW);
        continue;
      }
      rank_walk(n, lst, sub, spl, e, (unsigned)(s0 + h), err);
    }
  }
}

__global__ void k_rank_final(size_t n, const unsigned long long* __restrict__ sub,
                             const unsigned long long* __restrict__ vs, unsigned long long* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long s = sub[e];
    out[e] = (unsigned long long)((unsigned)vs[s >> 32] - (unsigned)s);
  }
}

// preorder position and subtree size from the ranks of the enter/exit events
__global__ void k_stack_from_ranks(int nn, const unsigned long long* __restrict__ lst,
                                   int* __restrict__ pos, int* __restrict__ size, int* __restrict__ stack,
                                   int* __restrict__ err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const unsigned re = (unsigned)lst[2 * (size_t)k];
    const unsigned rx = (unsigned)lst[2 * (size_t)k + 1];
    const int p = nn - (int)re;
    if (p < 0 || p >= nn) { atomicExch(err, DEV_STACK_ERROR); continue; }
    pos[k] = p;
    size[k] = (int)(re - rx);
    stack[p] = k;
  }
}

// ---------------------------------------------------------------------------
// host launchers

void launch_uplift(Ctx& c) {
  k_uplift<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, c.dt, c.u, c.h, c.b);
  c.count_launch();
}

void launch_find_receiver(Ctx& c, const double* h, int* rec, double* length) {
  dim3 blk(32, 8);
  dim3 grd((c.nx + 31) / 32, (c.ny + 7) / 8);
  k_find_receiver<<<grd, blk, 0, c.stream>>>(c.bd, h, c.ltab, rec, length);
  c.count_launch();
}

void launch_find_donors(Ctx& c, const int* rec, int* ndon, int* don) {
  k_find_donors<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, rec, ndon, don);
  c.count_launch();
}

// Wyllie list ranking over `n` packed entries, ping-ponging between a and b.
// Returns the buffer that holds the result.
static unsigned long long* wyllie(Ctx& c, size_t n, unsigned long long* a, unsigned long long* b) {
  int rounds = 1;
  while (((size_t)1 << rounds) < n) ++rounds;
  for (int r = 0; r < rounds; ++r) {
    k_list_rank_round<<<grid1d(n), kBlock, 0, c.stream>>>(n, a, b);
    c.count_launch();
    std::swap(a, b);
  }
  return a;
}

// Suffix sums of `n` packed entries (succ << 32 | weight) in the low words of
// the returned buffer (a or b).  Lists of 2^16 entries or more are ranked by
// sublist walks (n <= 2*nn: the scratch is sized for that), shorter ones by
// Wyllie alone.
unsigned long long* list_rank(Ctx& c, size_t n, unsigned long long* a, unsigned long long* b) {
  if (n < ((size_t)1 << 16) || n > 2 * (size_t)c.nn) return wyllie(c, n, a, b);
  const size_t s0 = (n + kRankStride - 1) / kRankStride;
  cudaMemsetAsync(c.s_rank_pred, 0, s0 * kRankStride, c.stream);  // whole flag words past n too
  cudaMemsetAsync(c.s_rank_nheads, 0, sizeof(unsigned), c.stream);
  k_rank_pred<<<grid1d(n), kBlock, 0, c.stream>>>(n, a, c.s_rank_pred, c.s_rank_sa, s0);
  k_rank_walk<<<(unsigned)((s0 + 127) / 128), 128, 0, c.stream>>>(n, s0, a, c.s_rank_pred, b, c.s_rank_sa,
                                                                    c.s_rank_nheads, c.d_err);
  c.count_launch(2);
  const unsigned long long* v = wyllie(c, s0 + kRankMaxHeads, c.s_rank_sa, c.s_rank_sb);
  k_rank_final<<<grid1d(n), kBlock, 0, c.stream>>>(n, b, v, a);
  c.count_launch();
  return a;
}

// Builds ndon/don/stack(+pos,size) for the receiver array `rec`.
void build_stack(Ctx& c, const int* rec, int* ndon, int* don, int* stack, int* pos, int* size) {
  const int nn = c.nn;
  launch_find_donors(c, rec, ndon, don);
  k_root_flags<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, rec, c.s_flag);
  c.count_launch();
  exclusive_scan_int(c, c.s_flag, c.s_scan, nn + 1);  // s_scan[nn] = number of roots
  k_root_list<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, rec, c.s_scan, c.s_roots, c.s_root_rank);
  c.count_launch();
  k_euler_tour<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, rec, ndon, don, c.s_roots, c.s_root_rank,
                                                     c.s_scan + nn, c.s_list_a);
  c.count_launch();
  unsigned long long* res = list_rank(c, 2 * (size_t)nn, c.s_list_a, c.s_list_b);
  k_stack_from_ranks<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, res, pos, size, stack, c.d_err);
  c.count_launch();
}

}  // namespace fsb
