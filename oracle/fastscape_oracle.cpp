// Oracle: a single-threaded CPU restatement of fastscapelib-fortran's continental
// time step (FastScape_Execute_Step with marine, stratigraphy and flexure
// switched off; advection runs when velocities are set).
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that tests/, the smoke
// test and the benchmark's cpu_baseline leg compare the CUDA library against.
// It is never part of the product path.
//
// The reference cannot be compiled in this environment (it is Fortran and no
// Fortran compiler is installed), so parity with the reference itself is
// UNPINNED: this restatement follows the Fortran statement by statement and
// cites, for every routine, the reference file:line it restates, and the
// tests check every stage of it against a second, independent literal
// transliteration in Python (tests/fortran_literal.py, tests/test_oracle.py).
// Fortran semantics that matter for bit-exactness are kept:
//   * 1-based node numbering ij = i + (j-1)*nx internally; the C-ABI exports
//     0-based node ids (value - 1).
//   * no fused multiply-add (build with -ffp-contract=off), left-to-right
//     evaluation of products/quotients, x**2 == x*x, x**y == pow(x, y).
//   * the Numerical Recipes quicksort (loc_min_3_indexx) is reproduced exactly,
//     including its non-stable treatment of equal keys.
//   * the Kahn/LIFO multiple-flow stack of find_mult_rec is reproduced exactly.
//
// Build: g++ -O2 -ffp-contract=off -fPIC -shared (see oracle/Makefile).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cfloat>
#include <string>
#include <vector>
#include <algorithm>

namespace {

typedef std::vector<double> dvec;
typedef std::vector<int> ivec;

// Diagnostic of the n = 1.5 powers (off unless fso_pow15_diag(1) is called):
// every multiple-flow Newton solve is repeated with x**1.5 and x**0.5 taken
// as x*sqrt(x) and sqrt(x), the GPU's evaluation, on the same inputs; the
// reference's result is kept and the differences are counted.
struct Pow15Diag {
  bool on = false;
  long long solves = 0, iters = 0, iter_diff = 0, h_diff = 0, max_iters = 0, long_solves = 0;
  double max_rel = 0.0;
} g_pow15;

// Fortran tiny(1d0)
const double TINY = DBL_MIN;

struct LocMinDebug {
  // captured from the last LocalMinima call (all 1-based like the reference)
  int nbasins = 0, basin0 = 0, nconn = 0, tree_size = 0, nlocmin_before = 0, nlocmin_after = 0;
  ivec basins, outlets;
  ivec conn_b1, conn_b2, conn_n1, conn_n2;   // as produced by connect_basins
  dvec conn_w;
  ivec sort_id;                              // loc_min_3_indexx permutation
  ivec tree;                                 // Kruskal acceptance order
  ivec ob1, ob2, on1, on2;                   // after order_tree (oriented)
  ivec rec_pre, stack_pre;                   // receivers/stack entering LocalMinima
  dvec length_pre;
};

struct Ctx {
  int nx = 0, ny = 0, nn = 0, step = 0;
  bool setup_done = false;
  int ibc = 1111;
  int i1 = 1, i2 = 1, j1 = 1, j2 = 1;
  bool xcyc = false, ycyc = false;
  std::vector<char> bc;  // bounds_bc, 1-based
  double xl = 0, yl = 0, dt = 0, kfsed = 0, m = 0, n = 0, kdsed = 0, g1 = 0, g2 = 0, p = 0;
  double sealevel = 0;
  bool runSPL = false, runDiffusion = false, runUplift = false, runMarine = false;
  bool sfd = false;
  int nGS = 0;
  dvec h, u, length, a, erate, etot, catchv, catch0, b, precip, kf, kd, sedflux, g, pmfd;
  dvec lake_depth, hwater;
  dvec vx, vy;  // advection velocities (SetV, ctx:616-632)
  bool runAdvect = false;
  ivec stack, ndon, rec, don;  // don(8,nn): don[(ij-1)*8 + k-1]
  ivec mnrec, mstack, mrec;
  dvec mwrec, mlrec;
  LocMinDebug dbg;
  std::string err;
};

Ctx g_ctx;
Ctx* C = &g_ctx;

inline int& DON(ivec& d, int k, int ij) { return d[(size_t)(ij - 1) * 8 + (k - 1)]; }

// ---------------------------------------------------------------------------
// SetBC  -- src/FastScape_ctx.f90:565-593.  write(cbc,'(i4)') then digit tests.
void set_bc(Ctx& c, int jbc) {
  c.ibc = jbc;
  char cbc[8];
  if (jbc > 9999 || jbc < -999) std::strcpy(cbc, "****");
  else std::snprintf(cbc, sizeof cbc, "%4d", jbc);
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  std::fill(c.bc.begin(), c.bc.end(), 0);
  c.i1 = 1; c.i2 = nx; c.j1 = 1; c.j2 = ny;
  if (cbc[3] == '1') c.i1 = 2;
  if (cbc[1] == '1') c.i2 = nx - 1;
  if (cbc[0] == '1') c.j1 = 2;
  if (cbc[2] == '1') c.j2 = ny - 1;
  if (cbc[3] == '1') for (int ij = 1; ij <= nn; ij += nx) c.bc[ij] = 1;
  if (cbc[1] == '1') for (int ij = nx; ij <= nn; ij += nx) c.bc[ij] = 1;
  if (cbc[0] == '1') for (int ij = 1; ij <= nx; ++ij) c.bc[ij] = 1;
  if (cbc[2] == '1') for (int ij = nx * (ny - 1) + 1; ij <= nn; ++ij) c.bc[ij] = 1;
  c.xcyc = (cbc[3] != '1' && cbc[1] != '1');
  c.ycyc = (cbc[0] != '1' && cbc[2] != '1');
}

// ---------------------------------------------------------------------------
// find_receiver -- src/FlowRouting.f90:302-362
void find_receiver(const dvec& h, int nx, int ny, double dx, double dy, ivec& rec, dvec& length,
                   int i1, int i2, int j1, int j2, bool xc, bool yc) {
  const int nn = nx * ny;
  for (int ij = 1; ij <= nn; ++ij) { rec[ij] = ij; length[ij] = 0.0; }
  for (int j = j1; j <= j2; ++j)
    for (int i = i1; i <= i2; ++i) {
      const int ij = i + (j - 1) * nx;
      double smax = TINY;
      for (int jj = -1; jj <= 1; ++jj)
        for (int ii = -1; ii <= 1; ++ii) {
          int iii = i + ii;
          if (iii < 1 && xc) iii += nx;
          iii = std::max(iii, 1);
          if (iii > nx && xc) iii -= nx;
          iii = std::min(iii, nx);
          int jjj = j + jj;
          if (jjj < 1 && yc) jjj += ny;
          jjj = std::max(jjj, 1);
          if (jjj > ny && yc) jjj -= ny;
          jjj = std::min(jjj, ny);
          const int ijk = iii + (jjj - 1) * nx;
          if (ijk != ij) {
            const double ax = dx * ii, ay = dy * jj;
            const double l = std::sqrt(ax * ax + ay * ay);
            const double slope = (h[ij] - h[ijk]) / l;
            if (slope > smax) { smax = slope; rec[ij] = ijk; length[ij] = l; }
          }
        }
    }
}

// find_donor -- src/FlowRouting.f90:366-389 (and loc_min_3_find_donors, LocalMinima.f90:881-900)
void find_donor(const ivec& rec, int nn, ivec& ndon, ivec& don) {
  std::fill(ndon.begin(), ndon.end(), 0);
  for (int ij = 1; ij <= nn; ++ij)
    if (rec[ij] != ij) {
      const int ijk = rec[ij];
      ndon[ijk] += 1;
      DON(don, ndon[ijk], ijk) = ij;
    }
}

// find_stack + find_stack_recursively -- src/FlowRouting.f90:393-443
// (and loc_min_3_find_stack, LocalMinima.f90:904-923,1050-1067).  The
// recursion is unrolled onto an explicit stack of (node, next donor slot);
// the visiting order is identical: roots ascending, donors in slot order.
void find_stack(const ivec& rec, ivec& don, const ivec& ndon, int nn, ivec& stack,
                const dvec* catch0, dvec* catchv) {
  int nstack = 0;
  if (catchv) *catchv = *catch0;
  std::vector<std::pair<int, int>> st;
  st.reserve(1024);
  for (int ij = 1; ij <= nn; ++ij) {
    if (rec[ij] != ij) continue;
    stack[++nstack] = ij;
    st.clear();
    st.push_back({ij, 1});
    while (!st.empty()) {
      auto& top = st.back();
      const int node = top.first;
      if (top.second > ndon[node]) { st.pop_back(); continue; }
      const int ijk = DON(don, top.second, node);
      top.second += 1;
      stack[++nstack] = ijk;
      if (catchv) (*catchv)[ijk] = (*catchv)[node];
      st.push_back({ijk, 1});
    }
  }
}

// ---------------------------------------------------------------------------
// LocalMinima pieces -- src/LocalMinima.f90

// compute_basins -- LocalMinima.f90:136-169
int compute_basins(const ivec& stack, const ivec& rec, ivec& basins, ivec& outlets, int n) {
  int ib = 0;
  for (int i = 1; i <= n; ++i) {
    const int is = stack[i];
    if (rec[is] == is) { ++ib; outlets[ib] = is; }
    basins[is] = ib;
  }
  return ib;
}

// connect_basins -- LocalMinima.f90:173-329.  The conn arrays grow as needed;
// the reference writes past nconn_max=6*nbasins silently, which is reported.
void connect_basins(int nbasins, const ivec& basins, const ivec& outlets, const ivec& rec,
                    const ivec& stack, const std::vector<char>& active_nodes, const dvec& h,
                    int nx, int ny, int& basin0, ivec& cb1, ivec& cb2, ivec& cn1, ivec& cn2,
                    dvec& cw) {
  const int n = nx * ny;
  static const int ii[8] = {-1, 1, 0, 0, -1, 1, -1, 1};
  static const int jj[8] = {0, 0, -1, 1, -1, -1, 1, 1};
  basin0 = -1;
  int ibasin = 1;
  ivec conn_pos(nbasins + 1, -1), conn_pos_used;
  conn_pos_used.reserve(64);
  bool active = false;
  cb1.clear(); cb2.clear(); cn1.clear(); cn2.clear(); cw.clear();
  for (int iis = 1; iis <= n; ++iis) {
    const int is = stack[iis];
    const int irec = rec[is];
    if (irec == is) {
      ibasin = basins[is];
      active = active_nodes[is] != 0;
      for (int u : conn_pos_used) conn_pos[u] = -1;
      conn_pos_used.clear();
      if (!active) {
        if (basin0 == -1) basin0 = ibasin;
        else {
          cb1.push_back(basin0); cb2.push_back(ibasin);
          cn1.push_back(-1); cn2.push_back(-1); cw.push_back(-1.e10);
        }
      }
    }
    if (active) {
      const int i = (is - 1) % nx + 1;
      const int j = (is - 1) / nx + 1;
      for (int k = 0; k < 8; ++k) {
        const int ki = i + ii[k], kj = j + jj[k];
        if (ki < 1 || ki > nx || kj < 1 || kj > ny) continue;
        const int inb = (kj - 1) * nx + ki;
        const int nbb = basins[inb];
        const int nbo = outlets[nbb];
        if (ibasin >= nbb && active_nodes[nbo]) continue;
        const double weight = std::max(h[is], h[inb]);
        const int ci = conn_pos[nbb];
        if (ci == -1) {
          cb1.push_back(ibasin); cb2.push_back(nbb);
          cn1.push_back(is); cn2.push_back(inb); cw.push_back(weight);
          conn_pos[nbb] = (int)cw.size();  // 1-based iconn
          conn_pos_used.push_back(nbb);
        } else if (weight < cw[ci - 1]) {
          cn1[ci - 1] = is; cn2[ci - 1] = inb; cw[ci - 1] = weight;
        }
      }
    }
  }
}

}  // namespace

// loc_min_3_indexx -- LocalMinima.f90:947-1046: Numerical Recipes index
// quicksort (median of three, Hoare partition, insertion sort below M=7).
// arr and indx are 1-based (arr[1..n]); exported for tests as well.
static int nr_indexx(int n, const double* arr, int* indx) {
  const int M = 7, NSTACK = 50;
  int istack[NSTACK + 1];
  for (int j = 1; j <= n; ++j) indx[j] = j;
  int jstack = 0, l = 1, ir = n;
  for (;;) {
    if (ir - l < M) {
      for (int j = l + 1; j <= ir; ++j) {
        const int indxt = indx[j];
        const double a = arr[indxt];
        int i;
        for (i = j - 1; i >= 1; --i) {
          if (arr[indx[i]] <= a) break;
          indx[i + 1] = indx[i];
        }
        if (i < 1) i = 0;
        indx[i + 1] = indxt;
      }
      if (jstack == 0) return 0;
      ir = istack[jstack];
      l = istack[jstack - 1];
      jstack -= 2;
    } else {
      const int k = (l + ir) / 2;
      std::swap(indx[k], indx[l + 1]);
      if (arr[indx[l + 1]] > arr[indx[ir]]) std::swap(indx[l + 1], indx[ir]);
      if (arr[indx[l]] > arr[indx[ir]]) std::swap(indx[l], indx[ir]);
      if (arr[indx[l + 1]] > arr[indx[l]]) std::swap(indx[l + 1], indx[l]);
      int i = l + 1, j = ir;
      const int indxt = indx[l];
      const double a = arr[indxt];
      for (;;) {
        do { ++i; } while (arr[indx[i]] < a);
        do { --j; } while (arr[indx[j]] > a);
        if (j < i) break;
        std::swap(indx[i], indx[j]);
      }
      indx[l] = indx[j];
      indx[j] = indxt;
      jstack += 2;
      if (jstack > NSTACK) return -1;  // reference: stop 'NSTACK too small'
      if (ir - i + 1 >= j - l) {
        istack[jstack] = ir;
        istack[jstack - 1] = i;
        ir = j - 1;
      } else {
        istack[jstack] = j - 1;
        istack[jstack - 1] = l;
        l = i;
      }
    }
  }
}

namespace {

// UnionFind / DoUnion -- LocalMinima.f90:766-832 (only parent(x) is compressed)
int uf_find(int x, ivec& parent) {
  int xp = x, xc = -1000;
  while (xc != xp) { xc = xp; xp = parent[xc]; }
  parent[x] = xc;
  return xc;
}
void uf_union(int x, int y, ivec& parent, ivec& rank) {
  const int xr = uf_find(x, parent), yr = uf_find(y, parent);
  if (xr != yr) {
    if (rank[xr] < rank[yr]) parent[xr] = yr;
    else {
      parent[yr] = xr;
      if (rank[xr] == rank[yr]) rank[xr] += 1;
    }
  }
}

// mst_kruskal -- LocalMinima.f90:333-385
bool mst_kruskal(const dvec& w, const ivec& cb1, const ivec& cb2, int nbasins, ivec& sort_id,
                 ivec& tree) {
  const int nconn = (int)w.size();
  sort_id.assign(nconn + 1, 0);
  if (nr_indexx(nconn, w.data() - 1, sort_id.data()) != 0) return false;
  ivec parent(nbasins + 1), rank(nbasins + 1, 0);
  for (int i = 1; i <= nbasins; ++i) parent[i] = i;
  tree.clear();
  for (int e = 1; e <= nconn; ++e) {
    const int eid = sort_id[e];
    const int b0 = cb1[eid - 1], b1 = cb2[eid - 1];
    const int f0 = uf_find(b0, parent), f1 = uf_find(b1, parent);
    if (f0 != f1) {
      tree.push_back(eid);
      uf_union(b0, b1, parent, rank);
    }
  }
  return true;
}

// order_tree -- LocalMinima.f90:389-533 (continuous_flow=.false. branch)
void order_tree(ivec& n1, ivec& n2, ivec& p1, ivec& p2, int num_nodes, int root, const ivec& tree) {
  const int ntree = (int)tree.size();
  ivec csize(num_nodes + 1, 0), cptr(num_nodes + 1, 0);
  for (int t = 0; t < ntree; ++t) {
    const int i = tree[t];
    csize[n1[i - 1]] += 1;
    csize[n2[i - 1]] += 1;
  }
  cptr[1] = 1;
  for (int i = 2; i <= num_nodes; ++i) {
    cptr[i] = cptr[i - 1] + csize[i - 1];
    csize[i - 1] = 0;
  }
  const int adj_size = cptr[num_nodes] + csize[num_nodes] - 1;
  csize[num_nodes] = 0;
  ivec adj(std::max(adj_size, 0) + 1, 0);
  for (int t = 0; t < ntree; ++t) {
    const int i = tree[t];
    const int a = n1[i - 1], b = n2[i - 1];
    adj[cptr[a] + csize[a]] = i;
    adj[cptr[b] + csize[b]] = i;
    csize[a] += 1;
    csize[b] += 1;
  }
  std::vector<std::pair<int, int>> st;
  st.push_back({root, root});
  while (!st.empty()) {
    const int node = st.back().first, parent = st.back().second;
    st.pop_back();
    for (int i = cptr[node]; i <= cptr[node] + csize[node] - 1; ++i) {
      const int e = adj[i] - 1;
      if (n1[e] == parent && node != parent) {
        // edge towards the parent: already oriented
      } else {
        if (node != n1[e]) {
          std::swap(n1[e], n2[e]);
          std::swap(p1[e], p2[e]);
        }
        st.push_back({n2[e], node});
      }
    }
  }
}

// correct_receivers_v2 -- LocalMinima.f90:601-662
void correct_receivers_v2(ivec& rec, dvec& dist, const ivec& outlets, const ivec& cb2,
                          const ivec& cn1, const ivec& cn2, const ivec& tree, int nx, double dx,
                          double dy) {
  for (size_t t = 0; t < tree.size(); ++t) {
    const int i = tree[t] - 1;
    const int node_to = cn1[i];
    const int node_from = cn2[i];
    if (node_from == -1) continue;
    const int outlet_from = outlets[cb2[i]];
    int next_node = rec[node_from];
    int cur_node = node_from;
    double previous_dist = dist[node_from];
    rec[node_from] = node_to;
    const double ddx = dx * (double)(((node_from - 1) % nx) - ((node_to - 1) % nx));
    const double ddy = dy * (double)(((node_from - 1) / nx) - ((node_to - 1) / nx));
    dist[node_from] = std::sqrt(ddx * ddx + ddy * ddy);
    while (cur_node != outlet_from) {
      const int rcv_next = rec[next_node];
      rec[next_node] = cur_node;
      const double tmp = previous_dist;
      previous_dist = dist[next_node];
      dist[next_node] = tmp;
      cur_node = next_node;
      next_node = rcv_next;
    }
  }
}

// LocalMinima -- LocalMinima.f90:1-132 (continuous_flow=.false., continuous_flow_v2=.true.)
bool local_minima(Ctx& c, double dx, double dy) {
  const int nn = c.nn, nx = c.nx, ny = c.ny;
  LocMinDebug& d = c.dbg;
  d.rec_pre = c.rec; d.stack_pre = c.stack; d.length_pre = c.length;
  d.basins.assign(nn + 1, 0);
  d.outlets.assign(nn + 1, 0);
  const int nbasins = compute_basins(c.stack, c.rec, d.basins, d.outlets, nn);
  d.nbasins = nbasins;
  std::vector<char> active(nn + 1, 0);
  for (int k = 1; k <= nn; ++k) active[k] = !c.bc[k];
  int nloc = 0;
  for (int k = 1; k <= nn; ++k) if (c.rec[k] == k && active[k]) ++nloc;
  d.nlocmin_before = nloc;
  connect_basins(nbasins, d.basins, d.outlets, c.rec, c.stack, active, c.h, nx, ny, d.basin0,
                 d.conn_b1, d.conn_b2, d.conn_n1, d.conn_n2, d.conn_w);
  d.nconn = (int)d.conn_w.size();
  if (d.nconn > 6 * nbasins) {
    c.err = "connect_basins: nconn exceeds nconn_max=6*nbasins (reference overflows here)";
    return false;
  }
  if (!mst_kruskal(d.conn_w, d.conn_b1, d.conn_b2, nbasins, d.sort_id, d.tree)) {
    c.err = "NSTACK too small in loc_min_3_indexx";
    return false;
  }
  d.tree_size = (int)d.tree.size();
  d.ob1 = d.conn_b1; d.ob2 = d.conn_b2; d.on1 = d.conn_n1; d.on2 = d.conn_n2;
  if (d.basin0 < 1) {
    c.err = "LocalMinima: no basin on a fixed boundary (the reference indexes out of bounds)";
    return false;
  }
  order_tree(d.ob1, d.ob2, d.on1, d.on2, nbasins, d.basin0, d.tree);
  correct_receivers_v2(c.rec, c.length, d.outlets, d.ob2, d.on1, d.on2, d.tree, nx, dx, dy);
  nloc = 0;
  for (int k = 1; k <= nn; ++k) if (c.rec[k] == k && active[k]) ++nloc;
  d.nlocmin_after = nloc;
  find_donor(c.rec, nn, c.ndon, c.don);
  find_stack(c.rec, c.don, c.ndon, nn, c.stack, nullptr, nullptr);
  return true;
}

// find_mult_rec -- src/FlowRouting.f90:147-298
bool find_mult_rec(Ctx& c, double dx, double dy) {
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  dvec& h0 = c.hwater;  // "water = h0"
  h0 = c.h;
  const double deltah = 1.e-8;
  for (int i = 1; i <= nn; ++i) {
    const int ijk = c.stack[i];
    const int ijr = c.rec[ijk];
    if (ijr != 0 && h0[ijr] > h0[ijk]) h0[ijk] = h0[ijr] + deltah;
  }
  std::fill(c.mnrec.begin(), c.mnrec.end(), 0);
  std::fill(c.mwrec.begin(), c.mwrec.end(), 0.0);
  for (int j = c.j1; j <= c.j2; ++j)
    for (int i = c.i1; i <= c.i2; ++i) {
      const int ij = (j - 1) * nx + i;
      for (int jj = -1; jj <= 1; ++jj) {
        int jjj = j + jj;
        if (jjj < 1 && c.ycyc) jjj += ny;
        jjj = std::max(jjj, 1);
        if (jjj > ny && c.ycyc) jjj -= ny;
        jjj = std::min(jjj, ny);
        for (int ii = -1; ii <= 1; ++ii) {
          int iii = i + ii;
          if (iii < 1 && c.xcyc) iii += nx;
          iii = std::max(iii, 1);
          if (iii > nx && c.xcyc) iii -= nx;
          iii = std::min(iii, nx);
          const int ijk = (jjj - 1) * nx + iii;
          if (h0[ij] > h0[ijk]) {
            const int k = ++c.mnrec[ij];
            c.mrec[(size_t)(ij - 1) * 8 + k - 1] = ijk;
            const double ax = ii * dx, ay = jj * dy;
            const double l = std::sqrt(ax * ax + ay * ay);
            c.mlrec[(size_t)(ij - 1) * 8 + k - 1] = l;
            c.mwrec[(size_t)(ij - 1) * 8 + k - 1] = (h0[ij] - h0[ijk]) / l;
          }
        }
      }
    }
  for (int ij = 1; ij <= nn; ++ij) {
    double* w = &c.mwrec[(size_t)(ij - 1) * 8];
    const int nr = c.mnrec[ij];
    if (c.p < 0.0) {
      double slope = 0.0;
      if (nr != 0) {
        double s = 0.0;
        for (int k = 0; k < nr; ++k) s += w[k];
        slope = (double)(float)(s / nr);  // real(...)
      }
      c.pmfd[ij] = (double)0.5f + (double)0.6f * slope;
    }
    for (int k = 0; k < nr; ++k) w[k] = std::pow(w[k], c.pmfd[ij]);
    double sumw = 0.0;
    for (int k = 0; k < nr; ++k) sumw += w[k];
    for (int k = 0; k < nr; ++k) w[k] = w[k] / sumw;
  }
  ivec ndon(nn + 1, 0), vis(nn + 1, 0), parse(nn + 1, 0);
  for (int ij = 1; ij <= nn; ++ij)
    for (int k = 0; k < c.mnrec[ij]; ++k) ndon[c.mrec[(size_t)(ij - 1) * 8 + k]] += 1;
  int nparse = 0, nstack = 0;
  std::fill(c.mstack.begin(), c.mstack.end(), 0);
  for (int ij = 1; ij <= nn; ++ij) {
    if (ndon[ij] == 0) parse[++nparse] = ij;
    while (nparse > 0) {
      const int ijn = parse[nparse--];
      c.mstack[++nstack] = ijn;
      for (int k = 0; k < c.mnrec[ijn]; ++k) {
        const int ijr = c.mrec[(size_t)(ijn - 1) * 8 + k];
        vis[ijr] += 1;
        if (vis[ijr] == ndon[ijr]) parse[++nparse] = ijr;
      }
    }
  }
  if (nstack != nn) { c.err = "error in stack"; return false; }
  return true;
}

// FlowRouting -- FlowRouting.f90:3-39 ; FlowRoutingSingleFlowDirection -- :43-93
bool flow_routing(Ctx& c) {
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  find_receiver(c.h, c.nx, c.ny, dx, dy, c.rec, c.length, c.i1, c.i2, c.j1, c.j2, c.xcyc, c.ycyc);
  find_donor(c.rec, c.nn, c.ndon, c.don);
  find_stack(c.rec, c.don, c.ndon, c.nn, c.stack, &c.catch0, &c.catchv);
  if (!local_minima(c, dx, dy)) return false;
  if (c.sfd) {
    c.hwater = c.h;
    const double deltah = 1.e-8;
    for (int i = 1; i <= c.nn; ++i) {
      const int ijk = c.stack[i], ijr = c.rec[ijk];
      if (ijr != 0 && c.hwater[ijr] > c.hwater[ijk]) c.hwater[ijk] = c.hwater[ijr] + deltah;
    }
  } else {
    if (!find_mult_rec(c, dx, dy)) return false;
  }
  for (int i = 1; i <= c.nn; ++i) c.lake_depth[i] = c.hwater[i] - c.h[i];
  return true;
}

// FlowAccumulation -- FlowRouting.f90:97-119 ; ...SingleFlowDirection -- :123-143
void flow_accumulation(Ctx& c) {
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  for (int i = 1; i <= c.nn; ++i) c.a[i] = dx * dy * c.precip[i];
  if (c.sfd) {
    for (int ij = c.nn; ij >= 1; --ij) {
      const int ijk = c.stack[ij];
      c.a[c.rec[ijk]] = c.a[c.rec[ijk]] + c.a[ijk];
    }
  } else {
    for (int ij = 1; ij <= c.nn; ++ij) {
      const int ijk = c.mstack[ij];
      for (int k = 0; k < c.mnrec[ijk]; ++k) {
        const int r = c.mrec[(size_t)(ijk - 1) * 8 + k];
        c.a[r] = c.a[r] + c.a[ijk] * c.mwrec[(size_t)(ijk - 1) * 8 + k];
      }
    }
  }
}

// StreamPowerLaw -- StreamPowerLaw.f90:3-206 ; ...SingleFlowDirection -- :210-400
// water(:) is fresh allocatable storage in the reference (never initialised);
// reads of entries not yet written in the current sweep see 0.0 here.
void stream_power_law(Ctx& c) {
  const int nn = c.nn;
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  dvec ht(nn + 1), kfint(nn + 1), dh(nn + 1), hp(nn + 1), elev(nn + 1);
  dvec water(nn + 1, 0.0), lwv(nn + 1, 0.0), lsed(nn + 1, 0.0);
  ivec lsill(nn + 1, 0);
  if (c.g1 >= 0.0) {
    for (int i = 1; i <= nn; ++i) {
      c.g[i] = c.g1;
      if (c.g2 > 0.0 && (c.h[i] - c.b[i]) > 1.0) c.g[i] = c.g2;
    }
  }
  for (int i = 1; i <= nn; ++i) {
    kfint[i] = c.kf[i];
    if (c.kfsed > 0.0 && (c.h[i] - c.b[i]) > 1.0) kfint[i] = c.kfsed;
  }
  double mx = 0.0;
  for (int i = 1; i <= nn; ++i) mx = std::max(mx, std::fabs(c.h[i]));
  const double tol = 1.e-4 * (mx + 1.0);
  double err = 2.0 * tol;
  ht = c.h;
  c.nGS = 0;
  double gmax = -DBL_MAX;
  for (int i = 1; i <= nn; ++i) gmax = std::max(gmax, c.g[i]);
  const bool n_is_one = std::fabs(c.n - 1.0) < TINY;
  while (err > tol && c.nGS < 99) {
    c.nGS += 1;
    hp = c.h;
    for (int i = 1; i <= nn; ++i) dh[i] = ht[i] - hp[i];
    if (c.sfd) {
      for (int ij = nn; ij >= 1; --ij) {
        const int ijk = c.stack[ij], ijr = c.rec[ijk];
        if (ijr != ijk) {
          dh[ijk] = dh[ijk] - (ht[ijk] - hp[ijk]);
          if (lsill[ijk] == ijk) lsed[ijk] = (dh[ijk] <= 0.0) ? 0.0 : dh[ijk];
          dh[ijk] = dh[ijk] + (ht[ijk] - hp[ijk]);
          dh[ijr] = dh[ijr] + dh[ijk];
        } else {
          lsed[ijk] = dh[ijk];
        }
      }
    } else {
      for (int ij = 1; ij <= nn; ++ij) {
        const int ijk = c.mstack[ij], ijr1 = c.rec[ijk];
        if (ijr1 != ijk) {
          dh[ijk] = dh[ijk] - (ht[ijk] - hp[ijk]);
          if (lsill[ijk] == ijk) lsed[ijk] = (dh[ijk] <= 0.0) ? 0.0 : dh[ijk];
          dh[ijk] = dh[ijk] + (ht[ijk] - hp[ijk]);
          for (int k = 0; k < c.mnrec[ijk]; ++k) {
            const int r = c.mrec[(size_t)(ijk - 1) * 8 + k];
            dh[r] = dh[r] + dh[ijk] * c.mwrec[(size_t)(ijk - 1) * 8 + k];
          }
        } else {
          lsed[ijk] = dh[ijk];
        }
      }
    }
    for (int i = 1; i <= nn; ++i)
      elev[i] = c.bc[i] ? ht[i] : ht[i] + (dh[i] - (ht[i] - hp[i])) * c.g[i] * dx * dy / c.a[i];

    auto visit = [&](int ijk) {
      const int ijr = c.rec[ijk];
      if (ijr == ijk) {
        water[ijk] = ht[ijk];
        lsill[ijk] = ijk;
        lwv[ijk] = 0.0;
        return;
      }
      const double w_rcv = water[ijr];
      if (elev[ijk] > w_rcv) {
        if (c.sfd) {
          if (n_is_one) {
            if (c.h[ijk] >= c.sealevel || !c.runMarine) {
              double f = elev[ijk], df = 1.0;
              const double fact = kfint[ijk] * c.dt * std::pow(c.a[ijk], c.m) / c.length[ijk];
              f = f + fact * c.h[ijr];
              df = df + fact;
              c.h[ijk] = f / df;
            }
          } else {
            if (ht[ijk] >= c.sealevel || !c.runMarine) {
              const double omega = 0.875 / c.n, tolp = 1.e-3;
              double errp = 2.0 * tolp;
              const double h0 = elev[ijk];
              while (errp > tolp) {
                double f = c.h[ijk] - h0, df = 1.0;
                if (ht[ijk] > ht[ijr]) {
                  const double fact = kfint[ijk] * c.dt * std::pow(c.a[ijk], c.m) / std::pow(c.length[ijk], c.n);
                  const double x = std::max(0.0, c.h[ijk] - c.h[ijr]);
                  f = f + fact * std::pow(x, c.n);
                  df = df + fact * c.n * std::pow(x, c.n - 1.0);
                }
                const double hn = c.h[ijk] - f / df;
                errp = std::fabs(hn - c.h[ijk]);
                c.h[ijk] = c.h[ijk] * (1.0 - omega) + hn * omega;
              }
            }
          }
        } else {
          const int nr = c.mnrec[ijk];
          const int* mr = &c.mrec[(size_t)(ijk - 1) * 8];
          const double* mw = &c.mwrec[(size_t)(ijk - 1) * 8];
          const double* ml = &c.mlrec[(size_t)(ijk - 1) * 8];
          if (nr > 0) {
            if (n_is_one) {
              if (c.h[ijk] >= c.sealevel || !c.runMarine) {
                double f = elev[ijk], df = 1.0;
                for (int k = 0; k < nr; ++k)
                  if (ht[ijk] >= ht[mr[k]]) {
                    const double fact = kfint[ijk] * c.dt * std::pow(c.a[ijk] * mw[k], c.m) / ml[k];
                    f = f + fact * c.h[mr[k]];
                    df = df + fact;
                  }
                c.h[ijk] = f / df;
              }
            } else {
              if (ht[ijk] >= c.sealevel || !c.runMarine) {
                const double omega = 0.875 / c.n, tolp = 1.e-3;
                double errp = 2.0 * tolp;
                const double h0 = elev[ijk];
                const double hstart = c.h[ijk];
                long long it = 0;
                while (errp > tolp) {
                  ++it;
                  double f = c.h[ijk] - h0, df = 1.0;
                  for (int k = 0; k < nr; ++k)
                    if (ht[ijk] > ht[mr[k]]) {
                      const double fact = kfint[ijk] * c.dt * std::pow(c.a[ijk] * mw[k], c.m) / std::pow(ml[k], c.n);
                      const double x = std::max(0.0, c.h[ijk] - c.h[mr[k]]);
                      f = f + fact * std::pow(x, c.n);
                      df = df + fact * c.n * std::pow(x, c.n - 1.0);
                    }
                  const double hn = c.h[ijk] - f / df;
                  errp = std::fabs(hn - c.h[ijk]);
                  c.h[ijk] = c.h[ijk] * (1.0 - omega) + hn * omega;
                }
                if (g_pow15.on && c.n == 1.5) {  // the same solve with x*sqrt(x), sqrt(x)
                  double hb = hstart, eb = 2.0 * tolp;
                  long long itb = 0;
                  while (eb > tolp && itb < 100000) {
                    ++itb;
                    double f = hb - h0, df = 1.0;
                    for (int k = 0; k < nr; ++k)
                      if (ht[ijk] > ht[mr[k]]) {
                        const double fact = kfint[ijk] * c.dt * std::pow(c.a[ijk] * mw[k], c.m) / std::pow(ml[k], c.n);
                        const double x = std::max(0.0, hb - c.h[mr[k]]);
                        const double r = std::sqrt(x);
                        f = f + fact * (x * r);
                        df = df + fact * c.n * r;
                      }
                    const double hn = hb - f / df;
                    eb = std::fabs(hn - hb);
                    hb = hb * (1.0 - omega) + hn * omega;
                  }
                  g_pow15.solves += 1;
                  g_pow15.iters += it;
                  if (it > g_pow15.max_iters) g_pow15.max_iters = it;
                  g_pow15.long_solves += it > 20;
                  g_pow15.iter_diff += itb != it;
                  g_pow15.h_diff += hb != c.h[ijk];
                  const double rel = std::fabs(hb - c.h[ijk]) / std::max(std::fabs(c.h[ijk]), 1.0);
                  if (rel > g_pow15.max_rel) g_pow15.max_rel = rel;
                }
              }
            }
          }
        }
        lsill[ijk] = ijk;
        lwv[ijk] = 0.0;
        if (c.h[ijk] < w_rcv) c.h[ijk] = w_rcv;
      } else {
        c.h[ijk] = elev[ijk];
        lsill[ijk] = lsill[ijr];
        if (lsill[ijk] != 0) lwv[lsill[ijk]] = lwv[lsill[ijk]] + (w_rcv - c.h[ijk]);
      }
      water[ijk] = std::max(w_rcv, c.h[ijk]);
    };
    if (c.sfd) for (int ij = 1; ij <= nn; ++ij) visit(c.stack[ij]);
    else for (int ij = nn; ij >= 1; --ij) visit(c.mstack[ij]);

    double s = 0.0;
    for (int i = 1; i <= nn; ++i) { const double d = c.h[i] - hp[i]; s += d * d; }
    err = std::sqrt(s / nn);
    if (gmax < TINY) err = 0.0;
  }
  for (int i = 1; i <= nn; ++i) c.b[i] = std::min(c.h[i], c.b[i]);
  for (int ij = 1; ij <= nn; ++ij) {
    const int ls = lsill[ij];
    if (ls != 0 && lwv[ls] > 0.0)
      c.h[ij] = c.h[ij] + std::max(0.0, std::min(lsed[ls], lwv[ls])) / lwv[ls] * (water[ij] - c.h[ij]);
  }
  for (int i = 1; i <= nn; ++i) {
    c.etot[i] = c.etot[i] + ht[i] - c.h[i];
    c.erate[i] = (ht[i] - c.h[i]) / c.dt;
    c.sedflux[i] = ht[i] - c.h[i];
  }
}

// tridag -- Diffusion.f90:164-202 (Numerical Recipes Thomas algorithm); arrays 1-based
bool tridag(const double* a, const double* b, const double* cc, const double* r, double* u, int n,
            double* gam) {
  if (b[1] == 0.0) return false;
  double bet = b[1];
  u[1] = r[1] / bet;
  for (int j = 2; j <= n; ++j) {
    gam[j] = cc[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    if (bet == 0.0) return false;
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 1; j >= 1; --j) u[j] = u[j] - gam[j + 1] * u[j + 1];
  return true;
}

// Diffusion -- Diffusion.f90:1-160 (ADI)
bool diffusion(Ctx& c) {
  const int nx = c.nx, ny = c.ny;
  char cbc[8];
  if (c.ibc > 9999 || c.ibc < -999) std::strcpy(cbc, "****");
  else std::snprintf(cbc, sizeof cbc, "%4d", c.ibc);
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  const double dt2 = c.dt / 2.0, dx2 = dx * dx, dy2 = dy * dy;
  auto I = [nx](int i, int j) { return (size_t)(j - 1) * nx + i; };  // 1-based 2-D -> 1-based 1-D
  dvec zint(c.nn + 1), kdint(c.nn + 1), zintp(c.nn + 1);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      const size_t ij = I(i, j);
      zint[ij] = c.h[ij];
      kdint[ij] = c.kd[ij];
      if (c.kdsed > 0.0 && (c.h[ij] - c.b[ij]) > 1.e-6) kdint[ij] = c.kdsed;
    }
  zintp = zint;
  auto K = [&](int i, int j) { return kdint[I(i, j)]; };
  auto fx = [&](double k1, double k2) { return (k1 + k2) / 2.0 * dt2 / dx2; };
  auto fy = [&](double k1, double k2) { return (k1 + k2) / 2.0 * dt2 / dy2; };
  {
    dvec f(nx + 1, 0.0), diag(nx + 1, 0.0), sup(nx + 1, 0.0), inf(nx + 1, 0.0), res(nx + 1, 0.0), gam(nx + 1, 0.0);
    for (int j = 2; j <= ny - 1; ++j) {
      for (int i = 2; i <= nx - 1; ++i) {
        const double fxp = fx(K(i + 1, j), K(i, j));
        const double fxm = fx(K(i - 1, j), K(i, j));
        const double fyp = fy(K(i, j + 1), K(i, j));
        const double fym = fy(K(i, j - 1), K(i, j));
        diag[i] = 1.0 + fxp + fxm;
        sup[i] = -fxp;
        inf[i] = -fxm;
        f[i] = zintp[I(i, j)] + fyp * zintp[I(i, j + 1)] - (fyp + fym) * zintp[I(i, j)] + fym * zintp[I(i, j - 1)];
      }
      if (cbc[3] == '1') {
        diag[1] = 1.0; sup[1] = 0.0; f[1] = zintp[I(1, j)];
      } else {
        const double fxp = fx(K(2, j), K(1, j));
        const double fyp = fy(K(1, j + 1), K(1, j));
        const double fym = fy(K(1, j - 1), K(1, j));
        diag[1] = 1.0 + fxp;
        sup[1] = -fxp;
        f[1] = zintp[I(1, j)] + fyp * zintp[I(1, j + 1)] - (fyp + fym) * zintp[I(1, j)] + fym * zintp[I(1, j - 1)];
      }
      if (cbc[1] == '1') {
        diag[nx] = 1.0; inf[nx] = 0.0; f[nx] = zintp[I(nx, j)];
      } else {
        const double fxm = fx(K(nx - 1, j), K(nx, j));
        const double fyp = fy(K(nx, j + 1), K(nx, j));
        const double fym = fy(K(nx, j - 1), K(nx, j));
        diag[nx] = 1.0 + fxm;
        inf[nx] = -fxm;
        f[nx] = zintp[I(nx, j)] + fyp * zintp[I(nx, j + 1)] - (fyp + fym) * zintp[I(nx, j)] + fym * zintp[I(nx, j - 1)];
      }
      if (!tridag(inf.data(), diag.data(), sup.data(), f.data(), res.data(), nx, gam.data())) return false;
      for (int i = 1; i <= nx; ++i) zint[I(i, j)] = res[i];
    }
  }
  {
    dvec f(ny + 1, 0.0), diag(ny + 1, 0.0), sup(ny + 1, 0.0), inf(ny + 1, 0.0), res(ny + 1, 0.0), gam(ny + 1, 0.0);
    // after "do j=2,ny-1" the loop variable is ny (Diffusion.f90:98,114)
    const int jq = std::max(2, ny);
    for (int i = 2; i <= nx - 1; ++i) {
      for (int j = 2; j <= ny - 1; ++j) {
        const double fxp = fx(K(i + 1, j), K(i, j));
        const double fxm = fx(K(i - 1, j), K(i, j));
        const double fyp = fy(K(i, j + 1), K(i, j));
        const double fym = fy(K(i, j - 1), K(i, j));
        diag[j] = 1.0 + fyp + fym;
        sup[j] = -fyp;
        inf[j] = -fym;
        f[j] = zint[I(i, j)] + fxp * zint[I(i + 1, j)] - (fxp + fxm) * zint[I(i, j)] + fxm * zint[I(i - 1, j)];
      }
      if (cbc[0] == '1') {
        diag[1] = 1.0; sup[1] = 0.0; f[1] = zint[I(i, 1)];
      } else {
        const double fxp = fx(K(i + 1, 1), K(i, jq));
        const double fxm = fx(K(i - 1, 1), K(i, 1));
        const double fyp = fy(K(i, 2), K(i, 1));
        diag[1] = 1.0 + fyp;
        sup[1] = -fyp;
        f[1] = zint[I(i, 1)] + fxp * zint[I(i + 1, 1)] - (fxp + fxm) * zint[I(i, 1)] + fxm * zint[I(i - 1, 1)];
      }
      if (cbc[2] == '1') {
        diag[ny] = 1.0; inf[ny] = 0.0; f[ny] = zint[I(i, ny)];
      } else {
        const double fxp = fx(K(i + 1, ny), K(i, ny));
        const double fxm = fx(K(i - 1, ny), K(i, ny));
        const double fym = fy(K(i, ny - 1), K(i, ny));
        diag[ny] = 1.0 + fym;
        inf[ny] = -fym;
        f[ny] = zint[I(i, ny)] + fxp * zint[I(i + 1, ny)] - (fxp + fxm) * zint[I(i, ny)] + fxm * zint[I(i - 1, ny)];
      }
      if (!tridag(inf.data(), diag.data(), sup.data(), f.data(), res.data(), ny, gam.data())) return false;
      for (int j = 1; j <= ny; ++j) zintp[I(i, j)] = res[j];
    }
  }
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      const size_t ij = I(i, j);
      c.etot[ij] = c.etot[ij] + c.h[ij] - zintp[ij];
      c.erate[ij] = c.erate[ij] + (c.h[ij] - zintp[ij]) / c.dt;
      c.h[ij] = zintp[ij];
    }
  for (int i = 1; i <= c.nn; ++i) c.b[i] = std::min(c.h[i], c.b[i]);
  return true;
}

void alloc_all(Ctx& c) {
  const size_t n1 = (size_t)c.nn + 1, n8 = (size_t)c.nn * 8;
  for (dvec* v : {&c.h, &c.u, &c.length, &c.a, &c.erate, &c.etot, &c.catchv, &c.catch0, &c.b,
                  &c.precip, &c.kf, &c.kd, &c.sedflux, &c.g, &c.pmfd, &c.lake_depth, &c.hwater,
                  &c.vx, &c.vy})
    v->assign(n1, 0.0);
  for (ivec* v : {&c.stack, &c.ndon, &c.rec, &c.mnrec, &c.mstack}) v->assign(n1, 0);
  c.don.assign(n8, 0);
  c.mrec.assign(n8, 0);
  c.mwrec.assign(n8, 0.0);
  c.mlrec.assign(n8, 0.0);
  c.bc.assign(n1, 0);
}

// Advect -- Advect.f90:1-103: implicit upwind x-pass over every row, then
// y-pass over every column, tridag for h, b and etot; then b = min(b, h).
bool advect(Ctx& c) {
  const int nx = c.nx, ny = c.ny;
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  auto I = [nx](int i, int j) { return (size_t)(j - 1) * nx + i; };
  auto pass = [&](int n, int lines, double d, const dvec& v, auto idx) {
    dvec diag(n + 1), sup(n + 1), inf(n + 1), rhs(n + 1), res(n + 1), gam(n + 1);
    for (int l = 1; l <= lines; ++l) {
      for (int t = 1; t <= n; ++t) {
        diag[t] = 1.0; sup[t] = 0.0; inf[t] = 0.0;
        const double vv = v[idx(t, l)];
        if (vv > 0.0) {
          diag[t] = 1.0 + vv * c.dt / d;
          inf[t] = -(vv * c.dt / d);
        } else if (vv < 0.0) {
          diag[t] = 1.0 - vv * c.dt / d;
          sup[t] = vv * c.dt / d;
        }
      }
      sup[1] = 0.0; diag[1] = 1.0; diag[n] = 1.0; inf[n] = 0.0;
      for (dvec* f : {&c.h, &c.b, &c.etot}) {
        for (int t = 1; t <= n; ++t) rhs[t] = (*f)[idx(t, l)];
        if (!tridag(inf.data(), diag.data(), sup.data(), rhs.data(), res.data(), n, gam.data())) return false;
        for (int t = 1; t <= n; ++t) (*f)[idx(t, l)] = res[t];
      }
    }
    return true;
  };
  if (!pass(nx, ny, dx, c.vx, [&](int t, int l) { return I(t, l); })) return false;
  if (!pass(ny, nx, dy, c.vy, [&](int t, int l) { return I(l, t); })) return false;
  for (int i = 1; i <= c.nn; ++i) c.b[i] = std::min(c.b[i], c.h[i]);
  return true;
}

// Stand-in for gfortran's random_number in SetUp (FastScape_ctx.f90:82,94): a
// fixed xorshift stream.  Every use of the API overwrites h with init_h, and
// catch0 only feeds copy_catchment, so the stream itself does not matter.
double lcg_uniform(uint64_t& s) {
  s ^= s << 13; s ^= s >> 7; s ^= s << 17;
  return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

int fail(const char* msg) { C->err = msg; return 1; }

}  // namespace

// ===========================================================================
// C-ABI (0-based node ids on export).  Mirrors the fastscape_* API of
// src/FastScape_api.f90.  Every function returns 0 on success; on failure it
// returns non-zero and fso_last_error() describes the problem where the
// reference would `stop`.
extern "C" {

const char* fso_last_error() { return C->err.c_str(); }

// FastScape_Init -- FastScape_api.f90:146 -> FastScape_ctx.f90:40-53
// on != 0: start the n = 1.5 power diagnostic (counters reset); out (may be
// null) receives solves, total iterations, solves whose iteration count
// differs, solves whose result differs, the largest relative difference,
// the most iterations of one solve and the solves of more than 20 iterations
int fso_pow15_diag(int on, double* out) {
  if (out) {
    out[5] = (double)g_pow15.max_iters;
    out[6] = (double)g_pow15.long_solves;
    out[0] = (double)g_pow15.solves;
    out[1] = (double)g_pow15.iters;
    out[2] = (double)g_pow15.iter_diff;
    out[3] = (double)g_pow15.h_diff;
    out[4] = g_pow15.max_rel;
  }
  if (on >= 0) {
    g_pow15 = Pow15Diag();
    g_pow15.on = on != 0;
  }
  return 0;
}

int fso_init() {
  g_ctx = Ctx();
  return 0;
}

// FastScape_Set_NX_NY -- api:475 -> ctx:397
int fso_set_nx_ny(int nx, int ny) { C->nx = nx; C->ny = ny; return 0; }

// FastScape_Setup -- api:160 -> ctx:57-113
int fso_setup() {
  Ctx& c = *C;
  if (c.nx == 0) return fail("FastScapeSetup - You need to set nx first");
  if (c.ny == 0) return fail("FastScapeSetup - You need to set ny first");
  c.nn = c.nx * c.ny;
  alloc_all(c);
  set_bc(c, 1111);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (int i = 1; i <= c.nn; ++i) c.h[i] = lcg_uniform(s);
  for (int i = 1; i <= c.nx; ++i) c.h[i] = 0.0;
  for (int i = c.nx * (c.ny - 1) + 1; i <= c.nn; ++i) c.h[i] = 0.0;
  for (int i = 1; i <= c.nn; i += c.nx) c.h[i] = 0.0;
  for (int i = c.nx; i <= c.nn; i += c.nx) c.h[i] = 0.0;
  c.b = c.h;
  std::fill(c.precip.begin(), c.precip.end(), 1.0);
  std::fill(c.pmfd.begin(), c.pmfd.end(), 1.0);
  for (int i = 1; i <= c.nn; ++i) c.catch0[i] = lcg_uniform(s);
  c.sealevel = 0.0;
  c.runSPL = c.runDiffusion = c.runMarine = c.runUplift = false;
  c.nGS = 0;
  c.setup_done = true;
  return 0;
}

int fso_destroy() { g_ctx = Ctx(); return 0; }

int fso_set_xl_yl(double xl, double yl) { C->xl = xl; C->yl = yl; return 0; }
int fso_set_dt(double dt) { C->dt = dt; return 0; }

// FastScape_Set_Erosional_Parameters -- api:523-536 -> ctx:423-450
int fso_set_erosional_parameters(const double* kf, double kfsed, double m, double n,
                                 const double* kd, double kdsed, double g1, double g2, double p) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("set_erosional_parameters - You need to run SetUp first");
  c.runSPL = true;
  for (int i = 1; i <= c.nn; ++i) { c.kf[i] = kf[i - 1]; c.kd[i] = kd[i - 1]; }
  c.kfsed = kfsed; c.m = m; c.n = n; c.kdsed = kdsed; c.g1 = g1; c.g2 = g2; c.p = p;
  for (int i = 1; i <= c.nn; ++i) c.pmfd[i] = p;
  c.sfd = false;
  if (p < -1.5) { c.sfd = true; c.p = 1.0; }
  double kdmax = -DBL_MAX;
  for (int i = 1; i <= c.nn; ++i) kdmax = std::max(kdmax, c.kd[i]);
  if (kdmax > TINY || kdsed > TINY) c.runDiffusion = true;
  return 0;
}

// FastScape_Set_BC -- api:602 -> ctx:565-593
int fso_set_bc(int jbc) {
  if (!C->setup_done) return fail("set_bc - You need to run SetUp first");
  set_bc(*C, jbc);
  return 0;
}

// FastScape_Set_U -- api:618 -> ctx:597-612
// FastScape_Set_V -- api:634 -> ctx:616-632
int fso_set_v(const double* ux, const double* uy) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("SetV - You need to run SetUp first");
  for (int i = 1; i <= c.nn; ++i) { c.vx[i] = ux[i - 1]; c.vy[i] = uy[i - 1]; }
  c.runAdvect = true;
  return 0;
}

int fso_set_u(const double* up) {
  if (!C->setup_done) return fail("set_u - You need to run SetUp first");
  C->runUplift = true;
  for (int i = 1; i <= C->nn; ++i) C->u[i] = up[i - 1];
  return 0;
}

// FastScape_Init_H -- api:267 -> ctx:339-350
int fso_init_h(const double* hp) {
  if (!C->setup_done) return fail("InitH - You need to run SetUp first");
  for (int i = 1; i <= C->nn; ++i) C->h[i] = hp[i - 1];
  C->b = C->h;
  return 0;
}

int fso_set_h(const double* hp) {  // ctx:636-644
  if (!C->setup_done) return fail("SetH - You need to run SetUp first");
  for (int i = 1; i <= C->nn; ++i) C->h[i] = hp[i - 1];
  return 0;
}
int fso_set_basement(const double* bp) {  // ctx:680-688
  if (!C->setup_done) return fail("SetBasement - You need to run SetUp first");
  for (int i = 1; i <= C->nn; ++i) C->b[i] = bp[i - 1];
  return 0;
}
int fso_set_precip(const double* pp) {  // ctx:648-656
  if (!C->setup_done) return fail("SetPrecip - You need to run SetUp first");
  for (int i = 1; i <= C->nn; ++i) C->precip[i] = pp[i - 1];
  return 0;
}
int fso_reset_cumulative_erosion() {  // ctx:368-374
  std::fill(C->etot.begin(), C->etot.end(), 0.0);
  return 0;
}

// FastScape_Execute_Step -- api:201-263 (advection, marine, strati are off)
int fso_execute_step() {
  Ctx& c = *C;
  if (!c.setup_done) return fail("Execute_Step - You need to run SetUp first");
  c.err.clear();
  if (c.runAdvect && !advect(c)) return fail("tridag failed");  // Advect first (api:209-214)
  if (c.runUplift) {  // Uplift.f90:9-10
    for (int i = 1; i <= c.nn; ++i) {
      const double du = c.u[i] * c.dt;
      c.h[i] = c.h[i] + du;
      c.b[i] = c.b[i] + du;
    }
  }
  if (c.runSPL) {
    if (!flow_routing(c)) return 1;
    flow_accumulation(c);
    stream_power_law(c);
  }
  if (c.runDiffusion) {
    if (!diffusion(c)) return fail("tridag failed");
  }
  c.step += 1;
  return 0;
}

// Diffusion.f90:1-160 alone on the current state (test entry: compares an
// ADI step on its own, e.g. on grids the full step refuses)
int fso_diffusion_only() {
  Ctx& c = *C;
  if (!c.setup_done) return fail("Diffusion - You need to run SetUp first");
  if (!diffusion(c)) return fail("tridag failed");
  return 0;
}

int fso_get_step(int* s) { *s = C->step; return 0; }
int fso_get_sizes(int* nx, int* ny) { *nx = C->nx; *ny = C->ny; return 0; }
int fso_get_nn() { return C->nn; }

// Copy-outs (ctx:158-335).  field ids:
// 0 h, 1 basement, 2 total erosion, 3 drainage area, 4 erosion rate, 5 lake depth,
// 6 length, 7 hwater, 8 sedflux, 9 catchment, 10 u, 11 precip, 12 kf, 13 kd
int fso_copy_double(int field, double* out) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("Copy - You need to run SetUp first");
  const dvec* src = nullptr;
  switch (field) {
    case 0: src = &c.h; break;
    case 1: src = &c.b; break;
    case 2: src = &c.etot; break;
    case 3: src = &c.a; break;
    case 4: src = &c.erate; break;
    case 5: src = &c.lake_depth; break;
    case 6: src = &c.length; break;
    case 7: src = &c.hwater; break;
    case 8: src = &c.sedflux; break;
    case 9: src = &c.catchv; break;
    case 10: src = &c.u; break;
    case 11: src = &c.precip; break;
    case 12: src = &c.kf; break;
    case 13: src = &c.kd; break;
    default: return fail("unknown field");
  }
  std::memcpy(out, src->data() + 1, sizeof(double) * c.nn);
  return 0;
}

// integer fields (0-based node ids): 0 rec, 1 ndon, 2 stack, 3 mnrec, 4 mstack,
// 5 basins (1-based basin ids as in the reference), 6 rec before LocalMinima,
// 7 stack before LocalMinima
int fso_copy_int(int field, int* out) {
  Ctx& c = *C;
  const ivec* src = nullptr;
  int sub = 1;
  switch (field) {
    case 0: src = &c.rec; break;
    case 1: src = &c.ndon; sub = 0; break;
    case 2: src = &c.stack; break;
    case 3: src = &c.mnrec; sub = 0; break;
    case 4: src = &c.mstack; break;
    case 5: src = &c.dbg.basins; sub = 0; break;
    case 6: src = &c.dbg.rec_pre; break;
    case 7: src = &c.dbg.stack_pre; break;
    default: return fail("unknown field");
  }
  if ((int)src->size() < c.nn + 1) return fail("field not computed yet");
  for (int i = 0; i < c.nn; ++i) out[i] = (*src)[i + 1] - sub;
  return 0;
}

// don / mrec as int32[nn][8] (0-based ids; unused slots -1), mwrec/mlrec as f64[nn][8]
int fso_copy_slots(int field, void* out) {
  Ctx& c = *C;
  const int nn = c.nn;
  if (field == 0 || field == 1) {
    const ivec& s = field == 0 ? c.don : c.mrec;
    const ivec& cnt = field == 0 ? c.ndon : c.mnrec;
    int* o = (int*)out;
    for (int ij = 1; ij <= nn; ++ij)
      for (int k = 0; k < 8; ++k)
        o[(size_t)(ij - 1) * 8 + k] = k < cnt[ij] ? s[(size_t)(ij - 1) * 8 + k] - 1 : -1;
    return 0;
  }
  if (field == 2 || field == 3) {
    const dvec& s = field == 2 ? c.mwrec : c.mlrec;
    double* o = (double*)out;
    for (int ij = 1; ij <= nn; ++ij)
      for (int k = 0; k < 8; ++k)
        o[(size_t)(ij - 1) * 8 + k] = k < c.mnrec[ij] ? s[(size_t)(ij - 1) * 8 + k] : 0.0;
    return 0;
  }
  return fail("unknown slot field");
}

// LocalMinima capture of the last step: counts, then arrays.
int fso_locmin_counts(int* out6) {
  const LocMinDebug& d = C->dbg;
  out6[0] = d.nbasins; out6[1] = d.basin0; out6[2] = d.nconn; out6[3] = d.tree_size;
  out6[4] = d.nlocmin_before; out6[5] = d.nlocmin_after;
  return 0;
}
// conn list as produced by connect_basins: b1,b2 (1-based basin ids), n1,n2
// (0-based node ids, -1 for virtual edges), weights; sort_id (0-based edge
// ids), tree (0-based edge ids, Kruskal order) and oriented (b1,b2,n1,n2).
int fso_locmin_arrays(int* b1, int* b2, int* n1, int* n2, double* w, int* sort_id, int* tree,
                      int* ob1, int* ob2, int* on1, int* on2) {
  const LocMinDebug& d = C->dbg;
  for (int i = 0; i < d.nconn; ++i) {
    b1[i] = d.conn_b1[i]; b2[i] = d.conn_b2[i];
    n1[i] = d.conn_n1[i] < 0 ? -1 : d.conn_n1[i] - 1;
    n2[i] = d.conn_n2[i] < 0 ? -1 : d.conn_n2[i] - 1;
    w[i] = d.conn_w[i];
    sort_id[i] = d.sort_id[i + 1] - 1;
    ob1[i] = d.ob1[i]; ob2[i] = d.ob2[i];
    on1[i] = d.on1[i] < 0 ? -1 : d.on1[i] - 1;
    on2[i] = d.on2[i] < 0 ? -1 : d.on2[i] - 1;
  }
  for (int i = 0; i < d.tree_size; ++i) tree[i] = d.tree[i] - 1;
  return 0;
}

int fso_get_ngs() { return C->nGS; }

// Standalone restatement of loc_min_3_indexx for known-answer tests:
// arr[0..n-1] -> indx[0..n-1] (0-based).  Returns -1 on NSTACK overflow.
int fso_indexx(int n, const double* arr, int* indx) {
  std::vector<int> ix(n + 1);
  const int rc = nr_indexx(n, arr - 1, ix.data());
  for (int i = 0; i < n; ++i) indx[i] = ix[i + 1] - 1;
  return rc;
}

// ---- derived fields and diagnostics of the API ----------------------------

// CopyChi -- FastScape_ctx.f90:228-251: along the stack, chi(k) = chi(rec(k))
// + (a0/a(k))**(m/n) * length(k) where a(k) > a0 = dx*dy*10, else 0.
int fso_copy_chi(double* out) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("CopyChi - You need to run SetUp first");
  dvec chi(c.nn + 1, 0.0);
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  const double a0 = dx * dy * 10.0;
  for (int ij = 1; ij <= c.nn; ++ij) {
    const int ijk = c.stack[ij];
    if (ijk < 1) continue;  // stack not built yet (no step run)
    if (c.a[ijk] > a0) chi[ijk] = chi[c.rec[ijk]] + std::pow(a0 / c.a[ijk], c.m / c.n) * c.length[ijk];
  }
  for (int i = 0; i < c.nn; ++i) out[i] = chi[i + 1];
  return 0;
}

// slope -- TerrainDerivatives.f90:3-35 (degrees; 0 on the grid's edges)
int fso_copy_slope(double* out) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("CopySlope - You need to run SetUp first");
  const int nx = c.nx, ny = c.ny;
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  const double con = 45.0 / std::atan(1.0);
  const dvec& h = c.h;
  dvec s(c.nn + 1, 0.0);
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      const int ij = i + (j - 1) * nx;
      const int ia = ij + nx - 1, ib = ia + 1, ic = ib + 1, id = ij - 1, iff = ij + 1;
      const int ig = ij - nx - 1, ih = ig + 1, ii = ih + 1;
      const double dzdx = ((h[ic] + 2.0 * h[iff] + h[ii]) - (h[ia] + 2.0 * h[id] + h[ig])) / 8.0 / dx;
      const double dzdy = ((h[ig] + 2.0 * h[ih] + h[ii]) - (h[ia] + 2.0 * h[ib] + h[ic])) / 8.0 / dy;
      s[ij] = dzdx * dzdx + dzdy * dzdy;
      if (s[ij] > DBL_MIN) s[ij] = std::atan(std::sqrt(s[ij])) * con;
    }
  for (int i = 0; i < c.nn; ++i) out[i] = s[i + 1];
  return 0;
}

// curvature -- TerrainDerivatives.f90:39-74 (0 on the grid's edges)
int fso_copy_curvature(double* out) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("CopyCurvature - You need to run SetUp first");
  const int nx = c.nx, ny = c.ny;
  const double dx = c.xl / (nx - 1), dy = c.yl / (ny - 1);
  const dvec& h = c.h;
  dvec cv(c.nn + 1, 0.0);
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      const int ij = i + (j - 1) * nx;
      const int i1 = ij + nx - 1, i2 = i1 + 1, i3 = i2 + 1, i4 = ij - 1, i5 = ij, i6 = ij + 1;
      const int i7 = ij - nx - 1, i8 = i7 + 1, i9 = i8 + 1;
      const double a = (h[i1] + h[i3] + h[i4] + h[i6] + h[i7] + h[i9]) / dx / dx / 12.0 -
                       (h[i2] + h[i5] + h[i8]) / dx / dx / 6.0;
      const double b = (h[i1] + h[i2] + h[i3] + h[i7] + h[i8] + h[i9]) / dy / dy / 12.0 -
                       (h[i4] + h[i5] + h[i6]) / dy / dy / 6.0;
      const double cc = (h[i3] + h[i7] - h[i1] - h[i9]) / dx / dy / 4.0;
      const double d = (h[i3] + h[i6] + h[i9] - h[i1] - h[i4] - h[i7]) / dx / 6.0;
      const double e = (h[i1] + h[i2] + h[i3] - h[i7] - h[i8] - h[i9]) / dy / 6.0;
      cv[ij] = 1.0 + d * d + e * e;
      if (cv[ij] > DBL_MIN)
        cv[ij] = (a * (1.0 + e * e) + b * (1.0 + d * d) - cc * d * e) / std::pow(cv[ij], 3.0 / 2.0);
    }
  for (int i = 0; i < c.nn; ++i) out[i] = cv[i + 1];
  return 0;
}

// compute_fluxes -- FastScape_ctx.f90:843-886: out3 = tectonic, erosion and
// boundary fluxes (erate accumulated downstream with max(0, .) at each node).
int fso_get_fluxes(double* out3) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("GetFluxes - You need to run SetUp first");
  const double surf = c.xl * c.yl / (c.nx - 1) / (c.ny - 1);
  double su = 0.0, se = 0.0;
  for (int i = 1; i <= c.nn; ++i) { su += c.u[i]; se += c.erate[i]; }
  dvec flux = c.erate;
  if (c.step > 0) {
    if (c.sfd) {
      for (int ij = c.nn; ij >= 1; --ij) {
        const int ijk = c.stack[ij];
        flux[ijk] = std::max(0.0, flux[ijk]);
        flux[c.rec[ijk]] = flux[c.rec[ijk]] + flux[ijk];
      }
    } else {
      for (int ij = 1; ij <= c.nn; ++ij) {
        const int ijk = c.mstack[ij];
        flux[ijk] = std::max(0.0, flux[ijk]);
        for (int k = 1; k <= c.mnrec[ijk]; ++k) {
          const size_t o = (size_t)(ijk - 1) * 8 + (k - 1);
          flux[c.mrec[o]] = flux[c.mrec[o]] + flux[ijk] * c.mwrec[o];
        }
      }
    }
  }
  double sb = 0.0;
  for (int i = 1; i <= c.nn; ++i) if (c.bc[i]) sb += flux[i];
  out3[0] = su * surf;
  out3[1] = se * surf;
  out3[2] = sb * surf;
  return 0;
}

// Make_VTK -- FastScape_ctx.f90:692-777 with -fconvert=big-endian
// (CMakeLists.txt:49): legacy binary VTK, big-endian float32.
static void put_be(FILE* fp, double v) {
  const float f = (float)v;
  unsigned u;
  std::memcpy(&u, &f, 4);
  const unsigned char b[4] = {(unsigned char)(u >> 24), (unsigned char)(u >> 16), (unsigned char)(u >> 8),
                              (unsigned char)u};
  std::fwrite(b, 1, 4, fp);
}
static bool vtk_one(const Ctx& c, const std::string& path, const dvec* z, double zc, const char* name,
                    const dvec* s1, double s1c, const double* f, double vex) {
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  const double dx = c.xl / (c.nx - 1), dy = c.yl / (c.ny - 1);
  char nxc[16], nyc[16], nnc[32];
  std::snprintf(nxc, sizeof nxc, "%6d", c.nx);
  std::snprintf(nyc, sizeof nyc, "%6d", c.ny);
  std::snprintf(nnc, sizeof nnc, "%12d", c.nn);
  std::fprintf(fp, "# vtk DataFile Version 3.0\nFastScape\nBINARY\nDATASET STRUCTURED_GRID\nDIMENSIONS %s %s 1\n"
                   "POINTS%s float\n", nxc, nyc, nnc);
  for (int j = 1; j <= c.ny; ++j)
    for (int i = 1; i <= c.nx; ++i) {
      put_be(fp, dx * (i - 1));
      put_be(fp, dy * (j - 1));
      put_be(fp, (z ? (*z)[i + (j - 1) * c.nx] : zc) * std::fabs(vex));
    }
  std::fprintf(fp, "POINT_DATA%s\n", nnc);
  std::fprintf(fp, "SCALARS %s float 1\nLOOKUP_TABLE default\n", name);
  for (int k = 1; k <= c.nn; ++k) put_be(fp, s1 ? (*s1)[k] : s1c);
  if (f) {
    std::fprintf(fp, "SCALARS HHHHH float 1\nLOOKUP_TABLE default\n");
    for (int k = 0; k < c.nn; ++k) put_be(fp, f[k]);
  }
  return std::fclose(fp) == 0;
}

int fso_vtk(const double* f, double vex, const char* dir) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("VTK - You need to run SetUp first");
  const std::string d = dir;
  char cstep[16];
  std::snprintf(cstep, sizeof cstep, "%07d", c.step);
  if (!vtk_one(c, d + "/Topography" + cstep + ".vtk", &c.h, 0.0, "H", &c.h, 0.0, f, vex)) return fail("VTK write");
  if (vex < 0.0) {
    if (!vtk_one(c, d + "/Basement" + cstep + ".vtk", &c.b, 0.0, "B", &c.b, 0.0, f, vex)) return fail("VTK write");
    if (!vtk_one(c, d + "/SeaLevel" + cstep + ".vtk", nullptr, c.sealevel, "SL", nullptr, c.sealevel, nullptr, vex))
      return fail("VTK write");
  }
  return 0;
}

// SetAllLayers -- FastScape_ctx.f90:660-676 (no stratigraphy): h, b += dh
int fso_set_all_layers(const double* dh) {
  Ctx& c = *C;
  if (!c.setup_done) return fail("SetAllLayers - You need to run SetUp first");
  for (int i = 1; i <= c.nn; ++i) { c.h[i] = c.h[i] + dh[i - 1]; c.b[i] = c.b[i] + dh[i - 1]; }
  return 0;
}

}  // extern "C"
