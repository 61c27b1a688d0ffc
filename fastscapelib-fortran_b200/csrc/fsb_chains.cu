// Heavy-path chain schedule of the receiver forest and the single-flow tree
// sweeps that run on it (lake fill, drainage area, stream power law).
//
// The tree recurrences of the reference are sequential loops over the stack:
//   hwater fill           src/FlowRouting.f90:73-89  (root -> leaves)
//   drainage area         src/FlowRouting.f90:123-143 (leaves -> root)
//   implicit SPL, g == 0  src/StreamPowerLaw.f90:291-373 (root -> leaves)
// Each node only needs its receiver (top-down) or its donors (bottom-up), so
// any schedule that respects the tree gives the same per-node arithmetic.
//
// Schedule.  Every node's heavy child is its donor with the largest subtree
// (first in ascending node order on ties).  A heavy-first preorder lays every
// heavy path out contiguously; a "chain" is one heavy path, from its head (a
// root or a light child) to a leaf.  One thread walks a whole chain, carrying
// the running value in registers, so a long river costs one dependent
// arithmetic step per node instead of one inter-thread hand-off.  A chain
// depends only on its head's parent (top-down) or on the chains hanging off
// it (bottom-up); its "light depth" -- the number of light edges above it,
// at most log2(nn) -- therefore orders the chains: tickets are handed out by
// light depth (increasing for top-down sweeps, decreasing for bottom-up), and
// within a light depth longer chains first.  Every wait then targets a chain
// with an earlier ticket, so the sweeps cannot deadlock; warps never mix light
// depths (groups are padded to multiples of 32).
//
// Heavy-first positions come from path sums over the receiver pointers
// (pointer jumping): pos(k) = sum over the root->k path of each node's offset
// within its parent's subtree (1 + sizes of the siblings laid out before it).
#include <cuda/atomic>
#include <climits>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// bounded wait for done[k] == epoch (relaxed polling, then an acquire
// fence); gives up once any wait has failed
// waits (bounded) until done[k] == epoch; the acquire load that sees it makes
// the chain's values released before the flag visible
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

__device__ inline void wait_flag(unsigned* done, int k, unsigned epoch, int* err) {
  int spins = 0, back = 32;
  while (ld_acquire_gpu(&done[k]) != epoch) {
    if (++spins > kSpinLimit) { atomicExch(err, DEV_SPIN_LIMIT); return; }
    if ((spins & 63) == 0 && *(volatile int*)err != 0) return;
    __nanosleep(back);
    if (back < 512) back <<= 1;
  }
}

// heavy child: donor with the largest subtree, first in ascending order on ties
__global__ void k_heavy(int nn, const int* __restrict__ ndon, const int* __restrict__ don,
                        const int* __restrict__ size, int* __restrict__ heavy) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int nd = ndon[k];
    int best = -1, bs = -1;
    for (int i = 0; i < nd; ++i) {
      const int d = don[(size_t)k * 8 + i];
      const int s = size[d];
      if (s > bs) { bs = s; best = d; }
    }
    heavy[k] = best;
  }
}

// sizes of the roots in ascending root order (for the root offsets)
__global__ void k_root_sizes(int nroots, const int* __restrict__ roots, const int* __restrict__ size,
                             int* __restrict__ out) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= nroots; r += gridDim.x * blockDim.x)
    out[r] = r < nroots ? size[roots[r]] : 0;
}

// offset of each node inside its parent's heavy-first layout, light flag in
// the high word; pointer = receiver (or -1 at roots)
__global__ void k_hf_offsets(int nn, const int* __restrict__ rec, const int* __restrict__ ndon,
                             const int* __restrict__ don, const int* __restrict__ size,
                             const int* __restrict__ heavy, const int* __restrict__ root_rank,
                             const int* __restrict__ root_off, unsigned long long* __restrict__ val,
                             int* __restrict__ nxt) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int r = rec[k];
    unsigned long long v;
    if (r == k) {
      v = (unsigned long long)(unsigned)root_off[root_rank[k]];
      nxt[k] = -1;
    } else {
      const int hv = heavy[r];
      if (k == hv) {
        v = 1ull;
      } else {
        unsigned off = 1u + (unsigned)size[hv];
        const int nd = ndon[r];
        for (int i = 0; i < nd; ++i) {
          const int d = don[(size_t)r * 8 + i];
          if (d >= k) break;
          if (d != hv) off += (unsigned)size[d];
        }
        v = (unsigned long long)off | (1ull << 32);
      }
      nxt[k] = r;
    }
    val[k] = v;
  }
}

// Path sums of the heavy-first offsets over the receiver forest without
// pointer jumping: node k's subtree is the interval [pos(k), pos(k) + size(k))
// of the DFS preorder, so adding w(k) at pos(k) and subtracting it at
// pos(k) + size(k) makes the prefix sum at pos(k) the sum over k's ancestors
// and k.  w = (light flag << 27) | offset: offsets sum to a heavy-first
// position (< nn <= 2^27) and light flags to a light depth (< 32), so the
// two fields never carry into each other; the marks wrap modulo 2^32 and
// cancel exactly.
constexpr int kPathOffBits = 27;

__global__ void k_path_marks(int nn, const unsigned long long* __restrict__ val, const int* __restrict__ pos,
                             const int* __restrict__ size, unsigned* __restrict__ marks, int* __restrict__ err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const unsigned long long v = val[k];
    const unsigned w = ((unsigned)(v >> 32) << kPathOffBits) | (unsigned)v;
    const int p = pos[k], e = p + size[k];
    if (p < 0 || e > nn || e <= p) {
      atomicExch(err, DEV_STACK_ERROR);
      continue;
    }
    atomicAdd(&marks[p], w);
    atomicAdd(&marks[e], 0u - w);
  }
}

// after an exclusive scan of the marks: the path sum of k (light depth in the high word)
__global__ void k_path_take(int nn, const int* __restrict__ pos, const unsigned* __restrict__ scan,
                            unsigned long long* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const unsigned s = scan[pos[k] + 1];
    out[k] = ((unsigned long long)(s >> kPathOffBits) << 32) | (s & ((1u << kPathOffBits) - 1u));
  }
}

// one synchronous pointer-jumping round of the path sums
__global__ void k_path_jump(int nn, const unsigned long long* __restrict__ vin, const int* __restrict__ nin,
                            unsigned long long* __restrict__ vout, int* __restrict__ nout, int* __restrict__ flag) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int p = nin[k];
    if (p < 0) {
      vout[k] = vin[k];
      nout[k] = -1;
    } else {
      vout[k] = vin[k] + vin[p];
      const int pp = nin[p];
      nout[k] = pp;
      if (pp >= 0) *flag = 1;
    }
  }
}

__global__ void k_hf_order(int nn, const unsigned long long* __restrict__ val, const int* __restrict__ rec,
                           const int* __restrict__ heavy, int* __restrict__ ord, int* __restrict__ hpos,
                           int* __restrict__ ldep, int* __restrict__ err) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const unsigned p = (unsigned)val[k];
    if (p >= (unsigned)nn) { atomicExch(err, DEV_STACK_ERROR); continue; }
    ord[p] = k;
    hpos[k] = (int)p;
    ldep[k] = (int)(val[k] >> 32);
  }
}

// chain starts: positions whose node is a root or a light child
__global__ void k_chain_flags(int nn, const int* __restrict__ ord, const int* __restrict__ rec,
                              const int* __restrict__ heavy, int* __restrict__ flag) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= nn; p += gridDim.x * blockDim.x) {
    if (p == nn) { flag[p] = 0; continue; }
    const int k = ord[p];
    const int r = rec[k];
    flag[p] = (r == k || heavy[r] != k) ? 1 : 0;
  }
}

// chain list (start positions ascending) with sort keys
//   top-down key:  light depth (6 bits) | ~length (26 bits)
//   bottom-up key: (63 - light depth)   | ~length
__global__ void k_chain_list(int nn, const int* __restrict__ flag, const int* __restrict__ scan,
                             int* __restrict__ cstart, int* __restrict__ cid) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nn; p += gridDim.x * blockDim.x) {
    if (!flag[p]) continue;
    const int c = scan[p];
    cstart[c] = p;
    cid[c] = c;
  }
}

// The light-depth histogram is counted per block in shared memory (few
// distinct depths: one global atomic per block and depth, not per chain).
__global__ void k_chain_keys(int nn, int nchains, const int* __restrict__ cstart, const int* __restrict__ ord,
                             const int* __restrict__ ldep, unsigned* __restrict__ key_td,
                             unsigned* __restrict__ key_bu, int* __restrict__ hist_td, int* __restrict__ hist_bu) {
  __shared__ int sh[64];
  for (int t = threadIdx.x; t < 64; t += blockDim.x) sh[t] = 0;
  __syncthreads();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nchains; c += gridDim.x * blockDim.x) {
    const int s = cstart[c];
    const int e = (c + 1 < nchains) ? cstart[c + 1] : nn;
    const unsigned len = (unsigned)(e - s);
    int ld = ldep[ord[s]];
    if (ld > 63) ld = 63;
    const unsigned inv = 0x3ffffffu - (len > 0x3ffffffu ? 0x3ffffffu : len);
    key_td[c] = ((unsigned)ld << 26) | inv;
    key_bu[c] = ((unsigned)(63 - ld) << 26) | inv;
    atomicAdd(&sh[ld], 1);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 64; t += blockDim.x)
    if (sh[t]) {
      atomicAdd(&hist_td[t], sh[t]);
      atomicAdd(&hist_bu[63 - t], sh[t]);
    }
}

// per-group offsets, padded to multiples of 32 (one thread)
__global__ void k_group_offsets(const int* __restrict__ hist, int* __restrict__ ustart, int* __restrict__ pstart,
                                int* __restrict__ total) {
  int u = 0, pz = 0;
  for (int g = 0; g < 64; ++g) {
    ustart[g] = u;
    pstart[g] = pz;
    u += hist[g];
    pz += (hist[g] + 31) & ~31;
  }
  *total = pz;
}

__global__ void k_ticket_scatter(int nchains, const unsigned* __restrict__ skey, const int* __restrict__ sid,
                                 const int* __restrict__ ustart, const int* __restrict__ pstart,
                                 int* __restrict__ tickets) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nchains; t += gridDim.x * blockDim.x) {
    const int g = (int)(skey[t] >> 26);
    tickets[pstart[g] + (t - ustart[g])] = sid[t];
  }
}

// ---------------------------------------------------------------------------
// chain sweeps

struct ChainView {
  const int* ord;      // heavy-first order
  const int* cstart;   // chain start positions (ascending), nchains entries
  const int* tickets;  // padded ticket list (chain ids or -1)
  int nchains, ntickets, nn;
  __device__ void range(int c, int& s, int& e) const {
    s = cstart[c];
    e = (c + 1 < nchains) ? cstart[c + 1] : nn;  // exclusive
  }
};

constexpr int kCF = 16;  // nodes per software-pipelined chunk (fill, area)
constexpr int kCS = 8;   // nodes per chunk (stream power)

// Top-down: hwater(k) = hwater(rec) > h(k) ? hwater(rec) + 1e-8 : h(k)
// (FlowRouting.f90:77-86); lake_depth = hwater - h.
__global__ void __launch_bounds__(128) k_fill_chains(ChainView cv, const int* __restrict__ rec,
                                                     const int* __restrict__ ndon, const double* __restrict__ h,
                                                     double* __restrict__ hwater, double* __restrict__ lake_depth,
                                                     unsigned* ticket, unsigned* done, unsigned epoch, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(ticket, 32u);
    w = __shfl_sync(FULL, w, 0);
    if ((int)w >= cv.ntickets) break;
    const int t = (int)w + lane;
    const int c = t < cv.ntickets ? cv.tickets[t] : -1;
    if (c < 0) continue;
    int s, e;
    cv.range(c, s, e);
    const int k0 = cv.ord[s];
    const int r0 = rec[k0];
    bool root = r0 == k0;
    double prev = 0.0;
    if (!root) {
      wait_flag(done, r0, epoch, err);
      prev = __ldcg(&hwater[r0]);
    }
    for (int p = s; p < e; p += kCF) {
      const int n = min(kCF, e - p);
      int kk[kCF], nd[kCF];
      double hh[kCF], out[kCF];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) kk[i] = cv.ord[p + i];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) { hh[i] = h[kk[i]]; nd[i] = ndon[kk[i]]; }
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) {
        const double v = root ? hh[i] : (prev > hh[i] ? prev + 1.0e-8 : hh[i]);
        root = false;
        out[i] = v;
        prev = v;
      }
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) { hwater[kk[i]] = out[i]; lake_depth[kk[i]] = out[i] - hh[i]; }
      fence_acq_rel();
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n && nd[i] > 1) *(volatile unsigned*)&done[kk[i]] = epoch;
    }
  }
}

// Bottom-up single-flow area: a(k) = dx*dy*precip(k) + a(d_m) + ... + a(d_1)
// (donors descending, the reverse-stack order of FlowRouting.f90:136-139);
// roots add themselves.  Only the chain head is read by another chain.
// Each chunk first lists its light donors (heads of other chains), reads all
// their done flags at once, fences once and reads all their areas at once;
// the chain recurrence then runs in registers in the original summation order.
constexpr int kLight = 16;  // light donors fetched together per chunk
// Finishers of the bottom-up recurrence v(k) = fin(k, base(k) + v(d_m) + ... + v(d_1)):
//   AreaFin  drainage area; a root adds itself (FlowRouting.f90:136-139)
//   FluxFin  compute_fluxes' sediment flux: base erate, max(0, .) before the
//            value goes downstream, a root adds itself (FastScape_ctx.f90:864-869)
//   GsFin    the erosion sum of a Gauss-Seidel iteration with g > 0
//            (StreamPowerLaw.f90:262-280): base ht-hp; a lake sill's own
//            share is taken out and kept as lake_sediment
//   VolFin   lake water volume: a flooded node passes its contribution
//            (w_rcv - h) and its flooded donors' up to its receiver; every
//            node records what its donors pass as its volume (a sill's volume)
struct AreaFin {
  const double* precip;
  double dxdy;
  __device__ double base(int k) const { return dxdy * precip[k]; }
  __device__ double finish(int, double acc, bool root) const { return root ? acc + acc : acc; }
};
struct FluxFin {
  const double* erate;
  __device__ double base(int k) const { return erate[k]; }
  __device__ double finish(int, double acc, bool root) const {
    acc = fmax(0.0, acc);
    return root ? acc + acc : acc;
  }
};
struct GsFin {
  const double *ht, *hp;
  const int* sill;
  double* lsed;
  __device__ double base(int k) const { return ht[k] - hp[k]; }
  __device__ double finish(int k, double acc, bool root) const {
    if (root) { lsed[k] = acc; return acc; }
    const double e = ht[k] - hp[k];
    const double t = acc - e;
    if (sill[k] == k) lsed[k] = t <= 0.0 ? 0.0 : t;
    return t + e;
  }
};
struct VolFin {
  const int* sill;
  const double* contrib;
  double* vol;
  __device__ double base(int) const { return 0.0; }
  __device__ double finish(int k, double acc, bool root) const {
    vol[k] = acc;
    return (!root && sill[k] != k) ? contrib[k] + acc : 0.0;
  }
};

template <class Fin>
__global__ void __launch_bounds__(128) k_area_chains(ChainView cv, const int* __restrict__ rec,
                                                     const int* __restrict__ ndon, const int* __restrict__ don,
                                                     Fin fin, double* __restrict__ a, unsigned* ticket,
                                                     unsigned* done, unsigned epoch, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    // one chain per warp, walked by lane 0: a bottom-up walk waits at every
    // junction whose light donor is not done, and lanes of one warp waiting
    // (with back-off) at different junctions slowed each other's walks
    // (1023^2 single flow: 8.7 -> 5.4 ms with one chain per warp)
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(ticket, 1u);
    w = __shfl_sync(FULL, w, 0);
    if ((int)w >= cv.ntickets) break;
    const int c = lane == 0 ? cv.tickets[(int)w] : -1;
    if (c < 0) continue;
    int s, e;
    cv.range(c, s, e);
    int child = -1;
    double ac = 0.0;
    for (int hi = e; hi > s; hi -= kCF) {
      const int n = min(kCF, hi - s);
      const int lo = hi - n;
      int kk[kCF], nd[kCF];
      double base[kCF];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) kk[i] = cv.ord[lo + i];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) {
        nd[i] = ndon[kk[i]];
        base[i] = fin.base(kk[i]);
        if (rec[kk[i]] == kk[i]) nd[i] |= 1 << 8;
      }
      // Only nodes with two or more donors have light donors (a node's only
      // donor is its heavy child, the next node down the chain); their donor
      // rows are prefetched together before the listing reads them.
#pragma unroll
      for (int i = 0; i < kCF; ++i)
        if (i < n && (nd[i] & 255) >= 2) prefetch_l1(&don[(size_t)kk[i] * 8]);
      // light donors of the chunk in processing order (i descending, q descending);
      // the heavy child of kk[i] is the next node down the chain
      int lid[kLight];
      double lv[kLight];
      int nl = 0;
      for (int i = n - 1; i >= 0; --i) {
        const int k = kk[i];
        const int heavy = i + 1 < n ? kk[i + 1] : child;
        if ((nd[i] & 255) < 2) continue;
        for (int q = (nd[i] & 255) - 1; q >= 0; --q) {
          const int d = don[(size_t)k * 8 + q];
          if (d != heavy && nl < kLight) lid[nl++] = d;
        }
      }
      if (nl) {
        bool ready = true;
        for (int j = 0; j < nl; ++j) ready &= *(volatile unsigned*)&done[lid[j]] == epoch;
        if (!ready)
          for (int j = 0; j < nl; ++j) wait_flag(done, lid[j], epoch, err);
        fence_acq_rel();
        for (int j = 0; j < nl; ++j) lv[j] = __ldcg(&a[lid[j]]);
      }
      int jl = 0;
#pragma unroll
      for (int i = kCF - 1; i >= 0; --i) if (i < n) {
        const int k = kk[i];
        const int ndk = nd[i] & 255;
        double acc = base[i];
        if (ndk == 1) acc = acc + ac;  // the heavy child alone
        else for (int q = ndk - 1; q >= 0; --q) {
          const int d = don[(size_t)k * 8 + q];
          double v;
          if (d == child) v = ac;
          else if (jl < kLight) v = lv[jl++];
          else {  // more light donors than one fetch holds: read this one on its own
            wait_flag(done, d, epoch, err);
            v = __ldcg(&a[d]);
          }
          acc = acc + v;
        }
        acc = fin.finish(k, acc, (nd[i] >> 8) != 0);
        a[k] = acc;
        ac = acc;
        child = k;
      }
    }
    fence_acq_rel();
    *(volatile unsigned*)&done[cv.ord[s]] = epoch;
  }
}

// CopyChi (FastScape_ctx.f90:228-251) top down: chi(k) = chi(rec(k)) +
// (a0/a(k))^(m/n) * length(k) where a(k) > a0, else 0; a root starts from 0.
__global__ void __launch_bounds__(128) k_chi_chains(ChainView cv, const int* __restrict__ rec,
                                                    const int* __restrict__ ndon, const double* __restrict__ a,
                                                    const double* __restrict__ length, double a0, double mn,
                                                    double* __restrict__ chi, unsigned* ticket, unsigned* done,
                                                    unsigned epoch, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(ticket, 32u);
    w = __shfl_sync(FULL, w, 0);
    if ((int)w >= cv.ntickets) break;
    const int t = (int)w + lane;
    const int c = t < cv.ntickets ? cv.tickets[t] : -1;
    if (c < 0) continue;
    int s, e;
    cv.range(c, s, e);
    const int k0 = cv.ord[s];
    const int r0 = rec[k0];
    double prev = 0.0;
    if (r0 != k0) {
      wait_flag(done, r0, epoch, err);
      prev = __ldcg(&chi[r0]);
    }
    for (int p = s; p < e; p += kCF) {
      const int n = min(kCF, e - p);
      int kk[kCF], nd[kCF];
      double term[kCF], aa[kCF], out[kCF];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) kk[i] = cv.ord[p + i];
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) {
        aa[i] = a[kk[i]];
        nd[i] = ndon[kk[i]];
        term[i] = pow(a0 / aa[i], mn) * length[kk[i]];
      }
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) {
        const double v = aa[i] > a0 ? prev + term[i] : 0.0;
        out[i] = v;
        prev = v;
      }
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n) chi[kk[i]] = out[i];
      fence_acq_rel();
#pragma unroll
      for (int i = 0; i < kCF; ++i) if (i < n && nd[i] > 1) *(volatile unsigned*)&done[kk[i]] = epoch;
    }
  }
}

// Top-down single-flow stream power law with g == 0 (StreamPowerLaw.f90:291-373):
// writes hnew and water; h keeps ht.  The per-node factor kf*dt*a^m/l(^n)
// does not depend on the recurrence and is computed for a whole chunk first.
// With GS (a Gauss-Seidel iteration of the g > 0 solve, StreamPowerLaw.f90:285-373)
// the deposition-corrected surface comes from `elev`, Newton starts from the
// current iterate `hstart`, and the lake bookkeeping is written: sill(k) = k
// for a node above its receiver's water, else sill(rec) with its volume
// contribution w_rcv - h(k) in contrib(k).  Without GS, elev = hstart = ht.
struct GsIo {
  const double* elev;
  const double* hstart;
  int* sill;
  double* contrib;
};

template <bool GS>
__global__ void __launch_bounds__(128) k_spl_chains(ChainView cv, const int* __restrict__ rec,
                                                    const int* __restrict__ ndon, const double* __restrict__ h,
                                                    const double* __restrict__ b, const double* __restrict__ kf,
                                                    const double* __restrict__ a, const double* __restrict__ length,
                                                    double kfsed, double dt, double m, double n, double omega,
                                                    int n_is_one, double* __restrict__ hnew,
                                                    double* __restrict__ water, GsIo gs, unsigned* ticket,
                                                    unsigned* done, unsigned epoch, int* err) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(ticket, 32u);
    w = __shfl_sync(FULL, w, 0);
    if ((int)w >= cv.ntickets) break;
    const int t = (int)w + lane;
    const int c = t < cv.ntickets ? cv.tickets[t] : -1;
    if (c < 0) continue;
    int s, e;
    cv.range(c, s, e);
    const int k0 = cv.ord[s];
    const int r0 = rec[k0];
    bool root = r0 == k0;
    double hr = 0.0, wr = 0.0, htr = 0.0;
    int sr = 0;
    if (!root) {
      wait_flag(done, r0, epoch, err);
      hr = __ldcg(&hnew[r0]);
      wr = __ldcg(&water[r0]);
      htr = h[r0];
      if (GS) sr = __ldcg(&gs.sill[r0]);
    }
    for (int p = s; p < e; p += kCS) {
      const int cn = min(kCS, e - p);
      int kk[kCS], nd[kCS], so[kCS];
      double ht[kCS], fact[kCS], ho[kCS], wo[kCS], el[kCS], h0[kCS], co[kCS];
#pragma unroll
      for (int i = 0; i < kCS; ++i) if (i < cn) kk[i] = cv.ord[p + i];
#pragma unroll
      for (int i = 0; i < kCS; ++i) if (i < cn) {
        const int k = kk[i];
        ht[i] = h[k];
        el[i] = GS ? gs.elev[k] : ht[i];
        h0[i] = GS ? gs.hstart[k] : ht[i];
        nd[i] = ndon[k];
        const double kfint = (kfsed > 0.0 && (ht[i] - b[k]) > 1.0) ? kfsed : kf[k];
        const double l = length[k];
        fact[i] = n_is_one ? kfint * dt * pow(a[k], m) / l : kfint * dt * pow(a[k], m) / pow(l, n);
      }
#pragma unroll
      for (int i = 0; i < kCS; ++i) if (i < cn) {
        double hk = ht[i], wk;
        int sk = kk[i];
        double ck = 0.0;
        if (root) {
          wk = ht[i];
          root = false;
        } else {
          const double elev = el[i];
          hk = h0[i];
          if (elev > wr) {
            if (n_is_one) {
              double f = elev, df = 1.0;
              f = f + fact[i] * hr;
              df = df + fact[i];
              hk = f / df;
            } else {
              const double tolp = 1.0e-3;
              double errp = 2.0 * tolp;
              int guard = 0;
              while (errp > tolp) {
                if (++guard > kNewtonLimit) {
                  atomicExch(err, DEV_NEWTON_LIMIT);
                  break;
                }
                double f = hk - elev, df = 1.0;
                if (ht[i] > htr) {
                  const double x = fmax(0.0, hk - hr);
                  double pn, pn1;
                  if (n == 1.5) {  // x^1.5 = x*sqrt(x), x^0.5 = sqrt(x)
                    pn1 = sqrt(x);
                    pn = x * pn1;
                  } else if (x > 0.0) {  // one pow: x^n = x * x^(n-1)
                    pn1 = pow(x, n - 1.0);
                    pn = x * pn1;
                  } else {
                    pn = pow(x, n);
                    pn1 = pow(x, n - 1.0);
                  }
                  f = f + fact[i] * pn;
                  df = df + fact[i] * n * pn1;
                }
                const double hn = hk - f / df;
                errp = fabs(hn - hk);
                hk = hk * (1.0 - omega) + hn * omega;
              }
            }
            if (hk < wr) hk = wr;
          } else {
            hk = elev;
            sk = sr;
            ck = wr - hk;
          }
          wk = fmax(wr, hk);
        }
        ho[i] = hk;
        wo[i] = wk;
        so[i] = sk;
        co[i] = ck;
        hr = hk;
        wr = wk;
        htr = ht[i];
        sr = sk;
      }
#pragma unroll
      for (int i = 0; i < kCS; ++i) if (i < cn) {
        hnew[kk[i]] = ho[i];
        water[kk[i]] = wo[i];
        if (GS) { gs.sill[kk[i]] = so[i]; gs.contrib[kk[i]] = co[i]; }
      }
      fence_acq_rel();
#pragma unroll
      for (int i = 0; i < kCS; ++i) if (i < cn && nd[i] > 1) *(volatile unsigned*)&done[kk[i]] = epoch;
    }
  }
}

}  // namespace

// Builds the heavy-first order and both ticket lists for the current
// receiver forest (rec, ndon, don, size, roots must be current).
void build_chains(Ctx& c) {
  const int nn = c.nn;
  cudaStream_t st = c.stream;
  k_heavy<<<grid1d(nn), kBlock, 0, st>>>(nn, c.ndon, c.don, c.size, c.ch_heavy);
  cudaMemcpyAsync(c.d_cnt + 15, c.s_scan + nn, sizeof(int), cudaMemcpyDeviceToDevice, st);
  fetch_counters(c, 20);
  c.nroots = c.h_cnt[15];
  const int nroots_h = c.nroots;
  k_root_sizes<<<grid1d(nroots_h + 1), kBlock, 0, st>>>(nroots_h, c.s_roots, c.size, c.ch_tmp);
  c.count_launch(2);
  exclusive_scan_int(c, c.ch_tmp, c.ch_tmp2, nroots_h + 1);
  k_hf_offsets<<<grid1d(nn), kBlock, 0, st>>>(nn, c.rec, c.ndon, c.don, c.size, c.ch_heavy, c.s_root_rank,
                                              c.ch_tmp2, c.ch_val, c.ch_nxt);
  c.count_launch();
  unsigned long long *va = c.ch_val, *vb = c.ch_val2;
  if ((size_t)nn < ((size_t)1 << kPathOffBits)) {
    // a scan over the DFS preorder of the current forest (pos, size)
    unsigned* marks = reinterpret_cast<unsigned*>(c.ch_tmp);
    unsigned* scan = reinterpret_cast<unsigned*>(c.ch_tmp2);
    cudaMemsetAsync(marks, 0, sizeof(unsigned) * (nn + 1), st);
    k_path_marks<<<grid1d(nn), kBlock, 0, st>>>(nn, va, c.pos, c.size, marks, c.d_err);
    c.count_launch();
    exclusive_scan_u32(c, marks, scan, nn + 1);
    k_path_take<<<grid1d(nn), kBlock, 0, st>>>(nn, c.pos, scan, vb);
    c.count_launch();
    std::swap(va, vb);
  } else {
    int *na = c.ch_nxt, *nb = c.ch_nxt2;
    // pointer jumping; the flag read back every 4 rounds says whether any
    // pointer moved in them (rounds after convergence change nothing)
    for (int round = 0; round < 20; ++round) {
      cudaMemsetAsync(c.d_cnt + 16, 0, sizeof(int), st);
      for (int r = 0; r < 4; ++r) {
        k_path_jump<<<grid1d(nn), kBlock, 0, st>>>(nn, va, na, vb, nb, c.d_cnt + 16);
        std::swap(va, vb);
        std::swap(na, nb);
      }
      c.count_launch(4);
      fetch_counters(c, 20);
      if (!c.h_cnt[16]) break;
    }
  }
  k_hf_order<<<grid1d(nn), kBlock, 0, st>>>(nn, va, c.rec, c.ch_heavy, c.ch_ord, c.ch_pos, c.ch_ldep, c.d_err);
  k_chain_flags<<<grid1d(nn + 1), kBlock, 0, st>>>(nn, c.ch_ord, c.rec, c.ch_heavy, c.ch_tmp);
  c.count_launch(2);
  exclusive_scan_int(c, c.ch_tmp, c.ch_tmp2, nn + 1);
  cudaMemcpyAsync(c.d_cnt + 17, c.ch_tmp2 + nn, sizeof(int), cudaMemcpyDeviceToDevice, st);
  fetch_counters(c, 20);
  const int nchains = c.h_cnt[17];
  c.nchains = nchains;
  k_chain_list<<<grid1d(nn), kBlock, 0, st>>>(nn, c.ch_tmp, c.ch_tmp2, c.ch_start, c.ch_cid);
  cudaMemsetAsync(c.ch_hist, 0, sizeof(int) * 128, st);
  k_chain_keys<<<grid1d(nchains), kBlock, 0, st>>>(nn, nchains, c.ch_start, c.ch_ord, c.ch_ldep, c.ch_key,
                                                   c.ch_key + nchains, c.ch_hist, c.ch_hist + 64);
  c.count_launch(2);
  for (int dir = 0; dir < 2; ++dir) {
    sort_pairs_u32(c, c.ch_key + (size_t)dir * nchains, c.ch_skey, c.ch_cid, c.ch_sid, nchains, 32);
    k_group_offsets<<<1, 1, 0, st>>>(c.ch_hist + 64 * dir, c.ch_goff, c.ch_goff + 64, c.d_cnt + 18 + dir);
    int* tk = dir == 0 ? c.ch_tk_td : c.ch_tk_bu;
    cudaMemsetAsync(tk, 0xff, sizeof(int) * ((size_t)nchains + 64 * 32), st);
    k_ticket_scatter<<<grid1d(nchains), kBlock, 0, st>>>(nchains, c.ch_skey, c.ch_sid, c.ch_goff, c.ch_goff + 64, tk);
    c.count_launch(2);
  }
  fetch_counters(c, 20);
  c.ntickets_td = c.h_cnt[18];
  c.ntickets_bu = c.h_cnt[19];
}

void ensure_chains(Ctx& c) {
  if (!c.chains_valid) {
    build_chains(c);
    c.chains_valid = true;
  }
}

static void next_epoch(Ctx& c) {
  c.epoch += 1;
  if (c.epoch == 0) {
    cudaMemsetAsync(c.done, 0, sizeof(unsigned) * c.nn, c.stream);
    c.epoch = 1;
  }
  cudaMemsetAsync(c.ticket, 0, sizeof(unsigned), c.stream);
}

// Persistent chain sweeps: up to 8 blocks per SM, and one block per 4096
// tickets below that.  Most chains of a sweep wait for others, so a few
// threads per thousand chains keep the critical path busy (at 2049^2 the
// sweeps take the same time as with one thread per chain), and the sweeps of
// small and mid-size grids leave the GPU to other streams.
#ifndef FSB_CHAIN_TICKETS_PER_BLOCK
#define FSB_CHAIN_TICKETS_PER_BLOCK 4096
#endif
// bottom-up sweeps take one chain per warp: one block per 512 tickets.  An
// instance that shares the device with others (fsb_set_concurrency) takes a
// quarter of the blocks: the persistent blocks of each instance hold SMs
// while they wait, and fewer of them let more instances run at once (256
// uneven single-flow grids on 32 workers: 3.22e8 -> 3.8e8 node-steps/s).
static int chain_blocks_bu(const Ctx& c, int ntickets) {
  const int per = 512 * c.launch_share;
  const int want = (ntickets + per - 1) / per;
  return want < 1 ? 1 : (want > 148 * 8 ? 148 * 8 : want);
}

static int chain_blocks(const Ctx& c, int ntickets) {
  const int per = FSB_CHAIN_TICKETS_PER_BLOCK * c.launch_share;
  const int want = (ntickets + per - 1) / per;
  return want < 1 ? 1 : (want > 148 * 8 ? 148 * 8 : want);
}

void fill_chains(Ctx& c) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_td, c.nchains, c.ntickets_td, c.nn};
  stage_begin(c, KT_FILL);
  k_fill_chains<<<chain_blocks(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.h, c.hwater, c.lake_depth, c.ticket,
                                                    c.done, c.epoch, c.d_err);
  stage_end(c, KT_FILL);
  c.count_launch();
}

void area_chains(Ctx& c) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_bu, c.nchains, c.ntickets_bu, c.nn};
  k_area_chains<<<chain_blocks_bu(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.don,
                                                                 AreaFin{c.precip, c.dx * c.dy}, c.a, c.ticket,
                                                                 c.done, c.epoch, c.d_err);
  c.count_launch();
}

void flux_chains(Ctx& c, double* flux) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_bu, c.nchains, c.ntickets_bu, c.nn};
  k_area_chains<<<chain_blocks_bu(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.don, FluxFin{c.erate}, flux,
                                                                 c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

void chi_chains(Ctx& c, double a0, double mn, double* chi) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_td, c.nchains, c.ntickets_td, c.nn};
  k_chi_chains<<<chain_blocks(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.a, c.length, a0, mn, chi, c.ticket,
                                                                c.done, c.epoch, c.d_err);
  c.count_launch();
}

void spl_chains(Ctx& c, double* hnew) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_td, c.nchains, c.ntickets_td, c.nn};
  const int n1 = fabs(c.n - 1.0) < 2.2250738585072014e-308;
  k_spl_chains<false><<<chain_blocks(c, cv.ntickets), 128, 0, c.stream>>>(
      cv, c.rec, c.ndon, c.h, c.b, c.kf, c.a, c.length, c.kfsed, c.dt, c.m, c.n, 0.875 / c.n, n1, hnew, c.water,
      GsIo{nullptr, nullptr, nullptr, nullptr}, c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

void spl_chains_gs(Ctx& c, const double* elev, const double* hstart, double* hnew, int* sill, double* contrib) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_td, c.nchains, c.ntickets_td, c.nn};
  const int n1 = fabs(c.n - 1.0) < 2.2250738585072014e-308;
  k_spl_chains<true><<<chain_blocks(c, cv.ntickets), 128, 0, c.stream>>>(
      cv, c.rec, c.ndon, c.h, c.b, c.kf, c.a, c.length, c.kfsed, c.dt, c.m, c.n, 0.875 / c.n, n1, hnew, c.water,
      GsIo{elev, hstart, sill, contrib}, c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

void gs_erosion_chains(Ctx& c, const double* hp, const int* sill, double* lsed, double* dh) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_bu, c.nchains, c.ntickets_bu, c.nn};
  k_area_chains<<<chain_blocks_bu(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.don, GsFin{c.h, hp, sill, lsed},
                                                                 dh, c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

void lake_volume_chains(Ctx& c, const int* sill, const double* contrib, double* vol, double* up) {
  next_epoch(c);
  ChainView cv{c.ch_ord, c.ch_start, c.ch_tk_bu, c.nchains, c.ntickets_bu, c.nn};
  k_area_chains<<<chain_blocks_bu(c, cv.ntickets), 128, 0, c.stream>>>(cv, c.rec, c.ndon, c.don, VolFin{sill, contrib, vol},
                                                                 up, c.ticket, c.done, c.epoch, c.d_err);
  c.count_launch();
}

}  // namespace fsb
