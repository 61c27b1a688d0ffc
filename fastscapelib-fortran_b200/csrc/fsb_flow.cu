// Multiple-flow receivers, multiple-flow sweeps (drainage area and implicit
// stream power law), the stream-power epilogue and ADI hillslope diffusion.
//
// Reference routines restated here (fastscapelib-fortran file:line):
//   find_mult_rec                 src/FlowRouting.f90:147-298
//   FlowAccumulation (MFD)        src/FlowRouting.f90:97-119
//   StreamPowerLaw (MFD)          src/StreamPowerLaw.f90:3-206 (the g > 0
//                                 iterations are driven from fsb_sediment.cu)
//   Diffusion + tridag            src/Diffusion.f90:1-202
// The single-flow tree sweeps live in fsb_chains.cu.
//
// Multiple-flow sweeps run over the receiver DAG with dependency counters:
// every node starts with the number of nodes it waits for; the thread that
// brings a counter to zero ("last arriver") continues with that node, and
// further nodes it makes ready go to a work queue.  Nothing waits on work that
// has not been scheduled, so the sweep needs no global order and cannot
// deadlock.  A producer hands its value to each dependent by storing it into
// one of the dependent's input slots before decrementing the dependent's
// counter; the consumer reads its slots and waits (bounded) on any that still
// hold the empty sentinel, so no fence is needed on either side.
#include <algorithm>
#include <cmath>
#include <cuda/atomic>
#include <cfloat>
#include <cstddef>

#include "fsb_kernels.cuh"

namespace fsb {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ inline unsigned long long ordered_key(double x) {
  unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

// ---- last-arriver sweep engine ----------------------------------------------
// Op::run(k, dep[]) computes node k, stores its outputs and lists k's
// dependents, largest priority (subtree size) first, prefetching their
// records; the engine then decrements their counters, continues with the
// first one made ready and queues the other ready ones.  The hop is bound by
// the latency of one thread's instructions as much as by its round trips, so
// the records hold the dependents as node indices in priority order: no
// decoding and no comparison on the critical path (2049^2 step 58.9 ->
// 52.1 ms against 4-bit codes with inline priorities).  Idle lanes claim queue slots in
// order (one atomic per warp) and keep a claim until a producer fills it.
// The kernel ends when every node is done.
// Control words: ctl[0] queue head, ctl[32] queue tail, ctl[64] nodes done
// (separate 128-byte lines).
// Only the first LANES lanes of a warp take nodes: a warp moves through a hop
// in lockstep, so fewer nodes per warp shorten the critical node's wait on
// its warp mates' loads and Newton iterations.  The sweeps are bound by their
// critical path, not by node throughput; at 2049^2 (B200) 8 lanes suit the
// area sweep and 1 lane the stream-power sweep (32 lanes: 25.8 and 46.1 ms,
// these: 24.4 and 41.2 ms).  Re-measured with the dependents stored as node
// indices: area sweep 14.2 ms with 8 lanes, 14.7 / 15.4 / 16.0 ms with 4 / 2 / 1
// (grids of side/4, /2, /1 blocks).
#ifndef FSB_LANES_ACC
#define FSB_LANES_ACC 8
#endif
#ifndef FSB_LANES_SPL
#define FSB_LANES_SPL 1
#endif
// Grid of a sweep: sqrt(nn)/SIDE_DIV blocks, 8 to 592 (4 per SM).  The
// sweeps are bound by their critical path, whose length grows with the grid
// side, and the nodes in flight it needs grow with the side too; idle lanes
// poll the work queue, so more blocks than that slow a sweep down.  Measured
// on B200 (area with side/4, stream power with side/8): 513^2 17 ms/step
// against 32 with one block per 16384 nodes; 2049^2 unchanged (256 blocks
// for stream power beat 592: 35 against 40 ms).  Smaller grids leave the
// rest of the GPU to other streams.
#ifndef FSB_SIDE_DIV_ACC
#define FSB_SIDE_DIV_ACC 4
#endif
#ifndef FSB_SIDE_DIV_SPL
#define FSB_SIDE_DIV_SPL 8
#endif
template <class Op, int LANES>
__global__ void __launch_bounds__(128) k_last_arriver(Op op, int nn, int* cnt, int* queue, unsigned* ctl, int* err) {
  unsigned* qhead = ctl;
  unsigned* qtail = ctl + 32;
  unsigned* ndone = ctl + 64;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int cur = -1;
  long long slot = -1;
  unsigned local_done = 0;
  int back = 32;
  for (int it = 0; it < (1 << 24); ++it) {
    const bool want = lane < LANES && cur < 0 && slot < 0;
    const unsigned m = __ballot_sync(FULL, want);
    if (m) {
      const int leader = __ffs(m) - 1;
      unsigned base = 0;
      if (lane == leader) base = atomicAdd(qhead, (unsigned)__popc(m));
      base = __shfl_sync(FULL, base, leader);
      if (want) slot = (long long)base + __popc(m & lt);
    }
    if (cur < 0 && slot >= 0 && slot < nn) {
      const int v = ld_relaxed_gpu(&queue[slot]);
      if (v >= 0) { cur = v; slot = -1; }
    }
    int dep[8];
    unsigned rdy = 0;  // bit t: dependent t became ready and goes to the queue
    if (cur >= 0) {
      // No fence or acquire anywhere: op.run reads cur's inputs from its
      // slots, where each producer stored its value before its decrement,
      // and waits on a slot that still holds the sentinel.  (On B200 this
      // hand-off costs ~510 ns against ~860 ns with a release fence and an
      // acquire load, ~1160 ns with two fences.)
      const int nd = op.run(cur, dep);
      int nxt = -1;
      if (nd) {
        int old[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) old[t] = t < nd ? atomicSub(&cnt[dep[t]], 1) : 0;
#pragma unroll
        for (int t = 0; t < 8; ++t) rdy |= (old[t] == 1 ? 1u : 0u) << t;
        // continue with the first ready dependent (they come largest priority first)
#pragma unroll
        for (int t = 7; t >= 0; --t) nxt = ((rdy >> t) & 1u) ? dep[t] : nxt;
        rdy &= rdy - 1u;
      }
      ++local_done;
      cur = nxt;
    }
    if (__ballot_sync(FULL, rdy != 0)) {  // queue the other ready nodes: one atomic per warp
      const unsigned mine = __popc(rdy);
      unsigned off = mine;  // inclusive prefix of the lanes' counts (only lanes < LANES have any)
#pragma unroll
      for (int o = 1; o < LANES; o <<= 1) {
        const unsigned y = __shfl_up_sync(FULL, off, o);
        if (lane >= o) off += y;
      }
      const unsigned total = __shfl_sync(FULL, off, LANES - 1);
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(qtail, total);
      base = __shfl_sync(FULL, base, 0) + off - mine;
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if ((rdy >> t) & 1u) {
          if (base < (unsigned)nn) *(volatile int*)&queue[base] = dep[t];
          else atomicExch(err, DEV_OVERFLOW);
          ++base;
        }
    }
    const unsigned busy = __ballot_sync(FULL, cur >= 0);
    if (!busy) {
      const unsigned tot = __reduce_add_sync(FULL, local_done);
      if (lane == 0 && tot) atomicAdd(ndone, tot);
      local_done = 0;
      unsigned d = 0;
      int e = 0;
      if (lane == 0) { d = *(volatile unsigned*)ndone; e = *(volatile int*)err; }
      d = __shfl_sync(FULL, d, 0);
      e = __shfl_sync(FULL, e, 0);
      if (d >= (unsigned)nn || e != 0) return;
      __nanosleep(back);
      if (back < 256) back <<= 1;  // longer caps were measured slower (4 us: +1.6 ms at 2049^2)
    } else {
      back = 32;
    }
  }
  if (lane == 0) atomicExch(err, DEV_SPIN_LIMIT);
}


// initial queue: nodes whose counter is zero
__global__ void k_seed_queue(int nn, const int* __restrict__ cnt, int* __restrict__ queue, unsigned* qtail) {
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < nn; base += gridDim.x * blockDim.x) {
    const int k = base + threadIdx.x;
    const bool z = k < nn && cnt[k] == 0;
    const unsigned m = __ballot_sync(FULL, z);
    if (!m) continue;
    unsigned b = 0;
    const int leader = __ffs(m) - 1;
    if (lane == leader) b = atomicAdd(qtail, (unsigned)__popc(m));
    b = __shfl_sync(FULL, b, leader);
    if (z) queue[b + __popc(m & ((1u << lane) - 1u))] = k;
  }
}

// ---- per-node records of the multiple-flow sweeps ---------------------------
// Each node has one 128-byte line, built in parallel before a sweep, holding
// everything the sweep reads about the node except its dependencies' values.
// A node's dependents are stored as node indices (-1 past the last), sorted
// by priority, largest first: the upper 16 bits of the float value of the
// neighbour's single-flow subtree size (monotonic), ties in neighbour order.
// A sweep's hop then needs no decoding and no comparison to find the
// dependent to continue with: it is the first one made ready.  Inputs are
// 4-bit neighbour codes 1 + 3*(dj+1) + (di+1) (0 = empty slot), eight to a
// 32-bit word with slot t in bits 4t..4t+3, filled from slot 0; they are
// decoded with the grid's wrap-around.
//
// Area line:    aw[8]  summed weight of donor t's slots targeting k
//               base   dx*dy*precip(k)
//               dep[8] the distinct receivers (dependents)
//               don    codes of the distinct donors (inputs)
// Stream-power line:
//               fact[8] kf*dt*(a*w)^m/l^n of receiver slot t whose erosion
//                       term is gated on (ht(k) >= ht(q), or > for n != 1)
//               ht      h(k)
//               dep[8]  the donors that wait for k (gated, or rec == k)
//               q       codes of those receiver slots
//               meta    code of rec(k) (0: k is a root); bit 4 set when mnrec(k) > 0
// The values a sweep hands from node to node travel in slots: node k's inputs
// are Ctx::slots[k*kSlotStride + s] (area: s = donor position; stream power:
// s = gated-receiver position, 8 = rec's water, 9 = rec's lake sill as
// integer bits), all ones until written.  rpos / qmask / wflag tell a
// producer where its value goes in each dependent's slots; they are filled by
// a second pass over the consumers (k_acc_slotpos, k_spl_slotpos).
struct __align__(128) AccLine {
  double aw[8];
  double base;
  int dep[8];
  unsigned don;
  unsigned rpos;  // 4 bits per receiver t: this node's slot in that receiver's inputs
  int pad[4];
};
struct __align__(128) SplLine {
  double fact[8];
  double ht;
  int dep[8];
  unsigned q;
  int meta;
  unsigned qmask[2];  // 8 bits per dependent t (t < 4: qmask[0]): its gated slots that are this node
  unsigned wflag;     // bit t: this node is rec of dependent t (water, and the lake sill with g > 0)
  int pad;
};
static_assert(sizeof(AccLine) == 128 && sizeof(SplLine) == 128, "one line per node");
static_assert(offsetof(AccLine, dep) == 72 && offsetof(AccLine, don) == 104 && offsetof(AccLine, rpos) == 108,
              "AccLine words: aw 0-15, base 16-17, dep 18-25, don 26, rpos 27");
static_assert(offsetof(SplLine, dep) == 72 && offsetof(SplLine, q) == 104 && offsetof(SplLine, meta) == 108 &&
                  offsetof(SplLine, qmask) == 112 && offsetof(SplLine, wflag) == 120,
              "SplLine words: fact 0-15, ht 16-17, dep 18-25, q 26, meta 27, qmask 28-29, wflag 30");

__device__ inline unsigned short prio16(int size) { return (unsigned short)(__float_as_uint((float)size) >> 16); }

// The line builders keep their short lists in registers: every entry is
// addressed by an index known after unrolling, selected by a predicate.
// Inserts node v of priority p into dep[0..n) / pr[0..n) (n < 8), kept in
// decreasing priority with ties in insertion order.
__device__ inline void insert_by_priority(int (&dep)[8], unsigned (&pr)[8], int n, int v, unsigned p) {
  int pos = 0;  // entries of priority >= p stay in front
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
__device__ inline int4 pack2(double a, double b) {
  return make_int4(__double2loint(a), __double2hiint(a), __double2loint(b), __double2hiint(b));
}
// Writes a record line from its 32 words: eight 16-byte stores.
__device__ inline void store_line(void* dst, const int4 (&w)[8]) {
  int4* p = reinterpret_cast<int4*>(dst);
#pragma unroll
  for (int t = 0; t < 8; ++t) p[t] = w[t];
}

__device__ inline unsigned nbr_code(int di, int dj) { return 1u + 3u * (unsigned)(dj + 1) + (unsigned)(di + 1); }

// code of neighbour q of node (i, j); sets *err when q is not a 3x3 neighbour
__device__ inline unsigned nbr_code_of(int i, int j, int q, int nx, int ny, int* err) {
  int di = q % nx - i, dj = q / nx - j;
  if (di > 1) di -= nx; else if (di < -1) di += nx;
  if (dj > 1) dj -= ny; else if (dj < -1) dj += ny;
  if (di < -1 || di > 1 || dj < -1 || dj > 1 || (di == 0 && dj == 0)) {
    atomicExch(err, DEV_NOT_ADJACENT);
    return 0u;
  }
  return nbr_code(di, dj);
}

struct NbrDecoder {
  int nx, ny, i, j;
  __device__ NbrDecoder(int k, int nx_, int ny_) : nx(nx_), ny(ny_), i(k % nx_), j(k / nx_) {}
  __device__ int at(unsigned code) const {
    const int c = (int)code - 1;
    int x = i + c % 3 - 1, y = j + c / 3 - 1;
    x += x < 0 ? nx : (x >= nx ? -nx : 0);
    y += y < 0 ? ny : (y >= ny ? -ny : 0);
    return x + y * nx;
  }
};

// x^n and x^(n-1) for the Newton update.  For n = 1.5 they are evaluated as
// x*sqrt(x) and sqrt(x) (sqrt is correctly rounded); otherwise as x*x^(n-1)
// and x^(n-1) with one pow for x > 0 (within an ulp or two of pow(x, n)), and
// with two pows at x = 0.
struct NewtonPow {
  double n;
  int half3;  // n == 1.5
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

__device__ inline void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }
__device__ inline void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
// As soon as a node knows its dependents it prefetches their record lines
// into L1 and their slot rows into L2, overlapping those fetches with its own
// arithmetic and counter atomics (2049^2 step 60.5 -> 58.9 ms; prefetching
// only the continuation's line after the atomics, or the lines into L2
// only, measured slower).
template <class Line>
__device__ inline void prefetch_dependents(const Line* line, const double* slots, const int* dep, int nd) {
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (t < nd) {
      prefetch_l1(line + dep[t]);
      prefetch_l2(slots + (size_t)dep[t] * kSlotStride);
    }
}

// the first N 16-byte words of a record line (read-only during the sweep)
template <int N>
union LineWords {
  int4 v[N];
  double d[2 * N];
  unsigned u[4 * N];
  unsigned short s[8 * N];
  __device__ explicit LineWords(const void* p) {
#pragma unroll
    for (int t = 0; t < N; ++t) v[t] = __ldg(reinterpret_cast<const int4*>(p) + t);
  }
};

// A consumer's input slot: strong relaxed loads, then a bounded wait while a
// slot still holds the all-ones sentinel (its producer's store is in flight).
constexpr long long kSlotEmpty = -1ll;
__device__ inline double slot_value(const double* p, double v, int* err) {
  int spins = 0;
  while (__double_as_longlong(v) == kSlotEmpty) {
    if (++spins > kSpinLimit) { atomicExch(err, DEV_SPIN_LIMIT); return 0.0; }
    __nanosleep(32);
    v = ld_relaxed_gpu(p);
  }
  return v;
}
// Bit t set when input slot t (in the 4-bit code word c) still holds the sentinel:
// one test for all of a node's inputs, so the usual case takes no branch per slot.
__device__ inline unsigned empty_slots(const double* v, unsigned c) {
  unsigned m = 0;
#pragma unroll
  for (int t = 0; t < 8; ++t)
    m |= (((c >> (4 * t)) & 15u) && __double_as_longlong(v[t]) == kSlotEmpty ? 1u : 0u) << t;
  return m;
}

// a(k) = dx*dy*precip(k) + sum over donors of a(d)*w(d->k) (FlowRouting.f90:109-115);
// k's dependents are its distinct receivers.  With `clamp` set and lines
// built on erate it is compute_fluxes' sediment flux (FastScape_ctx.f90:871-877):
// max(0, .) before the node's value goes downstream.
// With `gs` set (lines built on e = ht - hp) it is the erosion sum of a
// Gauss-Seidel iteration with g > 0 (StreamPowerLaw.f90:59-80): a sill's own
// share is taken out and kept as lake_sediment; a root keeps its whole sum.
struct AccMfdOp {
  const AccLine* line;
  double* a;
  int clamp;
  double* slots = nullptr;
  int* err = nullptr;
  int gs = 0;
  const int* rec = nullptr;
  const int* sill = nullptr;
  double* lsed = nullptr;
  __device__ int run(int k, int* dep) const {
    // the input slots do not depend on the line: load them together with it
    const double* in = slots + (size_t)k * kSlotStride;
    double av[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) av[t] = ld_relaxed_gpu(&in[t]);
    // aw = d[0..7], base = d[8], dep = u[18..25], don = u[26], rpos = u[27]
    const LineWords<7> L(line + k);
    const unsigned dc = L.u[26], rpos = L.u[27];
    if (empty_slots(av, dc)) {
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if ((dc >> (4 * t)) & 15u) av[t] = slot_value(&in[t], av[t], err);
    }
    int nd = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      dep[t] = (int)L.u[18 + t];
      nd += dep[t] >= 0;
    }
    prefetch_dependents(line, slots, dep, nd);
    double acc = L.d[8];
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if ((dc >> (4 * t)) & 15u) acc = acc + av[t] * L.d[t];
    if (clamp) acc = fmax(0.0, acc);
    if (gs) {
      if (rec[k] == k) {
        lsed[k] = acc;
      } else {
        const double e = L.d[8];
        const double t = acc - e;
        if (sill[k] == k) lsed[k] = t <= 0.0 ? 0.0 : t;
        acc = t + e;
      }
    }
    a[k] = acc;
#pragma unroll
    for (int t = 0; t < 8; ++t)  // hand the value to the receivers
      if (t < nd) st_relaxed_gpu(&slots[(size_t)dep[t] * kSlotStride + ((rpos >> (4 * t)) & 15u)], acc);
    return nd;
  }
};

// implicit stream power law over the multiple receivers with g == 0
// (StreamPowerLaw.f90:92-177): the new elevation and the water surface go to
// hw[k] = (h, water); h keeps ht.  k's dependents are the donors that read it.
// With GS (g > 0, StreamPowerLaw.f90:89-177 in a Gauss-Seidel iteration) the
// surface comes from `elev`, Newton starts from the current iterate `hstart`,
// and sill / contrib record the lake bookkeeping (as in k_spl_chains).
template <bool GS>
struct SplMfdOp {
  const SplLine* line;
  NewtonPow np;
  double omega;
  int n_is_one;
  double2* hw;
  double* slots = nullptr;
  int* err = nullptr;
  const double* elev = nullptr;
  const double* hstart = nullptr;
  int* sill = nullptr;
  double* contrib = nullptr;
  __device__ int run(int k, int* dep) const {
    // the input slots do not depend on the line: load them together with it
    const double* in = slots + (size_t)k * kSlotStride;
    double hq[8], wr, sv = 0.0;
#pragma unroll
    for (int t = 0; t < 8; ++t) hq[t] = ld_relaxed_gpu(&in[t]);
    wr = ld_relaxed_gpu(&in[8]);
    if (GS) sv = ld_relaxed_gpu(&in[9]);
    // fact = d[0..7], ht = d[8], dep = u[18..25], q = u[26], meta = u[27],
    // qmask = u[28..29], wflag = u[30]
    const LineWords<8> L(line + k);
    const unsigned qc = L.u[26], meta = L.u[27], wflag = L.u[30];
    const double ht = L.d[8];
    int nd = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      dep[t] = (int)L.u[18 + t];
      nd += dep[t] >= 0;
    }
    prefetch_dependents(line, slots, dep, nd);
    double hk = ht, wk = ht;
    int sk = k;
    double ck = 0.0;
    const unsigned rcode = meta & 15u;
    if (rcode) {
      wr = slot_value(&in[8], wr, err);
      if (empty_slots(hq, qc)) {
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if ((qc >> (4 * t)) & 15u) hq[t] = slot_value(&in[t], hq[t], err);
      }
      if (GS) hk = hstart[k];
      const double elev = GS ? this->elev[k] : ht;
      if (elev > wr) {
        if (meta & 16u) {  // mnrec(k) > 0
          if (n_is_one) {
            double f = elev, df = 1.0;
#pragma unroll
            for (int t = 0; t < 8; ++t)
              if ((qc >> (4 * t)) & 15u) {
                f = f + L.d[t] * hq[t];
                df = df + L.d[t];
              }
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
#pragma unroll
              for (int t = 0; t < 8; ++t)
                if ((qc >> (4 * t)) & 15u) {
                  const double x = fmax(0.0, hk - hq[t]);
                  double pn, pn1;
                  np.eval(x, pn, pn1);
                  f = f + L.d[t] * pn;
                  df = df + L.d[t] * np.n * pn1;
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
        if (GS) {
          sk = (int)__double_as_longlong(slot_value(&in[9], sv, err));
          ck = wr - hk;
        }
      }
      wk = fmax(wr, hk);
    }
    hw[k] = make_double2(hk, wk);
    if (GS) {
      sill[k] = sk;
      contrib[k] = ck;
    }
    // hand h (to the gated slots that are this node), water and the sill (to
    // the donors whose rec this node is) to the dependents
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t >= nd) break;
      double* out = slots + (size_t)dep[t] * kSlotStride;
      unsigned m = (L.u[28 + (t >> 2)] >> (8 * (t & 3))) & 0xffu;
      while (m) {  // usually one bit
        st_relaxed_gpu(&out[__ffs(m) - 1], hk);
        m &= m - 1u;
      }
      if ((wflag >> t) & 1u) {
        st_relaxed_gpu(&out[8], wk);
        if (GS) st_relaxed_gpu(&out[9], __longlong_as_double((long long)sk));
      }
    }
    return nd;
  }
};


// ---- find_mult_rec (FlowRouting.f90:200-243) --------------------------------
// MIXED: the receivers (FP64 comparisons of the filled surface) are the
// same; the slopes, their powers and the normalisation run in FP32 (the
// height differences are taken in FP64 and rounded once).
// a[n] = v for a register array (n in 0..7; no local-memory indexing)
template <class T>
__device__ inline void put8(T (&a)[8], int n, T v) {
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (t == n) a[t] = v;
}

template <bool MIXED>
__global__ void k_mfd_receivers(Bounds bd, double p, const double* __restrict__ h0, const double* __restrict__ ltab,
                                int* __restrict__ mrec, int* __restrict__ mnrec, double* __restrict__ mwrec,
                                double* __restrict__ mlrec) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int ij = blockIdx.x * blockDim.x + threadIdx.x; ij < nn; ij += gridDim.x * blockDim.x) {
    const int i = ij % nx, j = ij / nx;
    int nr = 0;
    int rr[8];
    double w[8], ll[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      rr[t] = -1;
      w[t] = 0.0;
      ll[t] = 0.0;
    }
    if (i >= bd.i1 && i <= bd.i2 && j >= bd.j1 && j <= bd.j2) {
      const double hij = h0[ij];
#pragma unroll
      for (int jj = -1; jj <= 1; ++jj) {
        const int jjj = wrap_clamp(j + jj, ny, bd.ycyc);
#pragma unroll
        for (int ii = -1; ii <= 1; ++ii) {
          const int iii = wrap_clamp(i + ii, nx, bd.xcyc);
          const int ijk = iii + jjj * nx;
          const double hk = h0[ijk];
          if (hij > hk) {
            const double l = __ldg(&ltab[(jj + 1) * 3 + (ii + 1)]);
            put8(rr, nr, ijk);
            put8(ll, nr, l);
            put8(w, nr, (hij - hk) / l);
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
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (t < nr) s = s + w[t];
        slope = (double)(float)(s / nr);
      }
      pe = (double)0.5f + (double)0.6f * slope;
    }
    double mw[8];
    if constexpr (MIXED) {
      float wf[8], sumf = 0.0f;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        wf[t] = t < nr ? powf((float)w[t], (float)pe) : 0.0f;
        if (t < nr) sumf = sumf + wf[t];
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) mw[t] = t < nr ? (double)(wf[t] / sumf) : 0.0;
    } else {
      double sumw = 0.0;
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        if (t < nr) w[t] = pow(w[t], pe);
        if (t < nr) sumw = sumw + w[t];
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) mw[t] = t < nr ? w[t] / sumw : 0.0;
    }
    // the three rows, padded past nr (-1 / 0), with 16-byte stores
    int4* r4 = reinterpret_cast<int4*>(mrec + (size_t)ij * 8);
    r4[0] = make_int4(rr[0], rr[1], rr[2], rr[3]);
    r4[1] = make_int4(rr[4], rr[5], rr[6], rr[7]);
    double2* w2 = reinterpret_cast<double2*>(mwrec + (size_t)ij * 8);
    double2* l2 = reinterpret_cast<double2*>(mlrec + (size_t)ij * 8);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      w2[t] = make_double2(mw[2 * t], mw[2 * t + 1]);
      l2[t] = make_double2(ll[2 * t], ll[2 * t + 1]);
    }
    mnrec[ij] = nr;
  }
}

// Area lines and counters: cnt_acc(k) = number of distinct donors of k.
__global__ void k_acc_lines(Bounds bd, double dxdy, const int* __restrict__ mrec, const int* __restrict__ mnrec,
                            const double* __restrict__ mwrec, const double* __restrict__ precip,
                            const int* __restrict__ prio, AccLine* __restrict__ line, int* __restrict__ cnt_acc,
                            int* err) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    const size_t o = (size_t)k * 8;
    // distinct receivers (dependents), largest priority first
    const int nr = mnrec[k];
    int mr[8], dep[8];
    unsigned pr[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      mr[t] = t < nr ? mrec[o + t] : -1;
      dep[t] = -1;
      pr[t] = 0u;
    }
    int rn = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t >= nr) break;
      const int q = mr[t];
      if (contains(mr, t, q)) continue;
      (void)nbr_code_of(i, j, q, nx, ny, err);  // checks that q is a neighbour
      insert_by_priority(dep, pr, rn++, q, prio16(prio[q]));
    }
    // distinct donors among the 3x3 neighbours and the summed weight of their slots to k
    unsigned don = 0;
    int an = 0, ns = 0;
    int seen[8];
    double aw[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) aw[t] = 0.0;
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
        const int nd = mnrec[d];
        double wsum = 0.0;
        int hits = 0;
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (t < nd && mrec[(size_t)d * 8 + t] == k) {
            const double w = mwrec[(size_t)d * 8 + t];
            wsum = hits ? wsum + w : w;
            ++hits;
          }
        if (hits && an < 8) {
          don |= nbr_code(ii, jj) << (4 * an);
          set_at(aw, an++, wsum);
        }
      }
    }
    const double base = dxdy * precip[k];
    const int4 w[8] = {pack2(aw[0], aw[1]), pack2(aw[2], aw[3]), pack2(aw[4], aw[5]), pack2(aw[6], aw[7]),
                       make_int4(__double2loint(base), __double2hiint(base), dep[0], dep[1]),
                       make_int4(dep[2], dep[3], dep[4], dep[5]),
                       make_int4(dep[6], dep[7], (int)don, 0),  // rpos: filled by k_acc_slotpos
                       make_int4(0, 0, 0, 0)};
    store_line(line + k, w);
    cnt_acc[k] = an;
  }
}

// Stream-power lines and counters: cnt_spl(k) = distinct gated receivers of k
// plus rec(k) when it is not among them (0 for a root).
__global__ void k_spl_lines(Bounds bd, int n_is_one, double kfsed, double dt, double m, double n,
                            const int* __restrict__ rec, const int* __restrict__ mrec, const int* __restrict__ mnrec,
                            const double* __restrict__ mwrec, const double* __restrict__ mlrec,
                            const double* __restrict__ h, const double* __restrict__ b, const double* __restrict__ kf,
                            const double* __restrict__ a, const int* __restrict__ prio, SplLine* __restrict__ line,
                            int* __restrict__ cnt_spl, int* err) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx, j = k / nx;
    const size_t o = (size_t)k * 8;
    const double htk = h[k];
    const int nr = mnrec[k];
    const int r = rec[k];
    const double kk = ((kfsed > 0.0 && (htk - b[k]) > 1.0) ? kfsed : kf[k]) * dt;
    const double ak = a[k];
    int qv[8], dep[8];
    unsigned pr[8];
    double fact[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      qv[t] = -1;
      dep[t] = -1;
      pr[t] = 0u;
      fact[t] = 0.0;
    }
    unsigned qc = 0;
    int nq = 0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      if (t >= nr) break;
      const int q = mrec[o + t];
      if (n_is_one ? (htk >= h[q]) : (htk > h[q])) {
        const double w = mwrec[o + t], l = mlrec[o + t];
        qc |= nbr_code_of(i, j, q, nx, ny, err) << (4 * nq);
        set_at(fact, nq, n_is_one ? kk * pow(ak * w, m) / l : kk * pow(ak * w, m) / pow(l, n));
        set_at(qv, nq++, q);
      }
    }
    int cs = 0;
    if (r != k) {
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < nq && !contains(qv, t, qv[t])) ++cs;
      if (!contains(qv, nq, r)) ++cs;
    }
    // donors that wait for k: they read hnew(k) (gated) or water(k) (rec == k),
    // largest priority first
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
        bool hits = false;
        const int nd = mnrec[d];
#pragma unroll
        for (int t = 0; t < 8; ++t) hits |= t < nd && mrec[(size_t)d * 8 + t] == k;
        const bool gated = hits && (n_is_one ? (h[d] >= htk) : (h[d] > htk));
        if ((gated || rd == k) && dn < 8) insert_by_priority(dep, pr, dn++, d, prio16(prio[d]));
      }
    }
    const int meta = (int)((r != k ? nbr_code_of(i, j, r, nx, ny, err) : 0u) | (nr > 0 ? 16u : 0u));
    const int4 w[8] = {pack2(fact[0], fact[1]), pack2(fact[2], fact[3]), pack2(fact[4], fact[5]),
                       pack2(fact[6], fact[7]),
                       make_int4(__double2loint(htk), __double2hiint(htk), dep[0], dep[1]),
                       make_int4(dep[2], dep[3], dep[4], dep[5]),
                       make_int4(dep[6], dep[7], (int)qc, meta),
                       make_int4(0, 0, 0, 0)};  // qmask, wflag: filled by k_spl_slotpos
    store_line(line + k, w);
    cnt_spl[k] = cs;
  }
}


// Slot positions, area: consumer r's donor at position t (in r's donor list)
// is told that its value goes to r's slot t, in the nibble of r in its own
// receiver list.
__global__ void k_acc_slotpos(int nx, int ny, AccLine* __restrict__ line) {
  const int nn = nx * ny;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nn; r += gridDim.x * blockDim.x) {
    const NbrDecoder nb(r, nx, ny);
    const unsigned dc = line[r].don;
    for (int t = 0; t < 8; ++t) {
      const unsigned c = (dc >> (4 * t)) & 15u;
      if (!c) break;
      const int d = nb.at(c);
      for (int i = 0; i < 8; ++i) {
        const int q = line[d].dep[i];
        if (q < 0) break;
        if (q == r) { atomicOr(&line[d].rpos, (unsigned)t << (4 * i)); break; }
      }
    }
  }
}

// Slot positions, stream power: consumer d's gated receiver q at position p
// sets bit p of q's mask for d; d's rec sets d's bit in its water flags.
__global__ void k_spl_slotpos(int nx, int ny, SplLine* __restrict__ line) {
  const int nn = nx * ny;
  for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < nn; d += gridDim.x * blockDim.x) {
    const NbrDecoder nb(d, nx, ny);
    const unsigned qc = line[d].q;
    auto index_in_deps = [&](int q) {
      for (int i = 0; i < 8; ++i) {
        const int v = line[q].dep[i];
        if (v < 0) break;
        if (v == d) return i;
      }
      return -1;
    };
    for (int p = 0; p < 8; ++p) {
      const unsigned c = (qc >> (4 * p)) & 15u;
      if (!c) break;
      const int q = nb.at(c);
      const int i = index_in_deps(q);
      if (i >= 0) atomicOr(&line[q].qmask[i >> 2], 1u << (8 * (i & 3) + p));
    }
    const unsigned rcode = (unsigned)line[d].meta & 15u;
    if (rcode) {
      const int r = nb.at(rcode);
      const int i = index_in_deps(r);
      if (i >= 0) atomicOr(&line[r].wflag, 1u << i);
    }
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
// The new elevation of node k is hnew[k * stride].
__global__ void k_spl_finish(int nn, double dt, const double* __restrict__ hnew, int stride, double* __restrict__ h,
                             double* __restrict__ b, double* __restrict__ etot, double* __restrict__ erate,
                             double* __restrict__ sedflux) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const double ht = h[k], hn = hnew[(size_t)k * stride];
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

// What a coefficient kernel stores for one equation a*z(t-1) + bb*z(t) +
// c*z(t+1) = f.  Plain (T = double): the coefficients and f.  Mixed
// precision (T = float): the coefficients rounded to float and, in place of
// f, the residual r = f - (a*z0(t-1) + bb*z0(t) + c*z0(t+1)) of the current
// surface z0, evaluated in FP64; the FP32 solve then gives the increment
// z - z0, which is added to z0 in FP64.
template <class T>
__device__ inline void store_equation(T* A, T* B, T* C, T* F, size_t o, double a, double bb, double c, double f,
                                      double zm, double z0, double zp) {
  if constexpr (sizeof(T) == sizeof(double)) {
    A[o] = a; B[o] = bb; C[o] = c; F[o] = f;
  } else {
    const double r = f - (a * zm + bb * z0 + c * zp);
    A[o] = (T)a; B[o] = (T)bb; C[o] = (T)c; F[o] = (T)r;
  }
}

// One equation a*z(t-1) + bb*z(t) + c*z(t+1) = f of the x pass (row j, column
// i; Diffusion.f90:45-86) and of the y pass (column i, row j; :97-138), in
// the reference's arithmetic.  z0m, z0, z0p are the current surface at
// t-1, t, t+1 (0 off the grid), for the mixed form's residual.
struct Equation {
  double a, bb, c, f, zm, z0, zp;
};
__device__ inline Equation x_equation(const Bounds& bd, double dt2, double dx2, double dy2,
                                      const double* __restrict__ K, const double* __restrict__ z, int i, int j) {
  const int nx = bd.nx;
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
  return {a, bb, c, f, i > 0 ? Z(i - 1, j) : 0.0, Z(i, j), i < nx - 1 ? Z(i + 1, j) : 0.0};
}
__device__ inline Equation y_equation(const Bounds& bd, double dt2, double dx2, double dy2,
                                      const double* __restrict__ K, const double* __restrict__ z, int i, int j) {
  const int nx = bd.nx, ny = bd.ny;
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
  return {a, bb, c, f, j > 0 ? Z(i, j - 1) : 0.0, Z(i, j), j < ny - 1 ? Z(i, j + 1) : 0.0};
}

// x pass coefficients for rows j=1..ny-2, stored transposed: element i of
// row j at [i*ny + j]
template <class T>
__global__ void k_diff_xcoef(Bounds bd, double dt2, double dx2, double dy2, const double* __restrict__ K,
                             const double* __restrict__ z, T* __restrict__ A, T* __restrict__ B,
                             T* __restrict__ C, T* __restrict__ F) {
  const int nx = bd.nx, ny = bd.ny;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y + 1;
  if (i >= nx || j > ny - 2) return;
  const Equation e = x_equation(bd, dt2, dx2, dy2, K, z, i, j);
  store_equation(A, B, C, F, (size_t)i * ny + j, e.a, e.bb, e.c, e.f, e.zm, e.z0, e.zp);
}

// y pass coefficients for columns i=1..nx-2 (natural layout [j*nx + i])
template <class T>
__global__ void k_diff_ycoef(Bounds bd, double dt2, double dx2, double dy2, const double* __restrict__ K,
                             const double* __restrict__ z, T* __restrict__ A, T* __restrict__ B,
                             T* __restrict__ C, T* __restrict__ F) {
  const int nx = bd.nx, ny = bd.ny;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i < 1 || i > nx - 2 || j >= ny) return;
  const Equation e = y_equation(bd, dt2, dx2, dy2, K, z, i, j);
  store_equation(A, B, C, F, (size_t)j * nx + i, e.a, e.bb, e.c, e.f, e.zm, e.z0, e.zp);
}

// tridag (Diffusion.f90:164-202) for independent systems s in [s0, s1):
// element t of system s at [t*L + s]; the solution overwrites F.  A block
// of 32 threads solves 32 systems, one each (the recurrence is sequential,
// and its arithmetic is the reference's).  Coefficients move through shared
// memory in chunks of kTC steps, double-buffered: the next chunk's copies
// are in flight while the recurrence runs through the current one, so it
// waits on its divisions, not on DRAM.  Every lane touches only its own
// column of the buffers.
constexpr int kTC = 16;
__device__ inline void cp_async_elem(double* smem, const double* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}

__device__ inline void cp_async_elem(float* smem, const float* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem));
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }

template <int N>
__device__ inline void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <class T>
__global__ void __launch_bounds__(32) k_thomas(int N, int L, int s0, int s1, const T* __restrict__ A,
                                               const T* __restrict__ B, const T* __restrict__ C,
                                               T* __restrict__ F, T* __restrict__ G,
                                               int* __restrict__ err) {
  __shared__ T sa[2][kTC][33], sb[2][kTC][33], sc[2][kTC][33], sf[2][kTC][33];
  const int lane = threadIdx.x;
  const int s = s0 + blockIdx.x * 32 + lane;
  const bool act = s < s1;
  // forward elimination
  auto load_fwd = [&](int buf, int t0) {
    const int tn = min(kTC, N - t0);
    if (act)
      for (int r = 0; r < tn; ++r) {
        const size_t o = (size_t)(t0 + r) * L + s;
        cp_async_elem(&sa[buf][r][lane], &A[o]);
        cp_async_elem(&sb[buf][r][lane], &B[o]);
        cp_async_elem(&sf[buf][r][lane], &F[o]);
        if (t0 + r > 0) cp_async_elem(&sc[buf][r][lane], &C[o - L]);
      }
    cp_async_commit();
  };
  T bet = 0, up = 0;
  bool bad = false;
  load_fwd(0, 0);
  for (int t0 = 0, k = 0; t0 < N; t0 += kTC, ++k) {
    const int buf = k & 1;
    const int tn = min(kTC, N - t0);
    if (t0 + kTC < N) {
      load_fwd(buf ^ 1, t0 + kTC);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();
    if (act && !bad) {
      for (int r = 0; r < tn; ++r) {
        const int t = t0 + r;
        if (t == 0) {
          bet = sb[buf][0][lane];
          if (bet == 0.0) { bad = true; break; }
          up = sf[buf][0][lane] / bet;
          sf[buf][0][lane] = up;
          sc[buf][0][lane] = 0.0;
        } else {
          const T g = sc[buf][r][lane] / bet;
          sc[buf][r][lane] = g;
          bet = sb[buf][r][lane] - sa[buf][r][lane] * g;
          if (bet == 0.0) { bad = true; break; }
          up = (sf[buf][r][lane] - sa[buf][r][lane] * up) / bet;
          sf[buf][r][lane] = up;
        }
      }
    }
    if (act)
      for (int r = 0; r < tn; ++r) {
        const size_t o = (size_t)(t0 + r) * L + s;
        F[o] = sf[buf][r][lane];
        G[o] = sc[buf][r][lane];
      }
    __syncwarp();
  }
  if (bad) { atomicExch(err, DEV_TRIDAG_ZERO); return; }
  // back substitution u(t) = u(t) - gam(t+1)*u(t+1), chunked from the end;
  // this lane's forward stores are visible to its own later loads
  auto load_bwd = [&](int buf, int t1) {
    const int tlo = max(0, t1 - kTC);
    if (act)
      for (int r = 0; r < t1 - tlo; ++r) {
        const size_t o = (size_t)(tlo + r) * L + s;
        cp_async_elem(&sf[buf][r][lane], &F[o]);
        cp_async_elem(&sc[buf][r][lane], &G[o + L]);
      }
    cp_async_commit();
  };
  if (act) up = F[(size_t)(N - 1) * L + s];
  if (N > 1) load_bwd(0, N - 1);
  for (int t1 = N - 1, k = 0; t1 > 0; t1 -= kTC, ++k) {
    const int buf = k & 1;
    const int tlo = max(0, t1 - kTC);
    const int tn = t1 - tlo;
    if (tlo > 0) {
      load_bwd(buf ^ 1, tlo);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncwarp();
    if (act)
      for (int r = tn - 1; r >= 0; --r) {
        up = sf[buf][r][lane] - sc[buf][r][lane] * up;
        sf[buf][r][lane] = up;
      }
    if (act)
      for (int r = 0; r < tn; ++r) F[(size_t)(tlo + r) * L + s] = sf[buf][r][lane];
    __syncwarp();
  }
}

// zint = x-pass result on rows 1..ny-2, h elsewhere (natural layout); in the
// mixed form the solve gave the increment, added to h in FP64
template <class T>
__global__ void k_diff_xgather(Bounds bd, const T* __restrict__ Ux, const double* __restrict__ h,
                               double* __restrict__ zint) {
  __shared__ T tile[32][33];
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
      if constexpr (sizeof(T) == sizeof(double))
        zint[o] = (j >= 1 && j <= ny - 2) ? tile[threadIdx.x][r] : h[o];
      else
        zint[o] = (j >= 1 && j <= ny - 2) ? h[o] + (double)tile[threadIdx.x][r] : h[o];
    }
  }
}

// mixed form of k_diff_finish: zintp = zint + the y-pass increment on columns
// 1..nx-2, h elsewhere
__global__ void k_diff_finish_m(Bounds bd, double dt, const float* __restrict__ dUy, const double* __restrict__ zint,
                                double* __restrict__ h, double* __restrict__ b, double* __restrict__ etot,
                                double* __restrict__ erate) {
  const int nx = bd.nx, nn = nx * bd.ny;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    const int i = k % nx;
    const double hk = h[k];
    const double zp = (i >= 1 && i <= nx - 2) ? zint[k] + (double)dUy[k] : hk;
    etot[k] = etot[k] + hk - zp;
    erate[k] = erate[k] + (hk - zp) / dt;
    h[k] = zp;
    b[k] = fmin(zp, b[k]);
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

void mfd_receivers(Ctx& c) {
  const int nn = c.nn;
  if (c.mixed)
    k_mfd_receivers<true><<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.p, c.hwater, c.ltab, c.mrec, c.mnrec, c.mwrec,
                                                               c.mlrec);
  else
    k_mfd_receivers<false><<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.p, c.hwater, c.ltab, c.mrec, c.mnrec,
                                                                c.mwrec, c.mlrec);
  c.count_launch();
  if (c.capture) {  // a topological order of mrec (the reference's mstack is a LIFO Kahn order)
    k_order_keys<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.stack, c.hwater, c.o_keys, c.o_vals);
    c.count_launch();
    sort_pairs_u64(c, c.o_keys, c.o_keys2, c.o_vals, c.o_vals2, nn);
    k_order_finish<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.o_vals2, c.o_pos, c.mstack);
    c.count_launch();
  }
}

template <int LANES, int SIDE_DIV, class Op>
static void run_sweep(Ctx& c, Op op, const int* cnt0) {
  const int nn = c.nn;
  op.slots = c.slots;
  op.err = c.d_err;
  cudaMemsetAsync(c.slots, 0xff, sizeof(double) * kSlotStride * (size_t)nn, c.stream);  // all slots empty
  cudaMemcpyAsync(c.la_cnt, cnt0, sizeof(int) * nn, cudaMemcpyDeviceToDevice, c.stream);
  cudaMemsetAsync(c.la_queue, 0xff, sizeof(int) * nn, c.stream);
  cudaMemsetAsync(c.la_ctl, 0, sizeof(unsigned) * 128, c.stream);
  k_seed_queue<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, cnt0, c.la_queue, c.la_ctl + 32);
  const int blocks = std::max(8, std::min(148 * 4, (int)std::sqrt((double)nn) / SIDE_DIV));
  k_last_arriver<Op, LANES><<<blocks, 128, 0, c.stream>>>(op, nn, c.la_cnt, c.la_queue, c.la_ctl, c.d_err);
  c.count_launch(2);
}

void fill_sweep(Ctx& c) { fill_chains(c); }

// Single-flow area with uniform precipitation P: the reference's loop
// (FlowRouting.f90:133-139) adds multiples m*v of v = dx*dy*P, m <= 2*nn.  When
// v's odd significand M has M*2*nn <= 2^53, every such partial sum is exact,
// so a(k) = v*size(k) (doubled at a root) bit for bit, whatever the order.
static bool exact_size_area(const Ctx& c, double& v) {
  if (!c.precip_uniform) return false;
  v = c.dx * c.dy * c.precip_value;
  if (!std::isfinite(v)) return false;
  if (v == 0.0) return true;
  int e = 0;
  const double f = std::frexp(std::fabs(v), &e);               // v = f * 2^e, f in [0.5, 1)
  unsigned long long M = (unsigned long long)std::ldexp(f, 53);  // exact: f has at most 53 bits
  while (!(M & 1ull)) M >>= 1;
  return (double)M * 2.0 * (double)c.nn <= 9007199254740992.0;
}

__global__ void k_area_from_size(int nn, double v, const int* __restrict__ size, const int* __restrict__ rec,
                                 double* __restrict__ a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nn; k += gridDim.x * blockDim.x) {
    double x = v * (double)size[k];
    if (rec[k] == k) x = x + x;
    a[k] = x;
  }
}

void accumulate(Ctx& c) {
  if (c.sfd) {
    double v = 0.0;
    if (exact_size_area(c, v)) {
      k_area_from_size<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, v, c.size, c.rec, c.a);
      c.count_launch();
    } else {
      area_chains(c);
    }
    return;
  }
  if (region_accumulate(c)) return;
  AccLine* line = static_cast<AccLine*>(c.mfd_line);
  k_acc_lines<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, c.dx * c.dy, c.mrec, c.mnrec, c.mwrec, c.precip, c.size,
                                                     line, c.cnt_acc, c.d_err);
  c.count_launch();
  k_acc_slotpos<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, line);
  c.count_launch();
  run_sweep<FSB_LANES_ACC, FSB_SIDE_DIV_ACC>(c, AccMfdOp{line, c.a, 0}, c.cnt_acc);
}

void gs_erosion_mfd(Ctx& c, const double* e, const int* sill, double* lsed, double* dh) {
  AccLine* line = static_cast<AccLine*>(c.mfd_line);
  k_acc_lines<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, 1.0, c.mrec, c.mnrec, c.mwrec, e, c.size, line,
                                                     c.cnt_acc, c.d_err);
  c.count_launch();
  k_acc_slotpos<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, line);
  c.count_launch();
  AccMfdOp op{line, dh, 0};
  op.gs = 1;
  op.rec = c.rec;
  op.sill = sill;
  op.lsed = lsed;
  run_sweep<FSB_LANES_ACC, FSB_SIDE_DIV_ACC>(c, op, c.cnt_acc);
}

void spl_mfd_gs(Ctx& c, const double* elev, const double* hstart, int* sill, double* contrib) {
  const int n1 = fabs(c.n - 1.0) < DBL_MIN;
  SplLine* line = static_cast<SplLine*>(c.mfd_line);
  k_spl_lines<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, n1, c.kfsed, c.dt, c.m, c.n, c.rec, c.mrec, c.mnrec, c.mwrec,
                                                     c.mlrec, c.h, c.b, c.kf, c.a, c.size, line, c.cnt_spl, c.d_err);
  c.count_launch();
  k_spl_slotpos<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, line);
  c.count_launch();
  SplMfdOp<true> op{line, NewtonPow{c.n, c.n == 1.5}, 0.875 / c.n, n1,
                    reinterpret_cast<double2*>(c.hw)};
  op.elev = elev;
  op.hstart = hstart;
  op.sill = sill;
  op.contrib = contrib;
  run_sweep<FSB_LANES_SPL, FSB_SIDE_DIV_SPL>(c, op, c.cnt_spl);
}

void flux_mfd(Ctx& c, double* flux) {
  AccLine* line = static_cast<AccLine*>(c.mfd_line);
  k_acc_lines<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, 1.0, c.mrec, c.mnrec, c.mwrec, c.erate, c.size, line,
                                                     c.cnt_acc, c.d_err);
  c.count_launch();
  k_acc_slotpos<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, line);
  c.count_launch();
  run_sweep<FSB_LANES_ACC, FSB_SIDE_DIV_ACC>(c, AccMfdOp{line, flux, 1}, c.cnt_acc);
}

void stream_power(Ctx& c) {
  const int n1 = fabs(c.n - 1.0) < DBL_MIN;
  const double omega = 0.875 / c.n;
  if (c.sfd) {
    spl_chains(c, c.hnew);
    k_spl_finish<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, c.dt, c.hnew, 1, c.h, c.b, c.etot, c.erate, c.sedflux);
    c.count_launch();
    return;
  }
  if (region_stream_power(c)) return;
  // the erosion factors need the drainage area: the lines are built now
  SplLine* line = static_cast<SplLine*>(c.mfd_line);
  k_spl_lines<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.bd, n1, c.kfsed, c.dt, c.m, c.n, c.rec, c.mrec, c.mnrec, c.mwrec,
                                                     c.mlrec, c.h, c.b, c.kf, c.a, c.size, line, c.cnt_spl, c.d_err);
  c.count_launch();
  k_spl_slotpos<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nx, c.ny, line);
  c.count_launch();
  double2* hw = reinterpret_cast<double2*>(c.hw);
  run_sweep<FSB_LANES_SPL, FSB_SIDE_DIV_SPL>(c, SplMfdOp<false>{line, NewtonPow{c.n, c.n == 1.5}, omega, n1, hw},
                                             c.cnt_spl);
  k_spl_finish<<<grid1d(c.nn), kBlock, 0, c.stream>>>(c.nn, c.dt, c.hw, 2, c.h, c.b, c.etot, c.erate, c.sedflux);
  c.count_launch();
}

void thomas_lines(Ctx& c, int N, int L, int s0, int s1, const double* A, const double* B, const double* C, double* F,
                  double* G) {
  if (s1 <= s0) return;
  k_thomas<double><<<(s1 - s0 + 31) / 32, 32, 0, c.stream>>>(N, L, s0, s1, A, B, C, F, G, c.d_err);
  c.count_launch();
}

// Mixed-precision ADI step: coefficients as in the plain form, each line
// solved in FP32 for the increment of the surface against the FP64 residual
// of the current surface, the increment added in FP64.
static void diffusion_mixed(Ctx& c) {
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  const double dt2 = c.dt / 2.0, dx2 = c.dx * c.dx, dy2 = c.dy * c.dy;
  double *K = c.dK, *Z = c.dZ;
  float *A = reinterpret_cast<float*>(c.dA), *B = reinterpret_cast<float*>(c.dB),
        *C = reinterpret_cast<float*>(c.dC), *F = reinterpret_cast<float*>(c.dF),
        *G = reinterpret_cast<float*>(c.dG);
  k_diff_kdint<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.kdsed, c.kd, c.h, c.b, K);
  dim3 gx((nx + 127) / 128, ny - 2);
  k_diff_xcoef<float><<<gx, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, c.h, A, B, C, F);
  stage_begin(c, KT_THOMAS_ROWS);
  k_thomas<float><<<(ny - 2 + 31) / 32, 32, 0, c.stream>>>(nx, ny, 1, ny - 1, A, B, C, F, G, c.d_err);
  stage_end(c, KT_THOMAS_ROWS);
  dim3 g2((nx + 31) / 32, (ny + 31) / 32);
  k_diff_xgather<float><<<g2, dim3(32, 8), 0, c.stream>>>(c.bd, F, c.h, Z);
  dim3 gy((nx + 127) / 128, ny);
  k_diff_ycoef<float><<<gy, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, Z, A, B, C, F);
  stage_begin(c, KT_THOMAS_COLS);
  k_thomas<float><<<(nx - 2 + 31) / 32, 32, 0, c.stream>>>(ny, nx, 1, nx - 1, A, B, C, F, G, c.d_err);
  stage_end(c, KT_THOMAS_COLS);
  k_diff_finish_m<<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.dt, F, Z, c.h, c.b, c.etot, c.erate);
  c.count_launch(7);
}

void diffusion(Ctx& c) {
  if (c.mixed) {
    diffusion_mixed(c);
    return;
  }
  const int nx = c.nx, ny = c.ny, nn = c.nn;
  const double dt2 = c.dt / 2.0, dx2 = c.dx * c.dx, dy2 = c.dy * c.dy;
  double *K = c.dK, *A = c.dA, *B = c.dB, *C = c.dC, *F = c.dF, *G = c.dG, *Z = c.dZ;
  k_diff_kdint<<<grid1d(nn), kBlock, 0, c.stream>>>(nn, c.kdsed, c.kd, c.h, c.b, K);
  c.count_launch();
  {
    dim3 g((nx + 127) / 128, ny - 2);
    k_diff_xcoef<double><<<g, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, c.h, A, B, C, F);
    // systems are rows j=1..ny-2 with element i at [i*ny + j]
    stage_begin(c, KT_THOMAS_ROWS);
    k_thomas<double><<<(ny - 2 + 31) / 32, 32, 0, c.stream>>>(nx, ny, 1, ny - 1, A, B, C, F, G, c.d_err);
    stage_end(c, KT_THOMAS_ROWS);
    dim3 g2((nx + 31) / 32, (ny + 31) / 32);
    k_diff_xgather<double><<<g2, dim3(32, 8), 0, c.stream>>>(c.bd, F, c.h, Z);
    c.count_launch(3);
  }
  {
    dim3 g((nx + 127) / 128, ny);
    k_diff_ycoef<double><<<g, 128, 0, c.stream>>>(c.bd, dt2, dx2, dy2, K, Z, A, B, C, F);
    stage_begin(c, KT_THOMAS_COLS);
    k_thomas<double><<<(nx - 2 + 31) / 32, 32, 0, c.stream>>>(ny, nx, 1, nx - 1, A, B, C, F, G, c.d_err);
    stage_end(c, KT_THOMAS_COLS);
    c.count_launch(2);
  }
  k_diff_finish<<<grid1d(nn), kBlock, 0, c.stream>>>(c.bd, c.dt, F, c.h, c.b, c.etot, c.erate);
  c.count_launch();
}

// The same ADI step on caller-supplied arrays: `scratch` holds 7*nx*ny
// doubles (kdint, the four coefficient arrays, the forward factors and the
// x-pass result); `err` receives DEV_TRIDAG_ZERO on a zero pivot.
void diffusion_raw(const Bounds& bd, double dx, double dy, double dt, double kdsed, const double* kd, double* h,
                   double* b, double* etot, double* erate, double* scratch, int* err, cudaStream_t st) {
  const int nx = bd.nx, ny = bd.ny, nn = nx * ny;
  const double dt2 = dt / 2.0, dx2 = dx * dx, dy2 = dy * dy;
  double* K = scratch;
  double* A = K + nn;
  double* B = A + nn;
  double* C = B + nn;
  double* F = C + nn;
  double* G = F + nn;
  double* Z = G + nn;
  k_diff_kdint<<<grid1d(nn), kBlock, 0, st>>>(nn, kdsed, kd, h, b, K);
  dim3 gx((nx + 127) / 128, ny - 2);
  k_diff_xcoef<double><<<gx, 128, 0, st>>>(bd, dt2, dx2, dy2, K, h, A, B, C, F);
  k_thomas<double><<<(ny - 2 + 31) / 32, 32, 0, st>>>(nx, ny, 1, ny - 1, A, B, C, F, G, err);
  dim3 gt((nx + 31) / 32, (ny + 31) / 32);
  k_diff_xgather<double><<<gt, dim3(32, 8), 0, st>>>(bd, F, h, Z);
  dim3 gy((nx + 127) / 128, ny);
  k_diff_ycoef<double><<<gy, 128, 0, st>>>(bd, dt2, dx2, dy2, K, Z, A, B, C, F);
  k_thomas<double><<<(nx - 2 + 31) / 32, 32, 0, st>>>(ny, nx, 1, nx - 1, A, B, C, F, G, err);
  k_diff_finish<<<grid1d(nn), kBlock, 0, st>>>(bd, dt, F, h, b, etot, erate);
}

}  // namespace fsb
