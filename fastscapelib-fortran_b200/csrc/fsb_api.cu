// C ABI of the continental step (include/fastscape_b200.h): instance
// lifecycle, setters, the step driver and copy-outs, plus the reference's own
// Fortran entry points on a process-wide instance.
//
// The step driver follows FastScape_Execute_Step (src/FastScape_api.f90:201-263)
// with advection, marine and stratigraphy switched off.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cfloat>
#include <string>
#include <vector>
#include <algorithm>
#include <mutex>

#include "fsb_kernels.cuh"
#include "../../include/fastscape_b200.h"

struct fsb_ctx {
  fsb::Ctx c;
};

namespace {

// Small pinned host buffers (counter read-backs) are recycled across
// instances instead of freed: freeing pinned memory synchronises the device,
// which would stall the other instances' streams.
std::mutex g_pinned_mu;
std::vector<int*> g_pinned_free;

int* pinned_counters() {
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  if (g_pinned_free.empty()) {
    const int kBuffers = 64;
    int* block = nullptr;
    if (cudaMallocHost((void**)&block, sizeof(int) * 32 * kBuffers) != cudaSuccess) return nullptr;
    for (int k = kBuffers - 1; k >= 0; --k) g_pinned_free.push_back(block + 32 * k);
  }
  int* p = g_pinned_free.back();
  g_pinned_free.pop_back();
  return p;
}

void recycle_counters(int* p) {
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  g_pinned_free.push_back(p);
}

thread_local std::string g_err;

int fail(const std::string& msg) {
  g_err = msg;
  return 1;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(std::string(what) + ": " + cudaGetErrorString(e));
}

#define FSB_CUDA(call)                                      \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
  } while (0)

// SetBC (FastScape_ctx.f90:565-593): write(cbc,'(i4)') and digit tests
void decode_bc(fsb::Ctx& c, int jbc) {
  char cbc[16];
  if (jbc > 9999 || jbc < -999) std::strcpy(cbc, "****");
  else std::snprintf(cbc, sizeof cbc, "%4d", jbc);
  fsb::Bounds& b = c.bd;
  b.nx = c.nx;
  b.ny = c.ny;
  b.fix_bottom = cbc[0] == '1';
  b.fix_right = cbc[1] == '1';
  b.fix_top = cbc[2] == '1';
  b.fix_left = cbc[3] == '1';
  b.i1 = b.fix_left ? 1 : 0;
  b.i2 = b.fix_right ? c.nx - 2 : c.nx - 1;
  b.j1 = b.fix_bottom ? 1 : 0;
  b.j2 = b.fix_top ? c.ny - 2 : c.ny - 1;
  b.xcyc = !b.fix_left && !b.fix_right;
  b.ycyc = !b.fix_bottom && !b.fix_top;
  c.ibc = jbc;
}

struct Layout {
  char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) & ~(size_t)255;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

// Assigns every device buffer of the instance inside `base` (or only sizes
// them when base is null) and returns the arena size.
size_t layout(fsb::Ctx& c, char* base) {
  const size_t N = (size_t)c.nn;
  Layout L{base};
  size_t hcap = 1024;
  while (hcap < 8 * N) hcap <<= 1;
  c.hash_cap = hcap;
  c.conn_cap = 5 * N + 64;
  const size_t E = c.conn_cap;
  c.h = L.take<double>(N); c.b = L.take<double>(N); c.u = L.take<double>(N);
  c.kf = L.take<double>(N); c.kd = L.take<double>(N); c.precip = L.take<double>(N);
  c.etot = L.take<double>(N); c.erate = L.take<double>(N); c.a = L.take<double>(N);
  c.length = L.take<double>(N); c.lake_depth = L.take<double>(N); c.hwater = L.take<double>(N);
  c.sedflux = L.take<double>(N);
  c.rec = L.take<int>(N); c.ndon = L.take<int>(N); c.don = L.take<int>(8 * N); c.stack = L.take<int>(N);
  c.pos = L.take<int>(N); c.size = L.take<int>(N);
  c.mrec = L.take<int>(8 * N); c.mnrec = L.take<int>(N); c.mstack = L.take<int>(N); c.mdmask = L.take<int>(N);
  c.mwrec = L.take<double>(8 * N); c.mlrec = L.take<double>(8 * N);
  c.ltab = L.take<double>(48);  // 9 lengths; their n-th powers at +16 (double) and +32 (float)
  c.rec_pre = L.take<int>(N); c.stack_pre = L.take<int>(N); c.basins = L.take<int>(N);
  c.length_pre = L.take<double>(N);
  c.s_flag = L.take<int>(N + 1); c.s_scan = L.take<int>(N + 1); c.s_roots = L.take<int>(N);
  c.s_root_rank = L.take<int>(N);
  c.s_list_a = L.take<unsigned long long>(2 * N); c.s_list_b = L.take<unsigned long long>(2 * N);
  c.s_rank_sa = L.take<unsigned long long>(fsb::rank_splitter_cap(2 * N));
  c.s_rank_sb = L.take<unsigned long long>(fsb::rank_splitter_cap(2 * N));
  c.s_rank_nheads = L.take<unsigned>(1);
  c.s_rank_pred = L.take<unsigned char>(2 * N + fsb::kRankStride);  // whole 16-byte flag groups
  c.ht_key = L.take<unsigned long long>(hcap); c.ht_wmin = L.take<unsigned long long>(hcap);
  c.ht_first = L.take<unsigned>(hcap); c.ht_best = L.take<unsigned>(hcap);
  c.e_b1 = L.take<int>(E); c.e_b2 = L.take<int>(E); c.e_n1 = L.take<int>(E); c.e_n2 = L.take<int>(E);
  c.e_w = L.take<double>(E);
  c.e_key = L.take<unsigned>(E); c.e_key2 = L.take<unsigned>(E);
  c.e_idx = L.take<int>(E); c.e_idx2 = L.take<int>(E);
  c.o_b1 = L.take<int>(E); c.o_b2 = L.take<int>(E); c.o_n1 = L.take<int>(E); c.o_n2 = L.take<int>(E);
  c.r_b1 = L.take<int>(E); c.r_b2 = L.take<int>(E); c.r_n1 = L.take<int>(E); c.r_n2 = L.take<int>(E);
  c.r_w = L.take<double>(E);
  c.nr_idx = L.take<int>(E + 2); c.nr_idx2 = L.take<int>(E + 2);
  c.nr_lf = L.take<int>(E + 2); c.nr_rf = L.take<int>(E + 2);
  c.nr_ls = L.take<int>(E + 2); c.nr_rs = L.take<int>(E + 2);
  c.nr_lpos = L.take<int>(E + 2); c.nr_rpos = L.take<int>(E + 2);
  c.nr_segof = L.take<int>(E + 2);
  c.nr_seg = L.take<int>(E + 8); c.nr_seg2 = L.take<int>(E + 8); c.nr_small = L.take<int>(E + 16);
  c.nr_med = L.take<int>(2 * (E / 8 + 8));
  c.nr_piv = L.take<double>(E / 2 + 8); c.nr_segmeta = L.take<int>(2 * E + 32);
  c.nr_child = L.take<int>(4 * ((E + 2) / 512 + 16));  // level segments hold > 512 keys
  c.nr_bsum_cap = 2 * 4096; c.nr_bsum = L.take<int>(c.nr_bsum_cap);
  c.e_rank = L.take<int>(E); c.e_inmst = L.take<int>(E); c.tree = L.take<int>(N);
  c.mst_comp = L.take<int>(N); c.mst_min = L.take<int>(N); c.mst_next = L.take<int>(N);
  c.arc_deg = L.take<int>(N + 1); c.arc_start = L.take<int>(N + 1); c.arc_slot = L.take<int>(2 * N);
  c.arc_adj = L.take<int>(2 * N);
  c.o_keys = L.take<unsigned long long>(N); c.o_keys2 = L.take<unsigned long long>(N);
  c.o_vals = L.take<int>(N); c.o_vals2 = L.take<int>(N); c.o_pos = L.take<int>(N);
  c.ch_heavy = L.take<int>(N); c.ch_tmp = L.take<int>(N + 1); c.ch_tmp2 = L.take<int>(N + 1);
  c.ch_nxt = L.take<int>(N); c.ch_nxt2 = L.take<int>(N);
  c.ch_val = L.take<unsigned long long>(N); c.ch_val2 = L.take<unsigned long long>(N);
  c.ch_ord = L.take<int>(N); c.ch_pos = L.take<int>(N); c.ch_ldep = L.take<int>(N); c.ch_start = L.take<int>(N);
  c.ch_cid = L.take<int>(N); c.ch_sid = L.take<int>(N); c.ch_hist = L.take<int>(128); c.ch_goff = L.take<int>(128);
  c.ch_tk_td = L.take<int>(N + 2048); c.ch_tk_bu = L.take<int>(N + 2048);
  c.ch_key = L.take<unsigned>(2 * N); c.ch_skey = L.take<unsigned>(N);
  c.la_queue = L.take<int>(N); c.la_cnt = L.take<int>(N); c.cnt_acc = L.take<int>(N); c.cnt_spl = L.take<int>(N);
  c.la_ctl = L.take<unsigned>(128);
  c.mfd_line = L.take<double>(16 * N); c.hw = L.take<double>(2 * N);
  c.slots = L.take<double>(fsb::kSlotStride * N);
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    c.ntplans = fsb::plan_tiles(c.nx, c.ny, sms, c.tplans, fsb::Ctx::kMaxPlans);
    for (auto& t : c.tplan_of) t = fsb::TileMap{};
    for (auto& f : c.tform_of) f = 0;
    size_t P = 0;
    int T = 0;
    c.rl_icap = 0;
    for (int i = 0; i < c.ntplans; ++i) {  // buffers for the largest of the candidate plans
      P = std::max(P, (size_t)c.tplans[i].padded());
      T = std::max(T, c.tplans[i].tiles());
      c.rl_icap = std::max(c.rl_icap, 2 * ((1 << c.tplans[i].ltx) + (1 << c.tplans[i].lty)) + 16);
    }
    c.rl_line = L.take<double>(16 * P);
    c.rl_val = L.take<double>(2 * P);
    c.rl_cnt0 = L.take<unsigned char>(P);
    c.rl_xcnt = L.take<int>(P);
    c.rl_inbox = L.take<int>((size_t)T * c.rl_icap);
    c.rl_itail = L.take<unsigned>((size_t)T);
  }
  c.s_scan2 = L.take<int>(N + 1);
  c.done = L.take<unsigned>(N); c.ticket = L.take<unsigned>(4);
  c.water = L.take<double>(N); c.hnew = L.take<double>(N);
  c.catch0 = L.take<double>(N); c.catchv = L.take<double>(N); c.red = L.take<double>(3 * 512 + 8);
  c.g = L.take<double>(N); c.vx = L.take<double>(N); c.vy = L.take<double>(N);
  c.dK = L.take<double>(N); c.dA = L.take<double>(N); c.dB = L.take<double>(N); c.dC = L.take<double>(N);
  c.dF = L.take<double>(N); c.dG = L.take<double>(N); c.dZ = L.take<double>(N);
  c.d_err = L.take<int>(4); c.d_cnt = L.take<int>(32);
  c.cub_tmp_bytes = fsb::cub_temp_bytes_needed(N, E);
  c.cub_tmp = L.take<char>(c.cub_tmp_bytes);
  return L.off + 256;
}

double xorshift_uniform(unsigned long long& s) {
  s ^= s << 13; s ^= s >> 7; s ^= s << 17;
  return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

int upload(fsb::Ctx& c, double* dst, const double* src, int where) {
  if (!src) return fail("null array");
  const cudaMemcpyKind kind = where == FSB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  FSB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * c.nn, kind, c.stream));
  if (where != FSB_DEVICE) FSB_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int need_setup(fsb_ctx* h, const char* who) {
  if (!h) return fail("null fsb_ctx");
  if (!h->c.setup_done) return fail(std::string(who) + " - You need to run SetUp first");
  return 0;
}

double* field_ptr(fsb::Ctx& c, int f) {
  switch (f) {
    case FSB_H: return c.h;
    case FSB_BASEMENT: return c.b;
    case FSB_TOTAL_EROSION: return c.etot;
    case FSB_DRAINAGE_AREA: return c.a;
    case FSB_EROSION_RATE: return c.erate;
    case FSB_LAKE_DEPTH: return c.lake_depth;
    case FSB_LENGTH: return c.length;
    case FSB_HWATER: return c.hwater;
    case FSB_SEDFLUX: return c.sedflux;
    case FSB_CATCHMENT: return c.catchv;
    case FSB_U: return c.u;
    case FSB_PRECIP: return c.precip;
    case FSB_KF: return c.kf;
    case FSB_KD: return c.kd;
    default: return nullptr;
  }
}

int check_device_error(fsb::Ctx& c) {
  int e = 0;
  FSB_CUDA(cudaMemcpyAsync(&e, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  FSB_CUDA(cudaGetLastError());
  if (e != 0) {
    cudaMemsetAsync(c.d_err, 0, sizeof(int), c.stream);
    switch (e) {
      case fsb::DEV_SPIN_LIMIT: return fail("device: a bounded wait gave up (dependency never published)");
      case fsb::DEV_STACK_ERROR: return fail("error in stack");
      case fsb::DEV_TRIDAG_ZERO: return fail("tridag failed");
      case fsb::DEV_OVERFLOW: return fail("device: buffer overflow");
      case fsb::DEV_NOT_ADJACENT: return fail("device: a receiver is not a neighbour of its donor");
      case fsb::DEV_NEWTON_LIMIT:
        return fail("stream power law: a Newton solve did not converge within " +
                    std::to_string(fsb::kNewtonLimit) + " iterations");
      default: return fail("device error " + std::to_string(e));
    }
  }
  return 0;
}

enum { ST_UPLIFT, ST_RECEIVERS, ST_STACK, ST_LOCMIN, ST_FILL, ST_MFD, ST_ACCUM, ST_SPL, ST_DIFFUSION, ST_ADVECT };

}  // namespace

namespace fsb {
void stage_begin(Ctx& c, int s) {
  if (!c.profile) return;
  if (!c.ev_begin[s]) {
    cudaEventCreate(&c.ev_begin[s]);
    cudaEventCreate(&c.ev_end[s]);
  }
  cudaEventRecord(c.ev_begin[s], c.stream);
}

void stage_end(Ctx& c, int s) {
  if (!c.profile) return;
  cudaEventRecord(c.ev_end[s], c.stream);
  c.ev_pending[s] = true;
}
}  // namespace fsb

namespace {
using fsb::stage_begin;
using fsb::stage_end;

void collect_stage_times(fsb::Ctx& c) {
  for (int s = 0; s < fsb::Ctx::kStages; ++s) {
    if (!c.ev_pending[s]) continue;
    float ms = 0.f;
    if (cudaEventSynchronize(c.ev_end[s]) == cudaSuccess &&
        cudaEventElapsedTime(&ms, c.ev_begin[s], c.ev_end[s]) == cudaSuccess) {
      c.stage_ms[s] += ms;
      c.stage_calls[s] += 1;
    }
    c.ev_pending[s] = false;
  }
}

int step_once(fsb::Ctx& c) {
  if (c.runAdvect) {  // Advect first (FastScape_api.f90:209-214)
    stage_begin(c, ST_ADVECT);
    fsb::advect(c);
    stage_end(c, ST_ADVECT);
  }
  if (c.runUplift) {
    stage_begin(c, ST_UPLIFT);
    fsb::launch_uplift(c);
    stage_end(c, ST_UPLIFT);
  }
  if (c.runSPL) {
    c.dx = c.xl / (c.nx - 1);
    c.dy = c.yl / (c.ny - 1);
    double lt[16] = {0};
    for (int jj = -1; jj <= 1; ++jj)
      for (int ii = -1; ii <= 1; ++ii) {
        const double ax = c.dx * ii, ay = c.dy * jj;
        lt[(jj + 1) * 3 + (ii + 1)] = std::sqrt(ax * ax + ay * ay);
      }
    FSB_CUDA(cudaMemcpyAsync(c.ltab, lt, sizeof lt, cudaMemcpyHostToDevice, c.stream));
    stage_begin(c, ST_RECEIVERS);
    fsb::launch_find_receiver(c, c.h, c.rec, c.length);
    stage_end(c, ST_RECEIVERS);
    stage_begin(c, ST_STACK);
    fsb::build_stack(c, c.rec, c.ndon, c.don, c.stack, c.pos, c.size);
    stage_end(c, ST_STACK);
    stage_begin(c, ST_LOCMIN);
    const bool ok = fsb::local_minima(c);
    stage_end(c, ST_LOCMIN);
    if (!ok) { g_err = c.err; return 1; }
    stage_begin(c, ST_FILL);
    c.chains_valid = false;  // a new forest
    fsb::ensure_chains(c);
    fsb::fill_sweep(c);
    stage_end(c, ST_FILL);
    if (!c.sfd) {
      stage_begin(c, ST_MFD);
      fsb::mfd_receivers(c);
      stage_end(c, ST_MFD);
    }
    stage_begin(c, ST_ACCUM);
    fsb::accumulate(c);
    stage_end(c, ST_ACCUM);
    stage_begin(c, ST_SPL);
    if (fsb::gs_active(c)) {
      if (fsb::stream_power_gs(c)) return 1;
    } else {
      fsb::stream_power(c);
      c.ngs = 1;
    }
    stage_end(c, ST_SPL);
  }
  if (c.runDiffusion) {
    c.dx = c.xl / (c.nx - 1);
    c.dy = c.yl / (c.ny - 1);
    stage_begin(c, ST_DIFFUSION);
    fsb::diffusion(c);
    stage_end(c, ST_DIFFUSION);
  }
  c.step += 1;
  if (c.runSPL) c.routed = true;
  const int rc = check_device_error(c);
  collect_stage_times(c);
  return rc;
}

}  // namespace

namespace fsb {
// lets other translation units report through fsb_last_error()
int report_error(const std::string& msg) { return fail(msg); }
}  // namespace fsb

extern "C" {

const char* fsb_last_error(void) { return g_err.c_str(); }

int fsb_create(fsb_ctx** out) {
  if (!out) return fail("null output pointer");
  *out = new fsb_ctx();
  return 0;
}

static void release(fsb::Ctx& c) {
  for (int s = 0; s < fsb::Ctx::kStages; ++s) {
    if (c.ev_begin[s]) cudaEventDestroy(c.ev_begin[s]);
    if (c.ev_end[s]) cudaEventDestroy(c.ev_end[s]);
    c.ev_begin[s] = c.ev_end[s] = nullptr;
    c.ev_pending[s] = false;
  }
  if (c.owns_arena && c.arena) cudaFree(c.arena);
  if (c.h_cnt) recycle_counters(c.h_cnt);
  c.arena = nullptr;
  c.h_cnt = nullptr;
  c.owns_arena = false;
  c.setup_done = false;
}

int fsb_destroy(fsb_ctx* h) {
  if (!h) return 0;
  release(h->c);
  delete h;
  return 0;
}

int fsb_set_nx_ny(fsb_ctx* h, int nx, int ny) {
  if (!h) return fail("null fsb_ctx");
  h->c.nx = nx;
  h->c.ny = ny;
  return 0;
}

int fsb_workspace_bytes(fsb_ctx* h, size_t* bytes) {
  if (!h || !bytes) return fail("null argument");
  fsb::Ctx& c = h->c;
  if (c.nx < 3 || c.ny < 3) return fail("FastScapeSetup - You need to set nx and ny (>= 3) first");
  if ((long long)c.nx * c.ny > (1ll << 28)) return fail("grid too large (nx*ny > 2^28)");
  c.nn = c.nx * c.ny;
  fsb::Ctx tmp = c;
  *bytes = layout(tmp, nullptr);
  return 0;
}

int fsb_set_stream(fsb_ctx* h, void* stream) {
  if (!h) return fail("null fsb_ctx");
  h->c.stream = (cudaStream_t)stream;
  return 0;
}

// FastScape_Setup -- ctx:57-113
int fsb_setup(fsb_ctx* h, void* arena, size_t bytes) {
  if (!h) return fail("null fsb_ctx");
  fsb::Ctx& c = h->c;
  if (c.nx == 0) return fail("FastScapeSetup - You need to set nx first");
  if (c.ny == 0) return fail("FastScapeSetup - You need to set ny first");
  size_t need = 0;
  if (fsb_workspace_bytes(h, &need)) return 1;
  cudaStream_t keep_stream = c.stream;
  release(c);
  c.stream = keep_stream;
  if (arena) {
    if (bytes < need) return fail("fsb_setup: arena smaller than fsb_workspace_bytes()");
    c.arena = (char*)arena;
    c.owns_arena = false;
  } else {
    FSB_CUDA(cudaMalloc((void**)&c.arena, need));
    c.owns_arena = true;
  }
  c.arena_bytes = need;
  layout(c, c.arena);
  // zero the whole arena once so that no index array ever holds garbage
  FSB_CUDA(cudaMemsetAsync(c.arena, 0, need, c.stream));
  c.h_cnt = pinned_counters();
  if (!c.h_cnt) return fail("pinned host memory for the counters could not be allocated");
  // defaults of SetUp
  decode_bc(c, 1111);
  std::vector<double> hv(c.nn);
  unsigned long long s = 0x9E3779B97F4A7C15ull;
  for (int i = 0; i < c.nn; ++i) hv[i] = xorshift_uniform(s);
  for (int i = 0; i < c.nx; ++i) { hv[i] = 0.0; hv[(size_t)c.nx * (c.ny - 1) + i] = 0.0; }
  for (int j = 0; j < c.ny; ++j) { hv[(size_t)j * c.nx] = 0.0; hv[(size_t)j * c.nx + c.nx - 1] = 0.0; }
  FSB_CUDA(cudaMemcpyAsync(c.h, hv.data(), sizeof(double) * c.nn, cudaMemcpyHostToDevice, c.stream));
  FSB_CUDA(cudaMemcpyAsync(c.b, hv.data(), sizeof(double) * c.nn, cudaMemcpyHostToDevice, c.stream));
  // catch0 continues the same stream (SetUp's second random_number, ctx:94)
  std::vector<double> cv(c.nn);
  for (int i = 0; i < c.nn; ++i) cv[i] = xorshift_uniform(s);
  FSB_CUDA(cudaMemcpyAsync(c.catch0, cv.data(), sizeof(double) * c.nn, cudaMemcpyHostToDevice, c.stream));
  std::vector<double> ones(c.nn, 1.0);
  FSB_CUDA(cudaMemcpyAsync(c.precip, ones.data(), sizeof(double) * c.nn, cudaMemcpyHostToDevice, c.stream));
  for (double* f : {c.u, c.etot, c.erate, c.a, c.length, c.lake_depth, c.hwater, c.sedflux, c.kf, c.kd, c.catchv})
    FSB_CUDA(cudaMemsetAsync(f, 0, sizeof(double) * c.nn, c.stream));
  FSB_CUDA(cudaMemsetAsync(c.done, 0, sizeof(unsigned) * c.nn, c.stream));
  FSB_CUDA(cudaMemsetAsync(c.s_flag, 0, sizeof(int) * (c.nn + 1), c.stream));
  FSB_CUDA(cudaMemsetAsync(c.d_err, 0, sizeof(int) * 4, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  c.epoch = 0;
  c.runSPL = c.runDiffusion = c.runUplift = false;
  c.sfd = false;
  c.p = 1.0;
  c.step = 0;
  c.routed = false;
  c.precip_uniform = true;
  c.precip_value = 1.0;
  c.g_positive = false;
  c.ngs = 0;
  c.runAdvect = false;
  c.setup_done = true;
  return 0;
}

int fsb_set_xl_yl(fsb_ctx* h, double xl, double yl) {
  if (!h) return fail("null fsb_ctx");
  h->c.xl = xl;
  h->c.yl = yl;
  return 0;
}

int fsb_set_dt(fsb_ctx* h, double dt) {
  if (!h) return fail("null fsb_ctx");
  h->c.dt = dt;
  return 0;
}

// SetErosionalParam -- ctx:423-450
int fsb_set_erosional_parameters(fsb_ctx* h, const double* kf, double kfsed, double m, double n,
                                 const double* kd, double kdsed, double g1, double g2, double p, int where) {
  if (need_setup(h, "set_erosional_parameters")) return 1;
  fsb::Ctx& c = h->c;
  c.runSPL = true;
  if (upload(c, c.kf, kf, where) || upload(c, c.kd, kd, where)) return 1;
  c.kfsed = kfsed; c.m = m; c.n = n; c.kdsed = kdsed; c.g1 = g1; c.g2 = g2; c.p = p;
  c.sfd = false;
  if (p < -1.5) { c.sfd = true; c.p = 1.0; }
  // runDiffusion when maxval(kd) > tiny or kdsed > tiny
  std::vector<double> hk(c.nn);
  FSB_CUDA(cudaMemcpyAsync(hk.data(), c.kd, sizeof(double) * c.nn, cudaMemcpyDeviceToHost, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  double mx = -DBL_MAX;
  for (double v : hk) mx = std::max(mx, v);
  if (mx > DBL_MIN || kdsed > DBL_MIN) c.runDiffusion = true;
  return 0;
}

int fsb_set_precision(fsb_ctx* h, int precision) {
  if (!h) return fail("null fsb_ctx");
  if (precision != FSB_PREC_FP64 && precision != FSB_PREC_MIXED)
    return fail("set_precision: precision must be FSB_PREC_FP64 or FSB_PREC_MIXED");
  h->c.mixed = precision == FSB_PREC_MIXED;
  return 0;
}

int fsb_set_concurrency(fsb_ctx* h, int instances) {
  if (!h) return fail("null fsb_ctx");
  if (instances < 1) return fail("set_concurrency: instances must be at least 1");
  h->c.launch_share = instances > 1 ? 4 : 1;
  return 0;
}

int fsb_get_precision(fsb_ctx* h, int* precision) {
  if (!h || !precision) return fail("null argument");
  *precision = h->c.mixed ? FSB_PREC_MIXED : FSB_PREC_FP64;
  return 0;
}

int fsb_set_bc(fsb_ctx* h, int bc) {
  if (need_setup(h, "set_bc")) return 1;
  decode_bc(h->c, bc);
  return 0;
}

int fsb_set_v(fsb_ctx* h, const double* vx, const double* vy, int where) {
  if (need_setup(h, "SetV")) return 1;
  if (upload(h->c, h->c.vx, vx, where) || upload(h->c, h->c.vy, vy, where)) return 1;
  h->c.runAdvect = true;
  return 0;
}

int fsb_set_u(fsb_ctx* h, const double* u, int where) {
  if (need_setup(h, "set_u")) return 1;
  h->c.runUplift = true;
  return upload(h->c, h->c.u, u, where);
}

int fsb_init_h(fsb_ctx* h, const double* hp, int where) {
  if (need_setup(h, "InitH")) return 1;
  if (upload(h->c, h->c.h, hp, where)) return 1;
  FSB_CUDA(cudaMemcpyAsync(h->c.b, h->c.h, sizeof(double) * h->c.nn, cudaMemcpyDeviceToDevice, h->c.stream));
  return 0;
}

int fsb_set_h(fsb_ctx* h, const double* hp, int where) {
  if (need_setup(h, "SetH")) return 1;
  return upload(h->c, h->c.h, hp, where);
}

int fsb_set_basement(fsb_ctx* h, const double* bp, int where) {
  if (need_setup(h, "SetBasement")) return 1;
  return upload(h->c, h->c.b, bp, where);
}

int fsb_set_precip(fsb_ctx* h, const double* pp, int where) {
  if (need_setup(h, "SetPrecip")) return 1;
  fsb::Ctx& c = h->c;
  if (upload(c, c.precip, pp, where)) return 1;
  // remember whether the field is uniform (the single-flow area then has an
  // exact closed form, see fsb::accumulate)
  std::vector<double> v(c.nn);
  FSB_CUDA(cudaMemcpyAsync(v.data(), c.precip, sizeof(double) * c.nn, cudaMemcpyDeviceToHost, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  bool uni = true;
  for (int k = 1; k < c.nn && uni; ++k) uni = std::memcmp(&v[k], &v[0], sizeof(double)) == 0;
  c.precip_uniform = uni;
  c.precip_value = v.empty() ? 1.0 : v[0];
  return 0;
}

int fsb_reset_cumulative_erosion(fsb_ctx* h) {
  if (need_setup(h, "ResetCumulativeErosion")) return 1;
  FSB_CUDA(cudaMemsetAsync(h->c.etot, 0, sizeof(double) * h->c.nn, h->c.stream));
  return 0;
}

int fsb_execute_step(fsb_ctx* h) {
  if (need_setup(h, "Execute_Step")) return 1;
  return step_once(h->c);
}

int fsb_execute_steps(fsb_ctx* h, int nsteps) {
  if (need_setup(h, "Execute_Step")) return 1;
  for (int i = 0; i < nsteps; ++i)
    if (step_once(h->c)) return 1;
  return 0;
}

int fsb_get_step(fsb_ctx* h, int* step) {
  if (!h || !step) return fail("null argument");
  *step = h->c.step;
  return 0;
}

int fsb_get_sizes(fsb_ctx* h, int* nx, int* ny) {
  if (!h || !nx || !ny) return fail("null argument");
  *nx = h->c.nx;
  *ny = h->c.ny;
  return 0;
}

int fsb_copy_field(fsb_ctx* h, int field, double* dst, int where) {
  if (need_setup(h, "Copy")) return 1;
  double* src = field_ptr(h->c, field);
  if (!src) return fail("unknown field");
  if (!dst) return fail("null destination");
  const cudaMemcpyKind kind = where == FSB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  FSB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * h->c.nn, kind, h->c.stream));
  if (where != FSB_DEVICE) FSB_CUDA(cudaStreamSynchronize(h->c.stream));
  return 0;
}

static int copy_out(fsb::Ctx& c, const double* src, double* dst, int where) {
  if (!dst) return fail("null destination");
  const cudaMemcpyKind kind = where == FSB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  FSB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * c.nn, kind, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  return check_device_error(c);
}

int fsb_copy_chi(fsb_ctx* h, double* dst, int where) {
  if (need_setup(h, "CopyChi")) return 1;
  fsb::Ctx& c = h->c;
  double* chi = c.hnew;  // free between steps
  if (!c.routed) {
    FSB_CUDA(cudaMemsetAsync(chi, 0, sizeof(double) * c.nn, c.stream));
  } else {
    const double a0 = (c.xl / (c.nx - 1)) * (c.yl / (c.ny - 1)) * 10.0;
    fsb::ensure_chains(c);
    fsb::chi_chains(c, a0, c.m / c.n, chi);
  }
  return copy_out(c, chi, dst, where);
}

int fsb_copy_slope(fsb_ctx* h, double* dst, int where) {
  if (need_setup(h, "CopySlope")) return 1;
  fsb::slope_field(h->c, h->c.dK);
  return copy_out(h->c, h->c.dK, dst, where);
}

int fsb_copy_curvature(fsb_ctx* h, double* dst, int where) {
  if (need_setup(h, "CopyCurvature")) return 1;
  fsb::curvature_field(h->c, h->c.dK);
  return copy_out(h->c, h->c.dK, dst, where);
}

int fsb_get_fluxes(fsb_ctx* h, double* tectonic, double* erosion, double* boundary) {
  if (need_setup(h, "GetFluxes")) return 1;
  if (!tectonic || !erosion || !boundary) return fail("GetFluxes: null output");
  fsb::Ctx& c = h->c;
  double* flux = c.hnew;  // free between steps
  if (!c.routed)          // no stack yet: the flux is erate itself
    FSB_CUDA(cudaMemcpyAsync(flux, c.erate, sizeof(double) * c.nn, cudaMemcpyDeviceToDevice, c.stream));
  else if (c.sfd)
    {
      fsb::ensure_chains(c);
      fsb::flux_chains(c, flux);
    }
  else
    fsb::flux_mfd(c, flux);
  fsb::flux_sums(c, flux, c.red, c.red + 3 * 512);
  double s3[3];
  FSB_CUDA(cudaMemcpyAsync(s3, c.red + 3 * 512, sizeof s3, cudaMemcpyDeviceToHost, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  if (check_device_error(c)) return 1;
  const double surf = c.xl * c.yl / (c.nx - 1) / (c.ny - 1);
  *tectonic = s3[0] * surf;
  *erosion = s3[1] * surf;
  *boundary = s3[2] * surf;
  return 0;
}

int fsb_set_all_layers(fsb_ctx* h, const double* dh, int where) {
  if (need_setup(h, "SetAllLayers")) return 1;
  fsb::Ctx& c = h->c;
  const double* src = dh;
  if (where != FSB_DEVICE) {
    if (upload(c, c.dK, dh, where)) return 1;
    src = c.dK;
  }
  fsb::add_layers(c, src);
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

extern "C++" {
namespace {
template <class T>
std::vector<T> to_host(fsb::Ctx& c, const T* src) {
  std::vector<T> v(c.nn);
  cudaMemcpyAsync(v.data(), src, sizeof(T) * c.nn, cudaMemcpyDeviceToHost, c.stream);
  cudaStreamSynchronize(c.stream);
  return v;
}
void min_mean_max(const std::vector<double>& v, double& lo, double& mean, double& hi) {
  lo = hi = v.empty() ? 0.0 : v[0];
  double s = 0.0;
  for (double x : v) { lo = std::min(lo, x); hi = std::max(hi, x); s += x; }
  mean = v.empty() ? 0.0 : s / v.size();
}
}  // namespace
}  // extern "C++"

int fsb_vtk(fsb_ctx* h, const double* f, int where, double vex, const char* dir) {
  if (need_setup(h, "VTK")) return 1;
  fsb::Ctx& c = h->c;
  const double* fd = f;
  if (where != FSB_DEVICE) {
    if (upload(c, c.dK, f, where)) return 1;
    fd = c.dK;
  }
  return fsb::write_vtk(c, fd, vex, dir);
}

int fsb_get_gs_iterations(fsb_ctx* h, int* n) {
  if (!h || !n) return fail("null argument");
  *n = h->c.ngs;
  return 0;
}

int fsb_view(fsb_ctx* h) {
  if (need_setup(h, "View")) return 1;
  fsb::Ctx& c = h->c;
  double lo, mean, hi, kfm, kdm;
  min_mean_max(to_host(c, c.kf), lo, kfm, hi);
  min_mean_max(to_host(c, c.kd), lo, kdm, hi);
  std::printf(" FastScapeContext:\n");
  std::printf(" nx,ny %d %d\n nn %d\n step %d\n", c.nx, c.ny, c.nn, c.step);
  std::printf(" xl,yl %.15g %.15g\n dt %.15g\n", c.xl, c.yl, c.dt);
  std::printf(" Kf,Kfsed,,m,n,Kd,Kdsed,G1,G2 %.15g %.15g %.15g %.15g %.15g %.15g %.15g %.15g\n", kfm, c.kfsed,
              c.m, c.n, kdm, c.kdsed, c.g1, c.g2);
  std::printf(" ibc %d\n", c.ibc);
  min_mean_max(to_host(c, c.h), lo, mean, hi);
  std::printf(" h %.15g %.15g %.15g\n", lo, mean, hi);
  min_mean_max(to_host(c, c.u), lo, mean, hi);
  std::printf(" u %.15g %.15g %.15g\n", lo, mean, hi);
  std::fflush(stdout);
  return 0;
}

int fsb_debug(fsb_ctx* h) {
  if (need_setup(h, "Debug")) return 1;
  fsb::Ctx& c = h->c;
  const std::vector<int> rec = to_host(c, c.rec), ndon = to_host(c, c.ndon), stack = to_host(c, c.stack);
  long long nil = 0, sdon = 0, self = 0, minima = 0;
  std::vector<char> seen(c.nn, 0);
  for (int k = 0; k < c.nn; ++k) {
    if (stack[k] >= 0 && stack[k] < c.nn) seen[stack[k]] = 1;
    sdon += ndon[k];
    self += rec[k] == k;
  }
  for (int k = 0; k < c.nn; ++k) nil += !seen[k];  // nodes the stack misses
  for (int j = c.bd.j1; j <= c.bd.j2; ++j)
    for (int i = c.bd.i1; i <= c.bd.i2; ++i) minima += rec[(size_t)j * c.nx + i] == j * c.nx + i;
  std::printf(" --------------------------------------------------------\n");
  std::printf(" Time step %d\n Debug information\n", c.step);
  std::printf(" Total number of nodes (nx*ny) %d\n", c.nn);
  std::printf(" Stack size %d\n", c.routed ? c.nn : 0);
  std::printf(" Number of nil elements in stack %lld\n", c.routed ? nil : 0LL);
  std::printf(" Total number of donors %lld\n Total number of self donors %lld\n", sdon, self);
  std::printf(" Total number of local minima %lld\n", minima);
  std::printf(" Number of Gauss-Siedel iterations (SPL) %d\n", c.ngs);
  std::printf(" Timing (device milliseconds, accumulated while profiling is on):\n");
  static const char* names[] = {"Uplift", "Receivers", "Stack", "LocalMinima", "LakeFill", "MFDReceivers",
                                "DrainageArea", "SPL", "Diffusion", "Advection"};  // stages; kernel timers follow
  for (int s = 0; s < fsb::Ctx::kStages && s < 10; ++s)
    if (c.stage_calls[s]) std::printf(" %s: %.6g\n", names[s], c.stage_ms[s]);
  std::fflush(stdout);
  return 0;
}

int fsb_field_device_ptr(fsb_ctx* h, int field, void** ptr) {
  if (need_setup(h, "field_device_ptr")) return 1;
  double* src = field_ptr(h->c, field);
  if (!src) return fail("unknown field");
  *ptr = src;
  return 0;
}

int fsb_copy_int_field(fsb_ctx* h, int field, int* dst, int where) {
  if (need_setup(h, "Copy")) return 1;
  fsb::Ctx& c = h->c;
  const int* src = nullptr;
  switch (field) {
    case FSB_REC: src = c.rec; break;
    case FSB_NDON: src = c.ndon; break;
    case FSB_STACK: src = c.stack; break;
    case FSB_MNREC: src = c.mnrec; break;
    case FSB_MSTACK: src = c.mstack; break;
    case FSB_BASINS: src = c.basins; break;
    case FSB_REC_PRE: src = c.rec_pre; break;
    case FSB_STACK_PRE: src = c.stack_pre; break;
    default: return fail("unknown int field");
  }
  const cudaMemcpyKind kind = where == FSB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  FSB_CUDA(cudaMemcpyAsync(dst, src, sizeof(int) * c.nn, kind, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int fsb_copy_slots(fsb_ctx* h, int field, void* dst, int where) {
  if (need_setup(h, "Copy")) return 1;
  fsb::Ctx& c = h->c;
  const void* src = nullptr;
  size_t esz = 4;
  switch (field) {
    case FSB_DON: src = c.don; break;
    case FSB_MREC: src = c.mrec; break;
    case FSB_MWREC: src = c.mwrec; esz = 8; break;
    case FSB_MLREC: src = c.mlrec; esz = 8; break;
    default: return fail("unknown slot field");
  }
  const cudaMemcpyKind kind = where == FSB_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  FSB_CUDA(cudaMemcpyAsync(dst, src, esz * 8 * c.nn, kind, c.stream));
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int fsb_set_capture(fsb_ctx* h, int on) {
  if (!h) return fail("null fsb_ctx");
  h->c.capture = on != 0;
  return 0;
}

int fsb_locmin_counts(fsb_ctx* h, int* out6) {
  if (!h || !out6) return fail("null argument");
  fsb::Ctx& c = h->c;
  out6[0] = c.nbasins; out6[1] = c.basin0; out6[2] = c.nconn; out6[3] = c.tree_size;
  out6[4] = c.nlocmin_before; out6[5] = c.nlocmin_after;
  return 0;
}

int fsb_copy_locmin(fsb_ctx* h, int* b1, int* b2, int* n1, int* n2, double* w, int* sort_id, int* tree,
                    int* ob1, int* ob2, int* on1, int* on2) {
  if (need_setup(h, "copy_locmin")) return 1;
  fsb::Ctx& c = h->c;
  const size_t ne = c.nconn, nt = c.tree_size;
  auto cp = [&](void* dst, const void* src, size_t bytes) -> int {
    if (bytes && dst) FSB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c.stream));
    return 0;
  };
  std::vector<int> idx1(ne + 2);
  if (cp(b1, c.e_b1, 4 * ne) || cp(b2, c.e_b2, 4 * ne) || cp(n1, c.e_n1, 4 * ne) || cp(n2, c.e_n2, 4 * ne) ||
      cp(w, c.e_w, 8 * ne) || cp(idx1.data(), c.nr_idx, 4 * (ne + 1)) || cp(tree, c.tree, 4 * nt) ||
      cp(ob1, c.o_b1, 4 * ne) || cp(ob2, c.o_b2, 4 * ne) || cp(on1, c.o_n1, 4 * ne) || cp(on2, c.o_n2, 4 * ne))
    return 1;
  FSB_CUDA(cudaStreamSynchronize(c.stream));
  if (sort_id)
    for (size_t t = 0; t < ne; ++t) sort_id[t] = idx1[t + 1] - 1;
  return 0;
}

int fsb_synchronize(fsb_ctx* h) {
  if (!h) return fail("null fsb_ctx");
  if (!h->c.setup_done) return 0;
  return check_device_error(h->c);
}

long long fsb_launch_count(fsb_ctx* h) { return h ? h->c.launches : 0; }

int fsb_set_profile(fsb_ctx* h, int on) {
  if (!h) return fail("null fsb_ctx");
  h->c.profile = on != 0;
  return 0;
}

int fsb_stage_times(fsb_ctx* h, double* ms, long long* calls, int n, int reset) {
  if (!h) return fail("null fsb_ctx");
  fsb::Ctx& c = h->c;
  for (int s = 0; s < n && s < fsb::Ctx::kStages; ++s) {
    if (ms) ms[s] = c.stage_ms[s];
    if (calls) calls[s] = c.stage_calls[s];
  }
  if (reset)
    for (int s = 0; s < fsb::Ctx::kStages; ++s) { c.stage_ms[s] = 0.0; c.stage_calls[s] = 0; }
  return 0;
}

// ---- the reference's Fortran entry points on a process-wide instance ----------
static fsb_ctx* g_single = nullptr;

static void die_on(int rc) {
  if (rc != 0) {
    std::fprintf(stderr, "%s\n", g_err.c_str());
    std::exit(1);
  }
}

void fastscape_init_(void) {
  if (g_single) fsb_destroy(g_single);
  die_on(fsb_create(&g_single));
}
void fastscape_setup_(void) { die_on(fsb_setup(g_single, nullptr, 0)); }
void fastscape_destroy_(void) {
  if (g_single) {
    release(g_single->c);
    g_single->c.setup_done = false;
  }
}
void fastscape_execute_step_(void) { die_on(fsb_execute_step(g_single)); }
void fastscape_init_h_(double* hp) { die_on(fsb_init_h(g_single, hp, FSB_HOST)); }
void fastscape_copy_h_(double* hp) { die_on(fsb_copy_field(g_single, FSB_H, hp, FSB_HOST)); }
void fastscape_copy_basement_(double* bp) { die_on(fsb_copy_field(g_single, FSB_BASEMENT, bp, FSB_HOST)); }
void fastscape_copy_total_erosion_(double* p) { die_on(fsb_copy_field(g_single, FSB_TOTAL_EROSION, p, FSB_HOST)); }
void fastscape_copy_drainage_area_(double* p) { die_on(fsb_copy_field(g_single, FSB_DRAINAGE_AREA, p, FSB_HOST)); }
void fastscape_copy_erosion_rate_(double* p) { die_on(fsb_copy_field(g_single, FSB_EROSION_RATE, p, FSB_HOST)); }
void fastscape_copy_lake_depth_(double* p) { die_on(fsb_copy_field(g_single, FSB_LAKE_DEPTH, p, FSB_HOST)); }
void fastscape_set_nx_ny_(const int* nnx, const int* nny) {
  if (!g_single) die_on(fsb_create(&g_single));
  die_on(fsb_set_nx_ny(g_single, *nnx, *nny));
}
void fastscape_set_xl_yl_(const double* xxl, const double* yyl) { die_on(fsb_set_xl_yl(g_single, *xxl, *yyl)); }
void fastscape_set_dt_(const double* dtt) { die_on(fsb_set_dt(g_single, *dtt)); }
void fastscape_set_erosional_parameters_(const double* kkf, const double* kkfsed, const double* mm,
                                         const double* nnn, const double* kkd, const double* kkdsed,
                                         const double* gg1, const double* gg2, const double* pp) {
  die_on(fsb_set_erosional_parameters(g_single, kkf, *kkfsed, *mm, *nnn, kkd, *kkdsed, *gg1, *gg2, *pp, FSB_HOST));
}
void fastscape_get_sizes_(int* nnx, int* nny) { die_on(fsb_get_sizes(g_single, nnx, nny)); }
void fastscape_get_step_(int* sstep) { die_on(fsb_get_step(g_single, sstep)); }
void fastscape_set_bc_(const int* jbc) { die_on(fsb_set_bc(g_single, *jbc)); }
void fastscape_set_u_(const double* up) { die_on(fsb_set_u(g_single, up, FSB_HOST)); }
void fastscape_set_v_(const double* ux, const double* uy) { die_on(fsb_set_v(g_single, ux, uy, FSB_HOST)); }
void fastscape_reset_cumulative_erosion_(void) { die_on(fsb_reset_cumulative_erosion(g_single)); }
void fastscape_set_h_(double* hp) { die_on(fsb_set_h(g_single, hp, FSB_HOST)); }
void fastscape_set_basement_(double* bp) { die_on(fsb_set_basement(g_single, bp, FSB_HOST)); }
void fastscape_set_precip_(double* pp) { die_on(fsb_set_precip(g_single, pp, FSB_HOST)); }
void fastscape_copy_chi_(double* p) { die_on(fsb_copy_chi(g_single, p, FSB_HOST)); }
void fastscape_copy_slope_(double* p) { die_on(fsb_copy_slope(g_single, p, FSB_HOST)); }
void fastscape_copy_curvature_(double* p) { die_on(fsb_copy_curvature(g_single, p, FSB_HOST)); }
void fastscape_copy_catchment_(double* p) { die_on(fsb_copy_field(g_single, FSB_CATCHMENT, p, FSB_HOST)); }
void fastscape_get_fluxes_(double* t, double* e, double* b) { die_on(fsb_get_fluxes(g_single, t, e, b)); }
void fastscape_set_all_layers_(double* dh) { die_on(fsb_set_all_layers(g_single, dh, FSB_HOST)); }
void fastscape_view_(void) { die_on(fsb_view(g_single)); }
void fastscape_vtk_(double* fp, double* vexp) { die_on(fsb_vtk(g_single, fp, FSB_HOST, *vexp, nullptr)); }
void fastscape_debug_(void) { die_on(fsb_debug(g_single)); }

}  // extern "C"
