// Device-resident state of one continental-step instance and the launchers
// that operate on it.  One Ctx mirrors the reference's FastScapeContext module
// (src/FastScape_ctx.f90:9-36) for the arrays the continental step touches.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <utility>

#include "fsb_common.cuh"

namespace fsb {

constexpr int kBlock = 256;
constexpr int kSlotStride = 16;  // doubles per node in Ctx::slots

inline unsigned grid1d(size_t n, int block = kBlock) {
  size_t g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;  // grid-stride loops beyond 64 blocks per SM
  if (g == 0) g = 1;
  return (unsigned)g;
}

// Tile-major numbering of the grid for the region-owned sweeps (fsb_region.cu):
// tiles of 2^ltx x 2^lty nodes, tile t = ty*ntx + tx, node (i, j) at
// g = t*2^(ltx+lty) + (j mod 2^lty)*2^ltx + (i mod 2^ltx).  Slots of partial
// tiles beyond the grid are padding.
struct TileMap {
  int nx = 0, ny = 0;
  int ltx = 0, lty = 0;
  int ntx = 0, nty = 0;  // ntx == 0: no plan
  __host__ __device__ int lr() const { return ltx + lty; }
  __host__ __device__ int tiles() const { return ntx * nty; }
  __host__ __device__ long long padded() const { return (long long)tiles() << lr(); }
  __host__ __device__ int g(int i, int j) const {
    const int t = (j >> lty) * ntx + (i >> ltx);
    return (t << lr()) | ((j & ((1 << lty) - 1)) << ltx) | (i & ((1 << ltx) - 1));
  }
};

struct Ctx {
  // ---- configuration (setters of FastScape_ctx.f90) ----
  int nx = 0, ny = 0, nn = 0;
  int ibc = 1111;
  Bounds bd{};
  double xl = 0, yl = 0, dt = 0, kfsed = -1, m = 0, n = 1, kdsed = -1, g1 = 0, g2 = 0, p = 0;
  double dx = 0, dy = 0;
  bool sfd = false, runSPL = false, runDiffusion = false, runUplift = false;
  bool setup_done = false;
  // mixed precision (fsb_set_precision): FP32 weights, area, Newton iterations
  // and tridiagonal solves; FP64 state, h update and residuals
  bool mixed = false;
  int launch_share = 1;  // 1: alone on the device; 4: beside other instances (persistent sweeps take 1/4 the blocks)
  bool capture = false;  // keep LocalMinima intermediates of the last step
  bool routed = false;   // a step has built receivers, stack, chains and area
  bool precip_uniform = true;  // every node has precipitation precip_value (SetUp: 1)
  double precip_value = 1.0;
  int step = 0;
  cudaStream_t stream = 0;
  long long launches = 0;  // kernels launched by this instance
  void count_launch(long long k = 1) { launches += k; }

  // ---- device arena ----
  char* arena = nullptr;
  size_t arena_bytes = 0;
  bool owns_arena = false;

  // ---- persistent fields (nn each unless noted) ----
  double *h = nullptr, *b = nullptr, *u = nullptr, *kf = nullptr, *kd = nullptr, *precip = nullptr;
  double *etot = nullptr, *erate = nullptr, *a = nullptr, *length = nullptr, *lake_depth = nullptr;
  double *hwater = nullptr, *sedflux = nullptr;
  double *catch0 = nullptr, *catchv = nullptr;  // catchment seeds (SetUp) and labels (ctx:17,94)
  double* red = nullptr;                         // 3*512 partial sums + 3 results (reductions)
  double* g = nullptr;                           // sediment parameter per node (ctx:17), kept across steps
  double *vx = nullptr, *vy = nullptr;           // advection velocities (ctx:17, SetV)
  bool runAdvect = false;
  bool g_positive = false;                       // max(g) > 0 at the last stream-power call
  int ngs = 0;                                   // Gauss-Seidel iterations of the last call
  int *rec = nullptr, *ndon = nullptr, *don = nullptr /*8*nn*/, *stack = nullptr;
  int *pos = nullptr, *size = nullptr;
  int *mrec = nullptr /*8*nn*/, *mnrec = nullptr, *mstack = nullptr, *mdmask = nullptr;
  double *mwrec = nullptr /*8*nn*/, *mlrec = nullptr /*8*nn*/;
  double* ltab = nullptr;  // 9 neighbour lengths of find_receiver / find_mult_rec

  // ---- captured intermediates (debug / parity) ----
  int *rec_pre = nullptr, *stack_pre = nullptr, *basins = nullptr, *outlets = nullptr;
  double* length_pre = nullptr;

  // ---- scratch ----
  int *s_flag = nullptr, *s_scan = nullptr, *s_roots = nullptr, *s_root_rank = nullptr;
  unsigned long long *s_list_a = nullptr, *s_list_b = nullptr;  // 2*nn each
  // list ranking by sublist walks: predecessor flags (2*nn bytes), the
  // splitter lists (ping-pong) and the count of list heads
  unsigned char* s_rank_pred = nullptr;
  unsigned long long *s_rank_sa = nullptr, *s_rank_sb = nullptr;
  unsigned* s_rank_nheads = nullptr;
  // LocalMinima
  size_t conn_cap = 0;       // capacity of edge arrays
  size_t hash_cap = 0;       // capacity (power of two) of the basin-pair hash
  unsigned long long *ht_key = nullptr, *ht_wmin = nullptr;
  unsigned *ht_first = nullptr, *ht_best = nullptr;
  int *e_b1 = nullptr, *e_b2 = nullptr, *e_n1 = nullptr, *e_n2 = nullptr;
  double* e_w = nullptr;
  unsigned *e_key = nullptr, *e_key2 = nullptr;
  int *e_idx = nullptr, *e_idx2 = nullptr;
  int *o_b1 = nullptr, *o_b2 = nullptr, *o_n1 = nullptr, *o_n2 = nullptr;  // oriented copies
  int *r_b1 = nullptr, *r_b2 = nullptr, *r_n1 = nullptr, *r_n2 = nullptr;  // unsorted edges
  double* r_w = nullptr;
  int* nr_bsum = nullptr;  // per-block stopper totals of the cooperative NR sort
  int nr_bsum_cap = 0;
  int *nr_idx = nullptr, *nr_idx2 = nullptr, *nr_lf = nullptr, *nr_rf = nullptr, *nr_ls = nullptr,
      *nr_rs = nullptr, *nr_lpos = nullptr, *nr_rpos = nullptr, *nr_segof = nullptr;
  int *nr_seg = nullptr, *nr_seg2 = nullptr;  // segments: pairs (l, ir), 1-based
  int *nr_small = nullptr;                    // small segments (l, ir)
  int *nr_med = nullptr;                      // segments of 8..512 elements (l, ir), finished in shared memory
  double* nr_piv = nullptr;
  int* nr_segmeta = nullptr;  // per segment: pv, i, j, T
  int* nr_child = nullptr;    // per level segment: i, left id, right id, j (cooperative levels)
  int *e_rank = nullptr, *e_inmst = nullptr, *tree = nullptr;
  int *mst_comp = nullptr, *mst_min = nullptr, *mst_next = nullptr;
  int *arc_deg = nullptr, *arc_start = nullptr, *arc_slot = nullptr, *arc_adj = nullptr;
  // MFD order
  unsigned long long *o_keys = nullptr, *o_keys2 = nullptr;
  int *o_vals = nullptr, *o_vals2 = nullptr, *o_pos = nullptr;
  // heavy-path chain schedule (fsb_chains.cu)
  int *ch_heavy = nullptr, *ch_tmp = nullptr, *ch_tmp2 = nullptr, *ch_nxt = nullptr, *ch_nxt2 = nullptr;
  unsigned long long *ch_val = nullptr, *ch_val2 = nullptr;
  int *ch_ord = nullptr, *ch_pos = nullptr, *ch_ldep = nullptr, *ch_start = nullptr, *ch_cid = nullptr,
      *ch_sid = nullptr, *ch_hist = nullptr, *ch_goff = nullptr, *ch_tk_td = nullptr, *ch_tk_bu = nullptr;
  unsigned *ch_key = nullptr, *ch_skey = nullptr;
  int nchains = 0, ntickets_td = 0, ntickets_bu = 0, nroots = 0;
  bool chains_valid = false;  // the chain schedule matches the current forest
  // last-arriver sweeps (multiple flow)
  int *la_queue = nullptr, *la_cnt = nullptr, *cnt_acc = nullptr, *cnt_spl = nullptr;
  void* mfd_line = nullptr;  // one 128-byte record per node (area, then stream power)
  double* hw = nullptr;      // (elevation, water surface) pairs of the stream-power sweep
  double* slots = nullptr;   // kSlotStride input slots per node of the multiple-flow sweeps
  // region-owned sweeps (fsb_region.cu): tile plan and tile-major buffers
  static constexpr int kMaxPlans = 3;
  TileMap tplans[kMaxPlans] = {};  // candidate plans (smallest tiles first)
  int ntplans = 0;
  TileMap tplan_of[8] = {};        // per sweep op: the tuned plan (ntx == 0: not yet)
  int tform_of[8] = {};            // per sweep op: the tuned kernel form (0: one node per warp)
  bool region_enabled = true;  // use them when the plan and a cooperative launch allow
  signed char region_ok[8] = {};  // per sweep op: 0 unchecked, 1 usable, -1 not on this device
  void* rl_line = nullptr;     // one 128-byte line per tile-major slot
  double* rl_val = nullptr;    // 2 doubles per slot: area, or (h, water)
  unsigned char* rl_cnt0 = nullptr;  // initial counters, one byte per slot
  int* rl_xcnt = nullptr;      // cross-tile inputs per slot
  int* rl_inbox = nullptr;     // per tile: nodes whose cross-tile inputs are all in
  unsigned* rl_itail = nullptr;
  int rl_icap = 0;
  unsigned* la_ctl = nullptr;  // head, tail, done count
  int* s_scan2 = nullptr;
  // sweeps
  unsigned *done = nullptr;  // epoch flags per node
  unsigned epoch = 0;
  unsigned* ticket = nullptr;
  double* water = nullptr;
  double* hnew = nullptr;  // elevation written by the stream-power sweep
  // diffusion scratch: kdint, tridiagonal coefficients, forward factors, x-pass result
  double *dK = nullptr, *dA = nullptr, *dB = nullptr, *dC = nullptr, *dF = nullptr, *dG = nullptr, *dZ = nullptr;
  // counters on device and their pinned host mirror
  int* d_err = nullptr;   // device error word
  int* d_cnt = nullptr;   // small device counters
  int* h_cnt = nullptr;   // pinned host mirror of d_cnt
  void* cub_tmp = nullptr;
  size_t cub_tmp_bytes = 0;

  // last LocalMinima counts (host)
  int nbasins = 0, basin0 = 0, nconn = 0, tree_size = 0, nlocmin_before = 0, nlocmin_after = 0;

  // per-stage device timing (CUDA events on the instance's stream)
  // stages: uplift receivers stack locmin fill mfd accum spl diffusion advection;
  // then single kernels inside them: the area sweep, the stream-power sweep,
  // the row and the column tridiagonal solves of the diffusion, the lake fill
  // sweep
  static constexpr int kStages = 15;
  bool profile = false;
  cudaEvent_t ev_begin[kStages] = {}, ev_end[kStages] = {};
  bool ev_pending[kStages] = {};
  double stage_ms[kStages] = {};
  long long stage_calls[kStages] = {};

  std::string err;
};

// per-stage / per-kernel CUDA events while profiling is on (fsb_api.cu)
enum { KT_AREA_SWEEP = 10, KT_SPL_SWEEP = 11, KT_THOMAS_ROWS = 12, KT_THOMAS_COLS = 13, KT_FILL = 14 };
void stage_begin(Ctx& c, int s);
void stage_end(Ctx& c, int s);

// sets the message fsb_last_error() returns; returns 1 (fsb_api.cu)
int report_error(const std::string& msg);

// routing (fsb_routing.cu)
void launch_uplift(Ctx& c);
void launch_find_receiver(Ctx& c, const double* h, int* rec, double* length);
void launch_find_donors(Ctx& c, const int* rec, int* ndon, int* don);
void build_stack(Ctx& c, const int* rec, int* ndon, int* don, int* stack, int* pos, int* size);
unsigned long long* list_rank(Ctx& c, size_t n, unsigned long long* a, unsigned long long* b);
// list ranking by sublist walks: a splitter every kRankStride entries plus each
// list head (at most kRankMaxHeads heads)
constexpr int kRankStride = 16;
constexpr int kRankMaxHeads = 64;
inline size_t rank_splitter_cap(size_t n) { return (n + kRankStride - 1) / kRankStride + kRankMaxHeads; }

// primitives (fsb_prims.cu)
void exclusive_scan_int(Ctx& c, const int* in, int* out, size_t n);
void exclusive_scan_u32(Ctx& c, const unsigned* in, unsigned* out, size_t n);
void inclusive_scan_int(Ctx& c, const int* in, int* out, size_t n);
void sort_pairs_u32(Ctx& c, const unsigned* kin, unsigned* kout, const int* vin, int* vout, size_t n, int end_bit);
void sort_pairs_u64(Ctx& c, const unsigned long long* kin, unsigned long long* kout, const int* vin,
                    int* vout, size_t n);
size_t cub_temp_bytes_needed(size_t nn, size_t nconn);
void fetch_counters(Ctx& c, int n);  // d_cnt[0..n) -> h_cnt (synchronises the stream)

// LocalMinima (fsb_locmin.cu); returns false and sets c.err on failure
bool local_minima(Ctx& c);

// chains (fsb_chains.cu)
void build_chains(Ctx& c);          // heavy-first order + ticket lists of the current forest
void ensure_chains(Ctx& c);         // build_chains unless the schedule is current
void fill_chains(Ctx& c);
void area_chains(Ctx& c);
void spl_chains(Ctx& c, double* hnew);
void flux_chains(Ctx& c, double* flux);               // compute_fluxes' flux, single flow
void chi_chains(Ctx& c, double a0, double mn, double* chi);
void flux_mfd(Ctx& c, double* flux);                  // compute_fluxes' flux, multiple flow
// tridiagonal systems s0..s1-1, element t of system s at [t*L + s], F solved in place
// region-owned multiple-flow sweeps (fsb_region.cu); false: not usable, the
// queue engine of fsb_flow.cu runs instead
int plan_tiles(int nx, int ny, int sms, TileMap* out, int max_plans);
bool region_accumulate(Ctx& c);
bool region_stream_power(Ctx& c);
void thomas_lines(Ctx& c, int N, int L, int s0, int s1, const double* A, const double* B, const double* C, double* F,
                  double* G);
void advect(Ctx& c);  // fsb_advect.cu
int write_vtk(Ctx& c, const double* f_dev, double vex, const char* dir);  // fsb_vtk.cu
// the stream power law with the sediment term g > 0 (fsb_sediment.cu)
bool gs_active(const Ctx& c);
int stream_power_gs(Ctx& c);
void spl_chains_gs(Ctx& c, const double* elev, const double* hstart, double* hnew, int* sill, double* contrib);
void gs_erosion_chains(Ctx& c, const double* hp, const int* sill, double* lsed, double* dh);
void lake_volume_chains(Ctx& c, const int* sill, const double* contrib, double* vol, double* up);
void gs_erosion_mfd(Ctx& c, const double* e, const int* sill, double* lsed, double* dh);
void spl_mfd_gs(Ctx& c, const double* elev, const double* hstart, int* sill, double* contrib);
// derived fields (fsb_derived.cu)
void catchment(Ctx& c);                               // catch = catch0 of the root, before LocalMinima
void slope_field(Ctx& c, double* out);
void curvature_field(Ctx& c, double* out);
void add_layers(Ctx& c, const double* dh);
void flux_sums(Ctx& c, const double* flux, double* part, double* out3);

// flow (fsb_flow.cu)
void fill_sweep(Ctx& c);            // hwater along the stack (SFD lake fill / MFD h0)
void mfd_receivers(Ctx& c);         // find_mult_rec: mrec, mnrec, mlrec, mwrec, order
void accumulate(Ctx& c);            // drainage area
void stream_power(Ctx& c);          // implicit stream power law (g == 0)
void diffusion(Ctx& c);             // ADI hillslope diffusion
void diffusion_raw(const Bounds& bd, double dx, double dy, double dt, double kdsed, const double* kd, double* h,
                   double* b, double* etot, double* erate, double* scratch, int* err, cudaStream_t st);

}  // namespace fsb
