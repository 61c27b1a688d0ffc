/*
 * fastscape_b200.h -- C ABI of the B200 (sm_100a) continental time step of
 * fastscapelib-fortran.
 *
 * Two families of entry points, both plain C with pointers and sizes:
 *
 *  1. fsb_*: handle-based.  One fsb_ctx is one model instance whose state lives
 *     in device memory.  Every call returns 0 on success and a non-zero code on
 *     failure; fsb_last_error() then describes the failure (where the
 *     reference would execute a Fortran `stop`).  Array arguments take a
 *     `where` flag: FSB_HOST for host memory, FSB_DEVICE for device memory.
 *     Node arrays are float64[nx*ny] in the reference layout
 *     ij = i + (j-1)*nx (x fastest), i.e. numpy reshape(ny, nx).
 *
 *  2. fastscape_*_: the reference's own Fortran entry points
 *     (src/FastScape_api.f90), same names as gfortran emits them, every
 *     argument by reference, operating on one process-wide instance.  A
 *     program or f2py wrapper linked against the reference can link against
 *     this library instead.  Like the reference they return nothing: on
 *     failure they print the message and exit(1), as the reference's `stop`.
 *
 * Citations are to fastscapelib-fortran (file:line).
 */
#ifndef FASTSCAPE_B200_H
#define FASTSCAPE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fsb_ctx fsb_ctx;

enum { FSB_HOST = 0, FSB_DEVICE = 1 };

/* float64 node fields for fsb_copy_field / fsb_field_device_ptr */
enum {
  FSB_H = 0,              /* elevation h            FastScape_Copy_H             api:299  */
  FSB_BASEMENT = 1,       /* basement b             FastScape_Copy_Basement      api:315  */
  FSB_TOTAL_EROSION = 2,  /* etot                   FastScape_Copy_Total_Erosion api:331  */
  FSB_DRAINAGE_AREA = 3,  /* a                      FastScape_Copy_Drainage_Area api:347  */
  FSB_EROSION_RATE = 4,   /* erate                  FastScape_Copy_Erosion_Rate  api:363  */
  FSB_LAKE_DEPTH = 5,     /* lake_depth             FastScape_Copy_Lake_Depth    api:459  */
  FSB_LENGTH = 6,         /* receiver distance (internal array length, ctx:17)           */
  FSB_HWATER = 7,         /* filled surface (internal array hwater, ctx:33)              */
  FSB_SEDFLUX = 8,        /* Sedflux (ctx:18)                                            */
  FSB_CATCHMENT = 9,      /* catch: catch0 of the node's root before LocalMinima
                             FastScape_Copy_Catchment api:427 (ctx:297-307, FlowRouting.f90:393-443) */
  FSB_U = 10, FSB_PRECIP = 11, FSB_KF = 12, FSB_KD = 13
};

/* int32 node fields for fsb_copy_int_field (node ids are 0-based: reference - 1) */
enum {
  FSB_REC = 0,        /* rec       (ctx:24)                                  */
  FSB_NDON = 1,       /* ndon      (ctx:24)                                  */
  FSB_STACK = 2,      /* stack     (ctx:24)                                  */
  FSB_MNREC = 3,      /* mnrec     (ctx:34)                                  */
  FSB_MSTACK = 4,     /* mstack    (ctx:34), a topological order, see docs   */
  FSB_BASINS = 5,     /* basin id of every node in the last LocalMinima (1-based ids) */
  FSB_REC_PRE = 6,    /* receivers entering the last LocalMinima          */
  FSB_STACK_PRE = 7   /* stack entering the last LocalMinima              */
};

/* [nn][8] slot fields for fsb_copy_slots (column-major (8,nn) of the reference) */
enum { FSB_DON = 0, FSB_MREC = 1, FSB_MWREC = 2, FSB_MLREC = 3 };

const char* fsb_last_error(void);

/* FastScape_Init (api:146 -> ctx:40-53) */
int fsb_create(fsb_ctx** out);
/* FastScape_Destroy (api:174 -> ctx:117-154); also frees the handle */
int fsb_destroy(fsb_ctx* c);
/* FastScape_Set_NX_NY (api:475 -> ctx:397) */
int fsb_set_nx_ny(fsb_ctx* c, int nx, int ny);
/* Device bytes fsb_setup needs for the current nx, ny (no reference counterpart:
   the reference allocates in SetUp, ctx:68-73). */
int fsb_workspace_bytes(fsb_ctx* c, size_t* bytes);
/* FastScape_Setup (api:160 -> ctx:57-113).  `arena` is caller-owned device
   memory of at least fsb_workspace_bytes(); NULL makes the library allocate
   (and free in fsb_destroy) the arena itself. */
int fsb_setup(fsb_ctx* c, void* arena, size_t bytes);
/* CUDA stream (cudaStream_t) all work of this instance is ordered on. */
int fsb_set_stream(fsb_ctx* c, void* stream);
/* FastScape_Set_XL_YL (api:491 -> ctx:410) */
int fsb_set_xl_yl(fsb_ctx* c, double xl, double yl);
/* FastScape_Set_DT (api:507 -> ctx:476) */
int fsb_set_dt(fsb_ctx* c, double dt);
/* FastScape_Set_Erosional_Parameters (api:523-536 -> ctx:423-450); p < -1.5
   selects single flow direction */
int fsb_set_erosional_parameters(fsb_ctx* c, const double* kf, double kfsed, double m, double n,
                                 const double* kd, double kdsed, double g1, double g2, double p,
                                 int where);
/* FastScape_Set_BC (api:602 -> ctx:565-593) */
int fsb_set_bc(fsb_ctx* c, int bc);
/* FastScape_Set_U (api:618 -> ctx:597-612) */
int fsb_set_u(fsb_ctx* c, const double* u, int where);
/* FastScape_Set_V (api:634 -> ctx:616-632): advection velocities vx, vy;
   switches advection on (Advect.f90, run first in each step) */
int fsb_set_v(fsb_ctx* c, const double* vx, const double* vy, int where);
/* Arithmetic of the step (no counterpart in the reference, which is FP64
   throughout).  FSB_PREC_FP64 (default): every float in FP64, as the
   reference.  FSB_PREC_MIXED: elevation state, the per-step h update and
   the ADI residuals stay FP64, integer routing stays exact; the multiple-flow
   slopes and weights, the drainage area, the stream-power erosion factors and
   Newton iterations (solved for the increment of h) and the tridiagonal
   solves (for the increment of the surface) run in FP32. */
enum { FSB_PREC_FP64 = 0, FSB_PREC_MIXED = 1 };
int fsb_set_precision(fsb_ctx* c, int precision);
int fsb_get_precision(fsb_ctx* c, int* precision);
/* How many instances share the device with this one (no counterpart in the
   reference, which runs one grid at a time).  1 (default): the persistent
   tree sweeps take as many blocks as keep one grid's critical path busy;
   more than 1: a quarter of those, leaving the SMs to the other instances
   (the batch runtime sets its number of workers).  The results do not
   depend on it. */
int fsb_set_concurrency(fsb_ctx* c, int instances);
/* FastScape_Init_H (api:267 -> ctx:339-350): h and basement b */
int fsb_init_h(fsb_ctx* c, const double* h, int where);
/* FastScape_Set_H (api:664 -> ctx:636-644) */
int fsb_set_h(fsb_ctx* c, const double* h, int where);
/* FastScape_Set_Basement (api:696 -> ctx:680-688) */
int fsb_set_basement(fsb_ctx* c, const double* b, int where);
/* FastScape_Set_Precip (api:712 -> ctx:648-656) */
int fsb_set_precip(fsb_ctx* c, const double* precip, int where);
/* FastScape_Reset_Cumulative_Erosion (api:650 -> ctx:368-374) */
int fsb_reset_cumulative_erosion(fsb_ctx* c);
/* FastScape_Execute_Step (api:201-263): uplift, flow routing with depression
   re-routing, drainage area, stream power law, diffusion.  Asynchronous on the
   instance's stream except where data-dependent sizes are read back. */
int fsb_execute_step(fsb_ctx* c);
/* nsteps consecutive FastScape_Execute_Step calls */
int fsb_execute_steps(fsb_ctx* c, int nsteps);
/* FastScape_Get_Step (api:572 -> ctx:501) */
int fsb_get_step(fsb_ctx* c, int* step);
/* FastScape_Get_Sizes (api:556 -> ctx:488) */
int fsb_get_sizes(fsb_ctx* c, int* nx, int* ny);
/* FastScape_Copy_* (api:299-471 -> ctx:158-335): copy a float64 field */
int fsb_copy_field(fsb_ctx* c, int field, double* dst, int where);
/* Device address of a float64 field inside the instance's arena */
int fsb_field_device_ptr(fsb_ctx* c, int field, void** ptr);
/* Integer routing arrays (0-based node ids) for inspection and parity tests */
int fsb_copy_int_field(fsb_ctx* c, int field, int* dst, int where);
/* Slot arrays [nn][8]: int32 for FSB_DON/FSB_MREC (-1 in unused slots),
   float64 for FSB_MWREC/FSB_MLREC */
int fsb_copy_slots(fsb_ctx* c, int field, void* dst, int where);
/* Keep the intermediate LocalMinima arrays of every step (off by default) */
int fsb_set_capture(fsb_ctx* c, int on);
/* counts of the last LocalMinima: nbasins, basin0, nconn, tree_size,
   local minima before and after re-routing (LocalMinima.f90:45,64-67,119-123) */
int fsb_locmin_counts(fsb_ctx* c, int* out6);
/* Arrays of the last LocalMinima (host memory, nconn / tree_size entries):
   connect_basins list (b1,b2 1-based basin ids; n1,n2 0-based nodes, -1 for
   virtual edges; w pass weights), the loc_min_3_indexx permutation (0-based
   edge ids), the Kruskal acceptance order (0-based edge ids) and the edges
   after order_tree. */
int fsb_copy_locmin(fsb_ctx* c, int* b1, int* b2, int* n1, int* n2, double* w, int* sort_id,
                    int* tree, int* ob1, int* ob2, int* on1, int* on2);
/* Blocks until the instance's stream is idle; reports device-side errors */
/* FastScape_Copy_Chi (api:379 -> ctx:228-251): chi along the stack of the last
   step, a0 = 10*dx*dy; zeros before the first step that routed flow. */
int fsb_copy_chi(fsb_ctx* c, double* dst, int where);
/* FastScape_Copy_Slope (api:395 -> ctx:255-272, TerrainDerivatives.f90:3-35), degrees */
int fsb_copy_slope(fsb_ctx* c, double* dst, int where);
/* FastScape_Copy_Curvature (api:411 -> ctx:276-293, TerrainDerivatives.f90:39-74) */
int fsb_copy_curvature(fsb_ctx* c, double* dst, int where);
/* FastScape_Get_Fluxes (api:762 -> ctx:843-886): tectonic, erosion and boundary fluxes */
int fsb_get_fluxes(fsb_ctx* c, double* tectonic, double* erosion, double* boundary);
/* FastScape_Set_All_Layers (api:680 -> ctx:660-676): h and b += dh (no stratigraphy) */
int fsb_set_all_layers(fsb_ctx* c, const double* dh, int where);
/* FastScape_View (api:188 -> ctx:378-393) and FastScape_Debug (api:588 -> ctx:513-561):
   summaries printed to stdout */
/* FastScape_VTK (api:728 -> ctx:692-777): writes <dir>/Topography<step>.vtk
   (and, for vex < 0, Basement<step>.vtk and SeaLevel<step>.vtk) in the legacy
   binary VTK format with big-endian float32 data, exactly as the reference
   built with -fconvert=big-endian; `f` is the extra scalar field (HHHHH),
   `dir` NULL means "VTK" in the current directory, created if missing. */
int fsb_vtk(fsb_ctx* c, const double* f, int where, double vex, const char* dir);
/* Gauss-Seidel iterations of the last stream-power call: the reference's
   nGSStreamPowerLaw (ctx:15, StreamPowerLaw.f90:250-378); 1 when g = 0. */
int fsb_get_gs_iterations(fsb_ctx* c, int* n);
int fsb_view(fsb_ctx* c);
int fsb_debug(fsb_ctx* c);
int fsb_synchronize(fsb_ctx* c);
/* Kernels this instance has launched so far (for throughput accounting) */
long long fsb_launch_count(fsb_ctx* c);
/* Per-stage device timing with CUDA events on the instance's stream, the
   counterpart of the reference's cpu_time accumulators (api:209-257,
   ctx:27).  Stages: 0 uplift, 1 receivers, 2 stack, 3 LocalMinima, 4 lake
   fill, 5 multiple-flow receivers, 6 drainage area, 7 stream power law,
   8 diffusion, 9 advection; then single kernels inside them: 10 the
   multiple-flow area sweep, 11 the multiple-flow stream-power sweep, 12 and
   13 the row and column tridiagonal solves of the diffusion, 14 the lake
   fill sweep.
   fsb_stage_times returns accumulated milliseconds and call counts for the
   first n of these and optionally resets them. */
int fsb_set_profile(fsb_ctx* c, int on);
int fsb_stage_times(fsb_ctx* c, double* ms, long long* calls, int n, int reset);

/* One ADI hillslope-diffusion step on caller-owned device arrays (h, b,
   etot, erate updated in place; kd read) that allocates nothing.  It has no
   counterpart in the reference.  It serves callers that cannot call
   cudaMalloc -- real-time loops that must not stall on the allocator,
   frameworks that own every allocation through their own pools, programs
   that must not grow their device footprint after start-up.  The scratch
   space lives in a static device array of the library sized for
   nx*ny <= 65536 nodes; larger grids are rejected with an error.  Every GPU
   that loads the library holds that array (about 3.7 MB) until exit.  Each
   call looks up the array's device address for the current device and
   context (a query that allocates nothing).  All calls share the array:
   calls that overlap on the GPU race.  The call waits for its work on
   `stream` (a cudaStream_t, may be NULL) to finish, reports a zero pivot as
   an error (fsb_last_error), and refuses to run while an earlier CUDA error
   of the calling thread is pending, leaving that error in place. */
int fsb_diffusion_step_noalloc(int nx, int ny, double xl, double yl, double dt, int bc, double kdsed,
                               const double* kd, double* h, double* b, double* etot, double* erate,
                               void* stream);

/* ---- many grids on one device ----
   No counterpart in the reference, which holds one grid per process
   (src/FastScape_ctx.f90:9-36).  A batch runs jobs -- a grid, its parameters
   and a number of continental steps, each the sequence FastScape_Init /
   Set_NX_NY / Setup / Set_XL_YL / Set_DT / Init_H / Set_Erosional_Parameters /
   Set_U / Set_Precip / Set_BC / Execute_Step x nsteps / Copy_H / Destroy of
   src/FastScape_api.f90 -- on worker threads with one CUDA stream each, so
   that jobs overlap on the GPU.  A job starts when its device workspace fits
   within the batch's memory budget beside the running jobs; jobs start in
   submission order.  Results do not depend on what else runs. */
typedef struct fsb_batch fsb_batch;
typedef struct fsb_job {
  int nx, ny;            /* grid size                                  api:475 */
  int bc;                /* boundary code                              api:602 */
  int nsteps;            /* continental steps to run                   api:201 */
  double xl, yl;         /* domain size                                api:491 */
  double dt;             /* time step                                  api:507 */
  double kfsed, m, n, kdsed, g1, g2, p;  /* erosional scalars          api:523 */
  const double* kf;      /* [nx*ny] host arrays                        api:523 */
  const double* kd;      /* [nx*ny]                                    api:523 */
  const double* u;       /* [nx*ny] uplift rate                        api:618 */
  const double* h0;      /* [nx*ny] initial elevation                  api:267 */
  const double* precip;  /* [nx*ny] or NULL for 1                      api:712 */
  double* h_out;         /* [nx*ny] elevation after nsteps, or NULL    api:299 */
  double* a_out;         /* [nx*ny] drainage area, or NULL             api:347 */
  double* etot_out;      /* [nx*ny] total erosion, or NULL             api:331 */
  int precision;         /* FSB_PREC_FP64 or FSB_PREC_MIXED (fsb_set_precision) */
} fsb_job;
/* `workers` threads (1..256) on CUDA device `device`; `mem_budget` bytes of
   device memory for job workspaces (0: 90% of the memory free now). */
int fsb_batch_create(fsb_batch** out, int device, int workers, size_t mem_budget);
/* Queues a job; the arrays it points to must stay valid until it is waited
   for.  A job whose workspace exceeds the whole budget is refused. */
int fsb_batch_submit(fsb_batch* b, const fsb_job* job, long long* id);
/* Blocks until job `id` has finished and forgets it; `status` receives 0 or
   the job's error code (whose message fsb_last_error then returns) and
   `times` (may be NULL) its submit, start and end times in seconds on one
   monotonic clock.  One thread waits per job: a second wait on the same id,
   while the first is blocked, returns an error. */
int fsb_batch_wait(fsb_batch* b, long long id, int* status, double* times);
/* Submits `njobs` jobs and waits for all of them; status[k] and
   times[3k..3k+2] as fsb_batch_wait (either may be NULL). */
int fsb_batch_run(fsb_batch* b, const fsb_job* jobs, int njobs, int* status, double* times);
/* Device bytes held by running jobs, the budget, running and queued jobs. */
int fsb_batch_memory(fsb_batch* b, size_t* in_use, size_t* budget, int* running, int* pending);
/* Waits for every submitted job, then stops the workers and frees the batch. */
int fsb_batch_destroy(fsb_batch* b);

/* ---- the reference's Fortran entry points (src/FastScape_api.f90) ---- */
void fastscape_init_(void);                                        /* api:146 */
void fastscape_setup_(void);                                       /* api:160 */
void fastscape_destroy_(void);                                     /* api:174 */
void fastscape_execute_step_(void);                                /* api:201 */
void fastscape_init_h_(double* hp);                                /* api:267 */
void fastscape_copy_h_(double* hp);                                /* api:299 */
void fastscape_copy_basement_(double* bp);                         /* api:315 */
void fastscape_copy_total_erosion_(double* etotp);                 /* api:331 */
void fastscape_copy_drainage_area_(double* ap);                    /* api:347 */
void fastscape_copy_erosion_rate_(double* eratep);                 /* api:363 */
void fastscape_copy_lake_depth_(double* lp);                       /* api:459 */
void fastscape_set_nx_ny_(const int* nnx, const int* nny);         /* api:475 */
void fastscape_set_xl_yl_(const double* xxl, const double* yyl);   /* api:491 */
void fastscape_set_dt_(const double* dtt);                         /* api:507 */
void fastscape_set_erosional_parameters_(const double* kkf, const double* kkfsed,
                                         const double* mm, const double* nnn,
                                         const double* kkd, const double* kkdsed,
                                         const double* gg1, const double* gg2,
                                         const double* pp);         /* api:523 */
void fastscape_get_sizes_(int* nnx, int* nny);                     /* api:556 */
void fastscape_get_step_(int* sstep);                              /* api:572 */
void fastscape_set_bc_(const int* jbc);                            /* api:602 */
void fastscape_set_u_(const double* up);                           /* api:618 */
void fastscape_set_v_(const double* ux, const double* uy);         /* api:634 */
void fastscape_reset_cumulative_erosion_(void);                    /* api:650 */
void fastscape_set_h_(double* hp);                                 /* api:664 */
void fastscape_set_basement_(double* bp);                          /* api:696 */
void fastscape_set_precip_(double* precipp);                       /* api:712 */
void fastscape_copy_chi_(double* chip);                            /* api:379 */
void fastscape_copy_slope_(double* slopep);                        /* api:395 */
void fastscape_copy_curvature_(double* curvaturep);                /* api:411 */
void fastscape_copy_catchment_(double* catchp);                    /* api:427 */
void fastscape_get_fluxes_(double* ttectonic_flux, double* eerosion_flux,
                           double* bboundary_flux);                /* api:762 */
void fastscape_set_all_layers_(double* dhp);                       /* api:680 */
void fastscape_view_(void);                                        /* api:188 */
void fastscape_vtk_(double* fp, double* vexp);                     /* api:728 */
void fastscape_debug_(void);                                       /* api:588 */

#ifdef __cplusplus
}
#endif

#endif /* FASTSCAPE_B200_H */
