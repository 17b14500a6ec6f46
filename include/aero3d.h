/*
 * aero3d.h - C ABI of the B200 3D Euler cut-cell solver (libaero3d.so).
 *
 * Drop-in for the solver entry points of WeiJungSong/3d_aero_lab `src/air_cfd.js`:
 * grid generation, cut-cell geometry (volume fractions, face apertures, thin-wing
 * baffles, fixed-state engine cells), the SSP-RK2 solver object and the force,
 * Trefftz and residual post-processing.  The reference calls these from JavaScript;
 * a Node N-API shim binds these functions one to one.
 *
 * Conventions
 *  - Every function returns an int status (A3D_OK == 0).  No exception crosses the
 *    ABI and there is no CPU fallback: if the GPU is missing or a CUDA call fails the
 *    status says so and a3d_last_error() returns the message of the failing call.
 *  - Only plain C types cross the ABI: pointers, sizes, doubles, floats.
 *  - Cell index q = (k*NY + j)*NX + i (src/air_cfd.js:45).
 *  - Conservative state is structure-of-arrays float32 (rho, rho*u, rho*v, rho*w, E),
 *    nondimensional with rho_inf = 1, a_inf = 1, p_inf = 1/gamma (src/air_cfd.js:8).
 *  - Solver calls are asynchronous on the solver's own CUDA stream except the ones
 *    that return host data (read, forces, trefftz, residual, diag), which synchronise.
 */
#ifndef AERO3D_H
#define AERO3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define A3D_OK             0
#define A3D_ERR_ARG        1  /* bad argument (null pointer, size out of range)          */
#define A3D_ERR_CUDA       2  /* a CUDA runtime call failed; see a3d_last_error()         */
#define A3D_ERR_NOMEM      3  /* device allocation failed                                 */
#define A3D_ERR_NONFINITE  4  /* the state holds NaN or Inf (detected on the device)      */
#define A3D_ERR_STATE      5  /* call not valid in the object's current state            */
#define A3D_ERR_BUDGET     6  /* request does not fit the server's device-memory budget  */
#define A3D_ERR_TIMEOUT    7  /* a bounded wait ran out                                   */
#define A3D_ERR_NODEVICE   8  /* no CUDA device is visible                                */

#define A3D_MAX_ENGINES 2
#define A3D_WAIT_LIMIT_DEFAULT 4194304u  /* try_waits per TMA copy (a3d_solver_set_wait_limit) */
#define A3D_MAX_EXITS   2
#define A3D_ENV_N       300   /* nacelle envelope table intervals (src/air_cfd.js:53)   */

/* ---- aircraft shape: what the inside tests need (src/aircraft.js, src/air_field.js) -- */
typedef struct a3d_surface {
  double x0, z0, semi, cr, ct;   /* root LE x, root z, semi-span (height for the fin), chords */
  double tanL;                   /* tan(sweep) as makeSurface computes it (aircraft.js:83)   */
  double tanD_pt, tanI_pt;       /* tan(dihedral), tan(incidence) used by surface points     */
  double tanD_deg, tanI_deg;     /* the same via DEG, as inLift/zMean compute them           */
  double tcR, tcT, camber;       /* thickness ratios root/tip, NACA camber                   */
  double sA;                     /* AirGeom attachment span (air_field.js:107)              */
  double bb[4];                  /* AirGeom bounding box x0, x1, z0, z1 (air_field.js:109)  */
} a3d_surface;

typedef struct a3d_engine {
  double x0, y, z;               /* lip station and axis (aircraft.js:132-141)               */
  int32_t internal;              /* 1: engine buried in the fuselage                          */
  int32_t env_n;                 /* 0: no nacelle envelope, else A3D_ENV_N                    */
  double env_xmax;               /* envelope length                                          */
  float env_R[A3D_ENV_N + 1];    /* envelope radius table, float32 (air_cfd.js:53-54)       */
  float pad_;
} a3d_engine;

typedef struct a3d_exit {
  int32_t type;                  /* fixed-state cell type: 4 bypass jet, 5 core jet          */
  int32_t pad_;
  double x, R, Rin;              /* exit station (engine frame), outer/inner radius          */
} a3d_exit;

typedef struct a3d_shape {
  double fus_L, fus_R0, fus_Ln, fus_Lt, fus_xt0, fus_Re, fus_noseP, fus_tailUp;
  a3d_surface wing, htail, vtail;
  double ref_b;                  /* reference span (cfdGrid core width)                      */
  double view_Rmax;              /* engine outer radius (cfdGrid margins)                    */
  double lip_x, lip_r;           /* intake lip (inlet sink layer)                            */
  int32_t n_engines, n_exits;
  a3d_engine engines[A3D_MAX_ENGINES];
  a3d_exit exits[A3D_MAX_EXITS];
} a3d_shape;

/* ---- library ------------------------------------------------------------------------ */
/* Message of the last failure on this thread ("" if none). */
const char* a3d_last_error(void);
/* ABI version, bumped on any change of a struct or signature. */
int a3d_abi_version(void);

/* ---- grid: cfdAxis/cfdGrid (src/air_cfd.js:14-44) -------------------------------- */
/* Builds the stretched half-domain grid for `target_cells`.  Face coordinates go to
 * xf/yf/zf (capacity `cap` each, float64, NX+1 / NY+1 / NZ+1 values); dims gets
 * NX, NY, NZ; h_out the near-body spacing; core_out the core box x0,x1,y1,z0,z1.   */
int a3d_grid_build(const a3d_shape* shape, double target_cells, int32_t cap,
                   double* xf, double* yf, double* zf, int32_t dims[3],
                   double* h_out, double core_out[5]);

/* ---- cut-cell geometry: cfdGeom (src/air_cfd.js:50-141), on the GPU ---------------- */
/* Evaluates the inside tests on the device and returns the reference's arrays:
 * t (u8[N]: 0 fluid, 1 solid, 3 inlet sink, 4 bypass jet, 5 core jet), phi (f32[N]),
 * ap0..ap2 (f32[N], +x/+y/+z face apertures), ap3 (f32[N], baffle slope dz/dx on
 * the +z face).  counts gets nSolid, nCut; vol gets volW, volH, volV.
 * Any of the output pointers may be NULL to skip that copy.                          */
int a3d_geom_build(const a3d_shape* shape, const int32_t dims[3],
                   const double* xf, const double* yf, const double* zf,
                   double h, double delta_deg,
                   uint8_t* t, float* phi, float* ap0, float* ap1, float* ap2, float* ap3,
                   int64_t counts[2], int32_t vol[3]);

/* ---- force list: cfdForceList (src/air_cfd.js:143-152), on the GPU ----------------- */
/* Number of list cells; then the list itself in cell order (any pointer may be NULL). */
typedef struct a3d_solver a3d_solver;
int a3d_solver_force_list(a3d_solver* s, int64_t* n_out, int64_t cap,
                          int64_t* q, double* cx, double* cz, double* x, double* z);

/* ---- solver object: CfdCPU/CfdGPU (src/air_cfd.js:157-259, 367-438) -------------- */
/* From caller geometry arrays, like `new CfdGPU(g, geo)`.  The arrays are copied to the
 * device; the caller keeps ownership.                                                 */
int a3d_solver_create(const int32_t dims[3], const double* xf, const double* yf,
                      const double* zf, const uint8_t* t, const float* phi,
                      const float* ap0, const float* ap1, const float* ap2,
                      const float* ap3, int device, a3d_solver** out);
/* Builds grid-resident geometry straight on the device from the shape (no host copy of
 * the N-sized arrays): cfdGeom + cfdForceList + solver in one call.                   */
int a3d_solver_create_shape(const a3d_shape* shape, const int32_t dims[3],
                            const double* xf, const double* yf, const double* zf,
                            double h, double delta_deg, int device, a3d_solver** out);
int a3d_solver_destroy(a3d_solver* s);
/* Grid size and the device the solver lives on. */
int a3d_solver_dims(a3d_solver* s, int32_t dims[3], int64_t* n_cells);
/* opt.cfl and opt.order (defaults 0.7 and 2, src/air_cfd.js:162). */
int a3d_solver_set_opt(a3d_solver* s, double cfl, int32_t order);
/* setFree(F[5]) (src/air_cfd.js:166): far-field conservative state. */
int a3d_solver_set_free(a3d_solver* s, const double F[5]);
/* setFix([sink, jetBypass, jetCore]) (src/air_cfd.js:167): 3 x 5 conservative states
 * for cell types 3, 4, 5.                                                             */
int a3d_solver_set_fix(a3d_solver* s, const double fix[15]);
/* reset() (src/air_cfd.js:168): Q = F everywhere, it = 0. */
int a3d_solver_reset(a3d_solver* s);
/* step(n) (src/air_cfd.js:252-258): n SSP-RK2 iterations, queued on the solver stream. */
int a3d_solver_step(a3d_solver* s, int32_t n);
/* Iterations done since reset. */
int a3d_solver_iterations(a3d_solver* s, int64_t* it);
/* read() (src/air_cfd.js:259): copies Q into five caller arrays of N floats
 * (rho, rho*u, rho*v, rho*w, E).  Synchronises.                                        */
int a3d_solver_read(a3d_solver* s, float* r, float* ru, float* rv, float* rw, float* E);
/* The dt field of CfdGPU.read() (src/air_cfd.js:435): each fluid cell's local time step in the
 * last iteration, 0 elsewhere and before the first iteration; N floats in cell order.     */
int a3d_solver_read_dt(a3d_solver* s, float* dt);
/* Uploads a state (warm start or checkpoint restore); same layout as read(). */
int a3d_solver_write(a3d_solver* s, const float* r, const float* ru, const float* rv,
                     const float* rw, const float* E);
/* cfdForces (src/air_cfd.js:443-452) over the force list, FP64 on the device.
 * out = {CL, CD, Cm}.  M is used as given (the controller passes max(M, 0.05)).       */
int a3d_solver_forces(a3d_solver* s, double alpha_deg, double M, double S, double xcg,
                      double zcg, double cref, double out[3]);
/* Trefftz-plane induced drag at station xT (src/air_cfd.js:560-570), FP64. */
int a3d_solver_trefftz(a3d_solver* s, double xT, double alpha_deg, double M, double S,
                       double* cdi);
/* Density residual (src/air_cfd.js:552-555): RMS of rho - rho_prev over fluid cells with
 * q % stride == 0, divided by the iterations since the previous call, in FP64; then
 * rho_prev = rho.  The first call only takes the snapshot and returns -1.
 * Returns A3D_ERR_NONFINITE if a sampled density is NaN/Inf.                          */
int a3d_solver_residual(a3d_solver* s, int32_t stride, double* res);
/* Largest Mach number over fluid cells with q % stride == 0 (src/air_cfd.js:571). */
int a3d_solver_mach_max(a3d_solver* s, int32_t stride, double* mmax);
/* Display sampling cfdStencil + cfdSample (src/air_cfd.js:455-482) on the device: primitive
 * states (rho, u, v, w, p) at n points xyz (FP64, x/y/z interleaved), so that surfaces,
 * slices and probes need no full read().  ok[p] = 0 where no fluid cell is near.        */
int a3d_solver_sample(a3d_solver* s, int32_t n, const double* xyz, double* out5, int32_t* ok);
/* Grid sequencing, interpState (src/app_cfd.js:322-357, called from setupCFD :271-278):
 * overwrite `fine`'s state with `coarse`'s current state interpolated onto its cells - a
 * coarse pre-converged start for a finer grid of the same geometry.  Trilinear over the eight
 * surrounding coarse centres with non-fluid corners dropped and the weights renormalised; the
 * nearest fluid coarse cell within +-3 cells if all eight are excluded; else the free stream.
 * Non-fluid target cells take the free stream (as after reset).  Resets `fine`'s iteration
 * count and residual snapshot like a3d_solver_reset.  Both solvers on one device; the copy
 * is ordered after the work already queued on `coarse` and before any work queued on it later.
 * The reference's function is 2-D (axisymmetric v2 solver); this is its 3-D form.        */
int a3d_solver_interp_state(a3d_solver* fine, const a3d_solver* coarse);
/* Stage kernel selection; no counterpart in the reference (it has one shader).
 * kernel 0: one thread per cell evaluating its six faces (the reference's structure);
 * kernel 2: z-marching 32 x 8-column tiles that evaluate every face once, fed by a TMA
 *           plane ring, three CTAs per SM;
 * kernel 4 (default): the same over 32 x 16-column tiles, each thread two x-adjacent cells
 *           in packed f32x2 arithmetic, two CTAs per SM.
 * (Numbers 1 and 3 belonged to two tiles since retired; they are refused.)
 * march_kz = z planes per thread block; 0 (the default) picks for the TMA tiles 32 planes if
 * that still launches four waves of CTAs, else the longest of 16, 8 or 4 planes that
 * launches two waves, else 2.                                                            */
int a3d_solver_set_kernel(a3d_solver* s, int32_t kernel, int32_t march_kz);
int a3d_solver_get_kernel(a3d_solver* s, int32_t* kernel, int32_t* march_kz);
/* Bounded device waits; no counterpart in the reference.  Every wait of a stage kernel (the
 * TMA tiles, kernels 2 and 4) for a TMA plane copy gives up after `limit` tries
 * (A3D_WAIT_LIMIT_DEFAULT unless set; 0 = give up at once): the kernel then waits, with the
 * default limit, for its copies in flight, flags the solver and leaves, and the next
 * a3d_solver_sync / read / reduction returns A3D_ERR_TIMEOUT once (the flag is then cleared;
 * the state of the failed stage is not meaningful, reset or write it).  Limit 0 makes every
 * wait run out without any fault, which is how the timeout path is tested.               */
int a3d_solver_set_wait_limit(a3d_solver* s, uint32_t limit);
/* Kernels 2 and 4 step the case as up to 4 z chunks of whole z runs on their own streams, each
 * chunk's stage waiting only for its neighbour chunks' previous stage: the tail of one stage
 * overlaps the start of the next.  0 = automatic (4 chunks from 0.8M cells up, else 1),
 * 1 = one launch per stage, 2..4 = that many chunks.  The results are the same bit for bit. */
int a3d_solver_set_chunks(a3d_solver* s, int32_t chunks);
/* The number of chunks (stage launches per RK stage) a3d_solver_step uses for this case.  */
int a3d_solver_get_chunks(a3d_solver* s, int32_t* chunks);
/* The solver's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
int a3d_solver_stream(a3d_solver* s, void** stream);
/* Blocks until all work queued on the solver's stream has finished. */
int a3d_solver_sync(a3d_solver* s);

/* ---- one case split into z slabs (several devices, or ranks) ---------------------- */
/* No counterpart in the reference (one case, one WebGL context).  A slab solver holds the
 * planes [z_lo, z_hi) of the case a3d_solver_create_shape builds on the full grid: its own
 * planes plus up to two halo planes on each side shared with the neighbouring slab.  Per
 * iteration the caller runs stage 1 on every slab, exchanges the halo planes of the stage-1
 * state (which = 1), runs stage 2, and exchanges the halo planes of the new state
 * (which = 0).  Restricted to its own planes (a3d_solver_set_owned), a slab's forces,
 * Trefftz integral and residual sums add up to the full case's, and Mach maxima combine by
 * max.                                                                                  */
int a3d_solver_create_shape_slab(const a3d_shape* shape, const int32_t dims[3],
                                 const double* xf, const double* yf, const double* zf,
                                 double h, double delta_deg, int32_t z_lo, int32_t z_hi,
                                 int device, a3d_solver** out);
/* Planes [k0, k1) (slab-local) that forces, Trefftz, residual and Mach maximum cover.    */
int a3d_solver_set_owned(a3d_solver* s, int32_t k0, int32_t k1);
/* One RK stage: 1 = first stage, 2 = second stage (completes the iteration).             */
int a3d_solver_stage(a3d_solver* s, int32_t which);
/* Halo exchange within one process: planes of src's current (which = 0) or stage-1
 * (which = 1) state into dst's buffer of the same role; stream-ordered on both solvers,
 * peer copy when they live on different devices.                                        */
int a3d_solver_copy_planes(a3d_solver* dst, int32_t dst_k0, a3d_solver* src, int32_t src_k0,
                           int32_t nk, int32_t which);
/* Device address of plane k of component c (planes of a component are contiguous,
 * plane_floats apart), for exchanges the caller runs on the solver's stream (NCCL).      */
int a3d_solver_plane_ptr(a3d_solver* s, int32_t which, int32_t c, int32_t k, void** ptr,
                         int64_t* plane_floats);
/* Halo push instead of copies: s's stage kernels also store the own planes that its lower
 * and upper neighbours (either may be NULL) keep as halo planes into the neighbours' buffers,
 * peer stores across devices.  Afterwards s advances only by a3d_solver_stage; call
 * a3d_solver_sync_neighbors on every slab after every stage of all slabs, so that each slab's
 * next stage waits for its neighbours' stores.  Stage kernels 0 and 2.                   */
int a3d_solver_set_neighbors(a3d_solver* s, a3d_solver* lo, a3d_solver* hi);
int a3d_solver_sync_neighbors(a3d_solver* s);
/* Sum of squared density changes and cell count behind the last a3d_solver_residual.     */
int a3d_solver_residual_parts(a3d_solver* s, double out[2]);

/* ---- batched solves: many cases advanced together -------------------------------- */
/* No counterpart in the reference (its controller runs one case).  A batch groups solver
 * objects living on one device; a3d_batch_step(n) advances every case by n SSP-RK2
 * iterations, two iterations captured once in a CUDA graph: either every case's own launches
 * run concurrently (mode 1) or one persistent kernel launch per stage pulls the tiles of all
 * cases from a shared queue (mode 0).  Each case keeps its own
 * state, forces, residual and Trefftz calls; the batch orders itself after each solver's
 * queued work and each solver's later work after the batch.                            */
typedef struct a3d_batch a3d_batch;
int a3d_batch_create(a3d_solver* const* solvers, int32_t n, a3d_batch** out);
int a3d_batch_destroy(a3d_batch* b);
int a3d_batch_step(a3d_batch* b, int32_t n);
int a3d_batch_sync(a3d_batch* b);
/* How the batch runs its cases.  Mode 1 (default): each case's own single-case stage
 * launches, each case on its own stream forked from the batch's, two iterations captured in
 * one CUDA graph whose per-case branches run concurrently; every case then computes exactly
 * what a3d_solver_step computes alone.  Mode 0: the persistent kernel above.
 * a3d_batch_tune times both and keeps the faster.  A solver stepped or reconfigured on its
 * own between batch steps makes the batch rebuild its table and graphs.                  */
int a3d_batch_set_mode(a3d_batch* b, int32_t mode);
int a3d_batch_get_mode(a3d_batch* b, int32_t* mode);
/* Tile schedule: z planes per tile (kz) and persistent CTAs per SM (1 to 3). */
int a3d_batch_set_schedule(a3d_batch* b, int32_t kz, int32_t ctas_per_sm);
int a3d_batch_get_schedule(a3d_batch* b, int32_t* kz, int32_t* ctas_per_sm, int64_t* tiles);
/* Autotuner: times every (kz, CTAs per SM) candidate of mode 0, then mode 1, for trial_iters
 * iterations on the real cases (states saved and restored), keeps the fastest (best_kz and
 * best_ctas are mode 0's best schedule; a3d_batch_get_mode tells the mode kept); best_ms =
 * ms per iteration of the kept choice.                                                   */
int a3d_batch_tune(a3d_batch* b, int32_t trial_iters, int32_t* best_kz, int32_t* best_ctas,
                   float* best_ms);

/* ---- continuous-batching solve server ----------------------------------------------- */
/* No counterpart in the reference (its controller steps one case per animation frame).  A
 * scheduler thread admits requests in arrival order while the estimated device memory of all
 * resident cases fits `hbm_budget_bytes` and fewer than `max_active` run; every round advances
 * all active cases by `chunk_iters` iterations in one batch (one persistent launch per RK
 * stage), then checks each case's FP64 density residual (every fluid cell) against its first
 * value.  A case finishes when the ratio is <= residual_drop or after max_iters iterations;
 * its forces and Trefftz drag are computed on the device and it leaves the batch at once.
 * With warm_start, finished cases stay resident keyed by `geometry_key` and a later request
 * with the same key starts from that state (least recently used ones are evicted first).  */
typedef struct a3d_server_config {
  double hbm_budget_bytes;
  double residual_drop;        /* e.g. 1e-3                                             */
  int32_t max_active;          /* slot cap                                              */
  int32_t chunk_iters;         /* iterations per round                                  */
  int32_t max_iters;           /* iteration cap per request                             */
  int32_t device;
  int32_t warm_start;          /* 1: keep finished cases resident for reuse              */
  int32_t kz;                  /* z planes per tile; 0: each case picks its own         */
  /* Grid sequencing (the reference's setupCFD, src/app_cfd.js:271-278, 398-403): a cold
   * request first solves a coarse case of cells/sequence cells until its residual dropped by
   * sequence_drop or it ran sequence_max_iters iterations, then starts the requested case
   * from that state (a3d_solver_interp_state).  0 or 1: off.  The requested case's res0 is
   * its own first residual from the free stream, measured over one chunk before the
   * interpolation, so residual_drop means the same with and without sequencing.           */
  int32_t sequence;
  int32_t sequence_max_iters;
  double sequence_drop;
} a3d_server_config;

typedef struct a3d_request {
  a3d_shape shape;
  double cells, M, alpha_deg, delta_deg;
  double F[5];                 /* far-field state (setFree)                              */
  double fix[15];              /* fixed states of types 3, 4, 5 (setFix)                 */
  double ref_S, ref_xcg, ref_zcg, ref_c;  /* force coefficients' reference values       */
  double xT;                   /* Trefftz plane station                                  */
  uint64_t geometry_key;       /* equal keys: same aircraft, cells and delta             */
} a3d_request;

typedef struct a3d_result {
  int32_t status;              /* A3D_OK or the failing call's status                    */
  int32_t warm;                /* 1: started from a resident converged state            */
  int64_t iterations;
  double CL, CD, Cm, CDi;
  double residual, res0;       /* last and first density residual                       */
  double t_submit, t_admit, t_done;  /* seconds on the server's clock                   */
  int64_t coarse_iterations;   /* iterations of the sequencing coarse case (0 if none)     */
} a3d_result;

typedef struct a3d_server a3d_server;
int a3d_server_create(const a3d_server_config* cfg, a3d_server** out);
/* Queues a request; A3D_ERR_BUDGET if it can never fit the budget. */
int a3d_server_submit(a3d_server* sv, const a3d_request* req, int64_t* id);
int a3d_server_poll(a3d_server* sv, int64_t id, a3d_result* out, int32_t* done);
/* Waits up to timeout_s for a result (A3D_ERR_TIMEOUT otherwise). */
int a3d_server_wait(a3d_server* sv, int64_t id, double timeout_s, a3d_result* out);
/* pending, active, completed, warm starts, rounds, resident bytes */
int a3d_server_stats(a3d_server* sv, int64_t out[6]);
int a3d_server_destroy(a3d_server* sv);

/* ---- force integral without device allocation ------------------------------------- */
/* No counterpart in the reference.  The same C_L, C_D, C_m as a3d_solver_forces, for callers
 * that hold the state and the force list in device memory of their own and cannot call
 * cudaMalloc (a host application that gives the addon a fixed device pool, or code that must
 * not change the device's allocation state).  Inputs: five device arrays of the conservative
 * state indexed by the reference cell index q, and the device force list (q, cx, cz, x, z) of
 * n cells, as a3d_solver_force_list returns it.  Scratch is a static device array inside the
 * library (about 96 KiB per GPU that loads it, held until exit), so n is limited to 1,048,576
 * list cells; longer lists are rejected with A3D_ERR_ARG.  The call allocates and frees
 * nothing.  The first call on a device looks up the scratch address on that device (make it
 * before any stream capture).  All calls share the scratch: calls that overlap on the GPU
 * (different streams, or several host threads at once) race.  Work is queued on `stream`
 * (NULL: the default stream) and the call waits for it; out = {CL, CD, Cm}.            */
int a3d_forces_noalloc(const float* r, const float* ru, const float* rv, const float* rw,
                       const float* E, int64_t n, const int64_t* q, const double* cx,
                       const double* cz, const double* x, const double* z,
                       double alpha_deg, double M, double S, double xcg, double zcg,
                       double cref, void* stream, double out[3]);

#ifdef __cplusplus
}
#endif
#endif /* AERO3D_H */
