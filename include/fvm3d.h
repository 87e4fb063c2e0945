/*
 * fvm3d.h — C ABI of the B200 explicit residual-and-update path.
 *
 * This library replaces the explicit time step of the FVM-3D-F90 structured
 * finite-volume Euler solver: `ClassTimeDiscret%solve`
 * (src/solve/class_time_discret.f90:125-156), which runs the Runge-Kutta stage
 * loop (class_time_discret.f90:159-196) over the space discretisation
 * (src/solve/class_space_discret.f90:120-176, 678-732) and the scheme kernels
 * (the src/scheme/ modules), and then the residual norms
 * (src/solve/class_iteration.f90:195-259 in file-local numbering of
 * class_iteration.f90: compute_residual_sub / update_sub).
 *
 * All entry points are plain C: pointers, sizes and int status codes. No
 * pointer passed in is retained after a call returns; host arrays stay owned
 * by the caller and are copied in and out. A context owns its device memory
 * and one CUDA stream; calls on one context are not re-entrant.
 *
 * Array convention for state exchange: Fortran column-major (ni,nj,nk,5) over
 * the real range of one block, i.e. exactly what `ClassBlockData%get_q()`
 * exposes (src/base/defs_block_data.f90:299-312). In C terms the element
 * (i,j,k,v) (0-based) sits at  i + ni*(j + nj*(k + nk*v)).
 * Variables are (rho, rho*u, rho*v, rho*w, rho*E), the equation slot order
 * set up in src/process/solver_sub.f90:131-143.
 */
#ifndef FVM3D_H
#define FVM3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FVM3D_ABI_VERSION 1
#define FVM_NEQ 5

/* ---- status codes (the ClassError flag+info convention,
 *      src/core/global_error.f90:18-33) ---------------------------------- */
enum fvm_status {
  FVM_OK = 0,
  FVM_ERR_INVALID = 1,     /* bad argument or configuration                 */
  FVM_ERR_CUDA = 2,        /* a CUDA runtime call failed                    */
  FVM_ERR_NOMEM = 3,       /* device or host allocation failed              */
  FVM_ERR_NONFINITE = 4,   /* NaN residual (class_iteration.f90:185-188)    */
  FVM_ERR_DIVERGED = 5,    /* residual above 1e10 (class_iteration.f90:180-184) */
  FVM_ERR_TIMEOUT = 6,     /* a bounded wait gave up                        */
  FVM_ERR_STATE = 7,       /* call out of order (e.g. step before set_state) */
  FVM_ERR_UNSUPPORTED = 8, /* id known to the reference but not implemented there either */
  FVM_ERR_BUSY = 9,        /* serving: no slot or memory free right now     */
  FVM_ERR_NOT_FOUND = 10,  /* serving: unknown request id                   */
  FVM_ERR_NEGATIVE = 11    /* reserved: uploads are not validated (as in the
                            * reference); a non-positive state surfaces as
                            * FVM_ERR_NONFINITE at the next step             */
};

/* ---- scheme ids: the namelist strings map to these integers exactly as in
 *      TypeDefs%SchemeIndex (src/defs/type_defs_scheme.f90:12-35, 41-84) ---- */
#define FVM_SCHEME_NULL (-1)
#define FVM_TIME_RUNGE_KUTTA 101   /* "Runge-Kutta"  */
#define FVM_TIME_BDF1 102          /* parsed by the reference, never run   */
#define FVM_RECON_SIMPLE 200       /* "simple"       */
#define FVM_RECON_MUSCL 201        /* "MUSCL"        */
#define FVM_RECON_WENO 202         /* "WENO"         */
#define FVM_RECON_WCNS 203         /* "WCNS": no implementation in the reference */
#define FVM_LIMITER_NONE 250       /* "none_"        */
#define FVM_LIMITER_MINMOD 251     /* "minmod_"      */
#define FVM_LIMITER_VANLEER 252    /* "VanLeer_"     */
#define FVM_LIMITER_VANALBADA 253  /* "vanAlbada_"   */
#define FVM_FLUX_ROE 300           /* "Roe"          */
#define FVM_FLUX_VANLEER 301       /* "VanLeer"      */
#define FVM_FLUX_HLLC 302          /* "HLLC": no implementation in the reference */
#define FVM_FLUX_AUSM 303          /* "AUSM"         */

/* timestep_set (class_time_discret.f90:94-122: only "fixed" exists there) */
enum fvm_timestep { FVM_DT_FIXED = 0, FVM_DT_CFL = 1, FVM_DT_CFL_LOCAL = 2 };
/* equation (type_defs_equation.f90: Euler / NS) */
enum fvm_equation { FVM_EQ_EULER = 0, FVM_EQ_NAVIER_STOKES = 1 };
/* compat: REFERENCE reproduces the reference's arithmetic including its
 * quirks; TEXTBOOK uses the published forms of WENO5-JS and Van Leer FVS. */
enum fvm_compat { FVM_COMPAT_REFERENCE = 0, FVM_COMPAT_TEXTBOOK = 1 };
/* precision of the reconstruction / flux arithmetic. State, RK accumulation,
 * dt and residual norms are FP64 in every mode. */
enum fvm_precision {
  FVM_PREC_FP64_EXACT = 0, /* FP64, the reference's operation order, no FMA    */
  FVM_PREC_FP64 = 1,       /* FP64, reassociated and FMA-contracted           */
  FVM_PREC_FP32_FLUX = 2   /* FP32 reconstruction + flux, FP64 state          */
};
/* boundary kind of one of the 6 ghost regions (defs_ghost_cell.f90:129-165:
 * 1 i-min, 2 i-max, 3 j-min, 4 j-max, 5 k-min, 6 k-max) */
enum fvm_bc {
  FVM_BC_TRANSMISSIVE = 0, /* zero-order extrapolation, defs_block_data.f90:226-256 */
  FVM_BC_PERIODIC = 1,     /* the block is its own donor across the opposite face  */
  FVM_BC_CONNECTED = 2     /* ghosts filled from donor blocks via fvm_connect      */
};

/* Solver configuration. Field names follow the namelist keys of
 * &Inviscid_Flux / &Time_Stepping (class_input.f90:137-162,
 * class_space_discret.f90:66-91, class_time_discret.f90:59-79). */
typedef struct fvm_config {
  int32_t struct_size;  /* = sizeof(fvm_config), checked by fvm_create        */
  int32_t idimension;   /* 2 or 3 (ClassGeometry%idimension)                   */
  int32_t equation;     /* fvm_equation                                        */
  int32_t reconstruct;  /* FVM_RECON_*                                         */
  int32_t limiter;      /* FVM_LIMITER_* or FVM_SCHEME_NULL (= none)           */
  int32_t flux_split;   /* FVM_FLUX_*                                          */
  int32_t time_scheme;  /* FVM_TIME_RUNGE_KUTTA                                */
  int32_t rk_stages;    /* 3 (SSP-RK3 of scheme_Runge_Kutta.f90) or 4 (classic RK4) */
  int32_t timestep_set; /* fvm_timestep                                        */
  int32_t compat;       /* fvm_compat                                          */
  int32_t precision;    /* fvm_precision                                       */
  int32_t store_rhs;    /* non-zero: keep the last stage's rhs for fvm_get_rhs */
  double kappa;         /* MUSCL kappa (default -1, as ClassSpaceDiscret)      */
  double entropy_fix;   /* Roe Harten coefficient (default 0.05)               */
  double gamma;         /* ratio of specific heats (default 1.4)               */
  double dt;            /* fix_timestep                                        */
  double cfl;           /* CFL number for FVM_DT_CFL / FVM_DT_CFL_LOCAL        */
  double mu;            /* dynamic viscosity, Navier-Stokes only               */
  double prandtl;       /* Prandtl number, Navier-Stokes only (default 0.71)   */
} fvm_config;

typedef struct fvm_ctx fvm_ctx;

/* Fill *cfg with the reference's defaults (MUSCL kappa -1, limiter NULL,
 * entropy_fix 0.05, gamma 1.4, 3 RK stages, fixed dt). */
int fvm_config_default(fvm_config* cfg);

/* Library ABI version (FVM3D_ABI_VERSION). */
int fvm_abi_version(void);

/* Create a solver context on the current CUDA device.
 * Replaces the set-up of ClassSpaceDiscret / ClassTimeDiscret /
 * ClassFlowField%allocate_memory (class_flow_field.f90:140-173). */
int fvm_create(const fvm_config* cfg, fvm_ctx** out);

/* Add one structured block with nvert real cells per axis and uniform cell
 * size dr (the `cell_size` of method_gridgen.f90:84-136 /
 * defs_block_geom.f90:306-314). For idimension 2, nvert[2] planes evolve
 * independently (the reference's 2D grid has nk = 2). Returns the 0-based
 * block id in *blk. All six regions start transmissive. */
int fvm_add_block(fvm_ctx* ctx, const int64_t nvert[3], const double dr[3], int* blk);

/* Set the kind of ghost region `region` (1..6) of block `blk`.
 * FVM_BC_PERIODIC makes the block its own donor across the opposite face. */
int fvm_set_boundary(fvm_ctx* ctx, int blk, int region, int kind);

/* Connect a box of ghost cells of block `blk` to real cells of block `donor`.
 * range[a][0..1] is the inclusive receiving box in blk's 0-based cell
 * indices (ghost cells are -3..-1 and n..n+2 along the face normal).
 * donor_type[a] = +-(1..3) maps receiver axis a onto donor axis
 * |donor_type[a]|-1, reversed when negative; donor_range[a][0..1] are the
 * donor indices (along that donor axis) matching range[a][0..1].
 * These are the ClassGeomFace connection semantics of
 * src/base/defs_face_geom.f90:43-82, 378-402 (connect_to), in cell indices.
 * Marks the regions touched as FVM_BC_CONNECTED. */
int fvm_connect(fvm_ctx* ctx, int blk, const int64_t range[3][2], int donor,
                const int64_t donor_range[3][2], const int32_t donor_type[3]);

/* Upload the conservative state of one block (layout above). */
int fvm_set_state(fvm_ctx* ctx, int blk, const double* q);
/* Download the conservative state of one block (layout above). */
int fvm_get_state(fvm_ctx* ctx, int blk, double* q);
/* The same for n blocks at once (q[i] is block blk[i]'s array, as above):
 * the per-block get_q() / set_q() exchanges of the reference
 * (src/base/defs_block_data.f90:299-312) in one call. The host-device copies
 * of consecutive blocks run back to back on a copy stream while the library
 * (un)packs the neighbouring block, and the call synchronises once, so the
 * host arrays are not touched after it returns. Results equal n calls of
 * fvm_set_state / fvm_get_state. */
int fvm_set_states(fvm_ctx* ctx, int n, const int* blk, const double* const* q);
int fvm_get_states(fvm_ctx* ctx, int n, const int* blk, double* const* q);
/* Download primitives (rho,u,v,w,p) of one block, same layout, computed as
 * convert_q_to_p_blk_sub (class_flow_field.f90:383-396). */
int fvm_get_primitive(fvm_ctx* ctx, int blk, double* p);
/* Download the last RK stage's rhs of one block (config.store_rhs != 0);
 * the array ClassBlockData%get_rhs() holds after a step. */
int fvm_get_rhs(fvm_ctx* ctx, int blk, double* rhs);

/* Advance nsteps explicit time steps (ClassTimeDiscret%solve, repeated).
 * On return *t is the physical time, res_abs[0..5] the absolute residuals
 * (per equation, then R_total) of the last step as
 * ClassIteration%compute_residual accumulates them over blocks, and
 * res_rel[0..5] (may be NULL) the residuals relative to step 1
 * (ClassIteration%update). Returns FVM_ERR_NONFINITE / FVM_ERR_DIVERGED when
 * the residual is NaN / above 1e10. t, res_abs may be NULL. */
int fvm_step(fvm_ctx* ctx, int nsteps, double* t, double* res_abs, double* res_rel);

/* Stop reasons of ClassIteration%converged (class_iteration.f90:145-192). */
enum fvm_stop {
  FVM_STOP_NONE = 0, FVM_STOP_MAX_STEP = 1, FVM_STOP_MAX_TIME = 2,
  FVM_STOP_ABS_RESIDUAL = 3, FVM_STOP_REL_RESIDUAL = 4
};
/* Run steps until a stop rule of ClassIteration%converged fires: step ==
 * max_step, t > total_time - 1e-10, R_total < absolute_residual, relative
 * R_total < relative_residual. Errors as fvm_step. *steps_done and *reason
 * may be NULL. max_step counts the context's steps from its first one (the
 * reference's iteration counter), not the steps of this call: a second
 * fvm_run continues from the current step, time and residuals, and returns
 * at once with FVM_STOP_MAX_STEP (0 steps done) when the count has already
 * reached max_step. */
int fvm_run(fvm_ctx* ctx, int64_t max_step, double total_time, double absolute_residual,
            double relative_residual, int64_t* steps_done, int* reason);

/* Current physical time, last dt and step count. */
int fvm_get_time(fvm_ctx* ctx, double* t, double* dt, int64_t* step);

/* Copy the last error message of ctx (or of the last failed fvm_create when
 * ctx is NULL) into buf (NUL-terminated, truncated to n bytes). */
int fvm_last_error(const fvm_ctx* ctx, char* buf, size_t n);

/* ---- batched and served cases (no counterpart in the reference, which runs
 *      one case per process) ------------------------------------------------
 * A context can hold many independent cases; fvm_step advances all of them in
 * lockstep (blocks of every case share each persistent stage launch), while
 * fvm_step's own t / residual outputs and error refer to the context's first
 * case. Cases can be added and removed between steps without touching the
 * state of the others. */

/* Fix the size of the state arena (padded cells per variable, the sum of
 * fvm_block_cells over the blocks it must hold) before the first upload: the
 * HBM budget of a served engine. Without it the arena holds exactly the
 * blocks present and grows when more are added. */
int fvm_reserve(fvm_ctx* ctx, int64_t cells);
/* Arena cells one block of this shape takes; its device bytes are
 * cells * 5 * 8 * (3 for SSP-RK3, 4 for RK4), +1 slab for Navier-Stokes. */
int fvm_block_cells(int idimension, const int64_t nvert[3], int64_t* cells);
/* Add a case with its own configuration (same rk_stages as the others). */
int fvm_add_case(fvm_ctx* ctx, const fvm_config* cfg, int* case_id);
/* fvm_add_block for a given case; block ids are unique across cases. */
int fvm_add_case_block(fvm_ctx* ctx, int case_id, const int64_t nvert[3], const double dr[3], int* blk);
/* Remove a case and free its arena ranges. Later additions reuse the ids of
 * removed cases (except case 0, the context's own first case) and of their
 * blocks, so a long-running engine's tables stay the size of its live set. */
int fvm_remove_case(fvm_ctx* ctx, int case_id);
/* Time, last dt, step count, residuals and status (FVM_OK, FVM_ERR_NONFINITE,
 * FVM_ERR_DIVERGED) of one case. Any pointer may be NULL. */
int fvm_case_state(fvm_ctx* ctx, int case_id, double* t, double* dt, int64_t* step, double* res_abs,
                   double* res_rel, int* status);

/* Autotuner hooks; no counterpart in the reference. fvm_tune_set forces the
 * tile shape (index 0: 32x8, 1: 16x16, 2: 32x8 with registers capped for two
 * resident CTAs per SM, 3: 16x8 on 128 threads, the heuristic's choice for 3D
 * FP32-flux and FP64 cases; -1 = heuristic) and z chunk length
 * (0 = heuristic) of the fused stage kernel for case `case_id`, keeping the
 * current state; fvm_tune_time_step runs `reps` full time steps (the state
 * advances) and returns the mean device time per step in ms.
 * fvm_tune_set_tail_split (3D; split 1..8, 1 = off, the default): when the
 * case's tasks fill the stage kernel's resident CTAs k times and r more, its
 * r shortest tasks are cut along z into `split` pieces (of at least 2
 * planes), so the last, partial round of the work queue is shorter. */
int fvm_tune_set(fvm_ctx* ctx, int case_id, int tile, int zchunk);
int fvm_tune_set_tail_split(fvm_ctx* ctx, int case_id, int split);
int fvm_tune_time_step(fvm_ctx* ctx, int reps, float* ms_per_step);
/* Profiling hooks; no counterpart in the reference. fvm_profile_step runs one
 * time step launch by launch with a CUDA event after each and returns the
 * device time of every launch (ms) and its kind (1 fused stage, 2 ghost
 * gather, 3 viscous, 4 finalize); fvm_kernel_launches_per_step gives the
 * number of kernels one (graph-captured) time step launches. */
int fvm_profile_step(fvm_ctx* ctx, float* ms, int32_t* kinds, int cap, int* n);
int fvm_kernel_launches_per_step(fvm_ctx* ctx, int* n);
/* Test hook of the failure path; no counterpart in the reference. With on
 * != 0 the stage kernels that fetch planes through tensor copies arm their
 * barrier but skip the copy, so their bounded wait (1 s) runs out: the next
 * fvm_step / fvm_case_state returns FVM_ERR_TIMEOUT once, and the context
 * stays usable (upload a state again after turning the hook off). */
int fvm_test_drop_tensor_copies(fvm_ctx* ctx, int on);
/* Test hook of the non-exact FP64 forms' reciprocal and reciprocal square
 * root (hardware approximation and one third-order correction); no
 * counterpart in the reference. Evaluates both over the host array x[0..n)
 * on the device into host arrays rcp_out / rsqrt_out. */
int fvm_test_fast_math(const double* x, int64_t n, double* rcp_out, double* rsqrt_out);

/* Residual norms of one block's rhs in device memory, as
 * ClassIteration%compute_residual_sub (class_iteration.f90, file-local
 * 210-248): rhs_dev is the Fortran (ni,nj,nk,5) array nvert describes;
 * res_dev points at 6 device doubles (per equation, then R_total) that are
 * updated as R = sqrt(R^2 + res2), so calls over the blocks of a case
 * accumulate like the reference (zero them before the first block). Runs on
 * `stream` (a cudaStream_t, NULL for the default stream) and returns after
 * it completes; allocates a scratch buffer of 40 bytes per k plane for the
 * call. Failures leave a message for fvm_last_error(NULL, ...). */
int fvm_residual_norms(const double* rhs_dev, const int64_t nvert[3], double* res_dev, void* stream);

/* fvm_residual_norms for callers that cannot allocate device memory; no
 * counterpart in the reference. Some host codes own every byte of GPU memory
 * through their own pool and forbid a library from allocating: this entry
 * point computes exactly what fvm_residual_norms computes but takes its
 * per-plane scratch from a fixed array inside the library (160 KiB per GPU
 * that loads it, kept until the process exits) and calls no allocator.
 * Limit: nvert[2] <= 4096 planes; larger blocks are rejected with
 * FVM_ERR_INVALID and a message for fvm_last_error(NULL, ...). Every call
 * looks up the array's device address on the current device (a host-side
 * query that allocates nothing); the first call on a device also loads the
 * library's device code there, so make that first call before any stream
 * capture. All calls share
 * the array: calls that overlap on the GPU (other host threads, other
 * streams) race, while calls in sequence are safe because every partial the
 * finalize reads is written by the same call first. Returns after `stream`
 * completes. */
int fvm_residual_norms_noalloc(const double* rhs_dev, const int64_t nvert[3], double* res_dev, void* stream);

/* Release the context and its device memory. */
int fvm_destroy(fvm_ctx* ctx);

/* ---- serving: requests queued and run with continuous batching inside the
 *      library. No counterpart in the reference, which runs one case per
 *      process; a server runs the step loop of solve_process
 *      (src/process/solver_sub.f90:196-207) for many cases at once.
 * A worker thread owned by the server admits submitted requests first come,
 * first served, while their arena cells (fvm_block_cells) fit the budget,
 * advances every admitted case together (one persistent launch per scheme
 * group and RK stage), and retires a case when its steps are done or its
 * residual became NaN / diverged, keeping its final state in host memory
 * until fvm_release. Cases with 3 and with 4 RK stages run in two engines
 * whose steps overlap on the device; each engine reserves the whole budget
 * when its first case arrives. A case's results equal its run alone bit for
 * bit. Calls may come from any host thread; all device work happens on the
 * worker thread, on the device current at fvm_server_create. */
typedef struct fvm_server fvm_server;

typedef struct fvm_server_config {
  int32_t struct_size;      /* = sizeof(fvm_server_config)                      */
  int32_t chunk_steps;      /* steps the running set advances between admissions */
  int64_t budget_cells;     /* arena cells the running set may hold (HBM budget) */
  int64_t max_active_cells; /* stop admitting once the running set holds this many
                             * cells (0 = no cap; an empty set admits one request) */
  int32_t max_queued;       /* fvm_case_submit returns FVM_ERR_BUSY beyond this many
                             * waiting requests                                   */
  int32_t pad_;
} fvm_server_config;

/* One block-to-block connection of a request, as fvm_connect takes it
 * (block indices local to the request). */
typedef struct fvm_connection {
  int32_t blk, donor;
  int64_t range[3][2];
  int64_t donor_range[3][2];
  int32_t donor_type[3];
  int32_t pad_;
} fvm_connection;

/* A case to run: its configuration, blocks and initial state (layout of
 * fvm_set_state), boundary kinds (bc[i] = {block, region 1..6, fvm_bc kind};
 * regions not listed stay transmissive) and connections, and the number of
 * time steps. Everything is copied by fvm_case_submit. */
typedef struct fvm_request {
  int32_t struct_size;        /* = sizeof(fvm_request)              */
  int32_t nblocks;
  const fvm_config* cfg;
  const int64_t* nvert;       /* [nblocks][3]                       */
  const double* dr;           /* [nblocks][3]                       */
  const double* const* q;     /* [nblocks] host arrays              */
  int32_t nbc, nconn;
  const int32_t* bc;          /* [nbc][3]                           */
  const fvm_connection* conn; /* [nconn]                            */
  int64_t steps;              /* time steps to run, >= 1            */
} fvm_request;

enum fvm_request_state { FVM_REQ_QUEUED = 0, FVM_REQ_RUNNING = 1, FVM_REQ_DONE = 2, FVM_REQ_FAILED = 3 };

/* Defaults: chunk 8 steps, budget 2^24 cells, no active cap, 1024 queued. */
int fvm_server_config_default(fvm_server_config* cfg);
int fvm_server_create(const fvm_server_config* cfg, fvm_server** out);
/* Queue a request; *request_id identifies it. FVM_ERR_BUSY when max_queued
 * requests are waiting, FVM_ERR_INVALID for a malformed request or one that
 * needs more cells than the whole budget. A configuration the engine rejects
 * fails the request later (state FVM_REQ_FAILED, status and message). */
int fvm_case_submit(fvm_server* srv, const fvm_request* req, int64_t* request_id);
/* State, steps done, physical time, time since submission (or from
 * submission to completion once finished, in seconds) and status
 * (FVM_OK or the error that failed it). Any output may be NULL.
 * FVM_ERR_NOT_FOUND for an unknown or released id. */
int fvm_poll(fvm_server* srv, int64_t request_id, int* state, int64_t* steps_done, double* t, double* latency_s,
             int* status);
/* Block until the request is done or failed, at most timeout_s seconds
 * (FVM_ERR_TIMEOUT otherwise). */
int fvm_wait(fvm_server* srv, int64_t request_id, double timeout_s, int* state);
/* Copy the final state of block `blk` (request-local index) of a finished
 * request into q (layout of fvm_get_state); FVM_ERR_BUSY before it finished. */
int fvm_fetch_state(fvm_server* srv, int64_t request_id, int blk, double* q);
/* Forget a finished request and free its host copy. */
int fvm_release(fvm_server* srv, int64_t request_id);
/* Cells the running set holds now and at most so far, running and queued
 * request counts. Any output may be NULL. */
int fvm_server_stats(fvm_server* srv, int64_t* active_cells, int64_t* peak_active_cells, int* running, int* queued);
int fvm_server_last_error(fvm_server* srv, char* buf, size_t n);
/* Stop the worker (running requests end as failed) and free everything. */
int fvm_server_destroy(fvm_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* FVM3D_H */
