/*
 * bhr.h -- C ABI of bh_ringdown_b200, a B200-native time-domain Teukolsky
 * solver that replaces the reference TD_GPU_code/HighOrder path.
 *
 * The reference has no library interface.  Its boundary is the C call
 *   void body(double *r_c, double *theta, double dtheta, double mass,
 *             double aa, double ss, double mm, double dx, double dt,
 *             int p, int my_rank)                  (HighOrder/body.cu:25-27)
 * driven by main() (HighOrder/main.c:25-62) with the grid and run knobs as
 * compile-time macros (HighOrder/parm.h:1-13), a .traj text file as source
 * input (HighOrder/body.cu:77,97-120) and hm*.dat files as output
 * (HighOrder/body.cu:63-78,204-212).  The entry points below cover that
 * call and its inputs and outputs; each comment names what it replaces.
 *
 * Conventions: plain C types only; the library owns all device memory and
 * streams; callers own host buffers.  Every call returns a bhr_status
 * (0 = OK); bhr_last_error_string() describes the last failure on the
 * calling thread.  No call exits the process or traps on the device.
 * Field arrays are row-major M x N doubles, idx(b,a) = N*b + a as in
 * HighOrder/parm.h:13 (theta rows b, radial columns a).
 */
#ifndef BHR_H
#define BHR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BHR_ABI_VERSION 3

typedef enum bhr_status {
  BHR_OK = 0,
  BHR_INVALID_ARG = 1,   /* bad parameter or size                          */
  BHR_OUT_OF_MEMORY = 2, /* device allocation failed or over budget        */
  BHR_CUDA_ERROR = 3,    /* a CUDA runtime call failed                     */
  BHR_NAN_DETECTED = 4,  /* non-finite value in the extracted waveform     */
  BHR_TIMEOUT = 5,       /* a bounded device wait gave up                  */
  BHR_IO_ERROR = 6,      /* file could not be read or written              */
  BHR_NO_DEVICE = 7      /* no CUDA device available                       */
} bhr_status;

/* BHR_SSPRK3: the reference's integrator (HighOrder/kern.cu:301-318,
 * 582-620).  BHR_RK4: classical four-stage Runge-Kutta, FP64 only, for runs
 * specified with RK4; the step's particle source is held fixed in all four
 * stages as in the reference's step.  bhr_step_noalloc and the batch engine
 * step SSP-RK3 only. */
typedef enum bhr_integrator { BHR_SSPRK3 = 0, BHR_RK4 = 1 } bhr_integrator;
typedef enum bhr_precision { BHR_FP64 = 0, BHR_MIXED = 1 } bhr_precision;
typedef enum bhr_init_kind { BHR_INIT_ZERO = 0, BHR_INIT_GAUSSIAN = 1 } bhr_init_kind;
/* Stage kernel tilings (chosen per device and grid by timing, or fixed by
 * the environment variable BHR_STAGE_TILING=block8|block16|persistent|
 * block8n|ring|strip12): one 64 x 8 or 64 x 16 tile per 256-thread block;
 * 64 x 16 tiles walked by one 512-thread block per SM; 64 x 8 tiles per
 * 128-thread block, four per SM; 64 x 8 tiles walked by two 256-thread
 * blocks per SM; stages 1 and 2 fused in one launch over 128-column strips
 * (the intermediate stage stays in shared memory; FP64 SSP-RK3 solves, stage
 * 3 as block8n). */
typedef enum bhr_tiling {
  BHR_TILING_BLOCK8 = 0,
  BHR_TILING_BLOCK16 = 1,
  BHR_TILING_PERSISTENT = 2,
  BHR_TILING_BLOCK8N = 3,
  BHR_TILING_RING = 4,
  BHR_TILING_STRIP12 = 5
} bhr_tiling;

/* Run parameters.  Replaces HighOrder/parm.h:1-13 (N, M, Xmax, Xmin, Fr, T,
 * PTSX, PTSY) and the constants of HighOrder/main.c:40-46 (mass, aa, ss,
 * dt) plus the m loop of HighOrder/main.c:50-55.  s = -2 is fixed, as in the
 * reference's coefficient formulas (HighOrder/kern.cu:142). */
typedef struct bhr_params {
  int N;              /* radial points (multiple of 64)                      */
  int M;              /* theta points (multiple of 16, >= 16)                */
  double Xmin, Xmax;  /* grid coordinate extent                              */
  double mass;        /* black-hole mass                                     */
  double a;           /* spin parameter                                      */
  double m;           /* azimuthal number                                    */
  double dt;          /* time step; <= 0 selects the Courant rule below      */
  double courant;     /* dt = courant*min(dx, r_c[0]*dtheta), then shrunk so
                         out_every/dt is an integer when out_every > 0       */
  double out_every;   /* output spacing in time for the Courant rule (0: none) */
  double T;           /* final time                                          */
  int Fr;             /* waveform row every Fr steps (0: from out_every)     */
  double out_start;   /* rows written once k*dt >= out_start (ref: Xmax+200) */
  int ext_col;        /* extraction column, -1 = N-1 (ref)                   */
  int PTSX, PTSY;     /* particle source patch (ref 128 x 128)               */
  double wr_fac;      /* wr = wr_fac*dx*(1 - r+/rp), ref 2                   */
  double wt_fac;      /* wt = wt_fac*dtheta, ref 6                           */
  int integrator;     /* bhr_integrator                                      */
  int precision;      /* bhr_precision                                       */
  int init_kind;      /* bhr_init_kind                                       */
  double init_center; /* Gaussian initial data psi = exp(-(x-c)^2/(2 w^2))   */
  double init_width;  /*   * swsh(l, m, theta), Pi = 0                       */
  double init_ell;
  int device;         /* CUDA device ordinal                                 */
} bhr_params;

/* Fills the reference's defaults (HighOrder/parm.h, HighOrder/main.c):
 * N=16000, M=256, Xmin=-50, Xmax=50, mass=1, a=1e-8, m=2, dt=0.002, T=1500,
 * Fr=50, out_start=Xmax+200, PTSX=PTSY=128, wr_fac=2, wt_fac=6. */
int bhr_params_default(bhr_params *p);

/* One particle state as HighOrder/body.cu:112-124 passes it to sourced(). */
typedef struct bhr_particle {
  double rp, tp, phip, E, lz, Q;
  double drdt, d2rdt2, d3rdt3;
  double dthdt, d2thdt2, d3thdt3;
  double dphidt, d2phidt2;
} bhr_particle;

typedef struct bhr_info {
  int N, M;
  double dx, dtheta, dt;
  int nt;             /* steps of a full run                                 */
  int Fr;
  int steps_done;
  int rows_done;      /* waveform rows produced so far                       */
  int has_source;
  double r_plus;
  size_t device_bytes;
  int tile_rows;      /* stage tile height the autotuner chose (8 or 16)   */
  int persistent;     /* 1: persistent stage kernels (one block per SM)      */
  int tiling;         /* bhr_tiling: the stage kernels this solve runs       */
  int prefetch_ahead; /* one-tile-per-block tilings: each block prefetches into
                         L2 the stage input of the block this many places
                         later in launch order (0: none); autotuned with the
                         tiling                                              */
} bhr_info;

typedef struct bhr_solver bhr_solver;

/* Grid of HighOrder/main.c:64-183 (x_c[N], r_c[N], theta[M]); host only. */
int bhr_grid(const bhr_params *p, double *x_c, double *r_c, double *theta);

/* Creates a solve: grid, coefficient tables, fields, initial data on the
 * device.  Replaces the set-up half of body() (HighOrder/body.cu:30-60)
 * and kernel_init (HighOrder/kern.cu:84-169). */
int bhr_solver_create(const bhr_params *p, bhr_solver **out);
void bhr_solver_destroy(bhr_solver *s);
int bhr_solver_info(const bhr_solver *s, bhr_info *info);

/* Trajectory input: rows of the 10 .traj columns t r theta dr/dt dtheta/dt
 * dphi/dt phi E Lz Q (row-major, nrows x 10).  The data are copied in.
 * Replaces the fopen/fscanf consumption of HighOrder/body.cu:77,97-120.
 * The per-step source records of the first 8192 steps are built before
 * this returns (a particle off the grid there is reported here); the rest
 * are built on a host thread while the solver steps, and a step call that
 * reaches a step whose particle is off the grid, inside the horizon or on a
 * pole returns that error (BHR_INVALID_ARG) without launching.  If a call
 * that replaces a trajectory fails, the solve keeps no usable records: its
 * step calls return BHR_INVALID_ARG until a trajectory is set. */
int bhr_solver_set_trajectory(bhr_solver *s, const double *rows, int nrows);
int bhr_solver_load_trajectory(bhr_solver *s, const char *path);

/* Advances nsteps full time steps (source, three SSP-RK3 stages with
 * closures, extraction, time integration, waveform rows on output steps).
 * Replaces one pass of the loop at HighOrder/body.cu:105-215. */
int bhr_solver_step(bhr_solver *s, int nsteps);
/* Runs to the final time and, when path_prefix is not NULL, writes
 * <dir>/hm0<m>_<name>.dat or hmm<|m|>_<name>.dat in the reference format
 * (HighOrder/body.cu:63-70,208) plus a %.17g companion <file>.full.
 * Replaces the whole of body(). */
int bhr_solver_run(bhr_solver *s, const char *out_dir, const char *name);

/* Writes waveform rows (as bhr_solver_waveform returns them) to
 * <dir>/hm<m>_<name>.dat (hmm<|m|>_ for m < 0) in the reference's row format
 * "%lf %g x14" (HighOrder/body.cu:208) and a "%.17g" companion <file>.full
 * with dE/dt appended.  Host only. */
int bhr_write_waveform(const char *out_dir, const char *name, double m, const double *t, const double *h,
                       const double *dedt, int nrows);

/* Waveform rows produced so far: t[r] (= timer - Xmax), h[r*14 + 2l] = h+
 * and h[r*14+2l+1] = hx for l = |m|+0..6, dedt[r] (HighOrder/body.cu:
 * 174-212).  Any output pointer may be NULL. */
int bhr_solver_waveform(bhr_solver *s, double *t, double *h, double *dedt, int max_rows, int *nrows);

/* Field access for checks: full M x N planes with the boundary closure
 * applied (what the reference holds after kernel_boundary2b). */
int bhr_solver_get_state(bhr_solver *s, double *qre, double *qim, double *pre, double *pim);
int bhr_solver_set_state(bhr_solver *s, const double *qre, const double *qim, const double *pre,
                         const double *pim);
/* psi at the extraction column after the last step (d_qre_buff/d_qim_buff
 * of HighOrder/kern.cu:750-751) and the running integrals int/dint of
 * HighOrder/body.cu:178-186. */
int bhr_solver_get_extraction(bhr_solver *s, double *psi_re, double *psi_im, double *int_re, double *int_im,
                              double *dint_re, double *dint_im);
/* Source planes (tred/timd of HighOrder/kern.cu:15-16) for the current step
 * as the device built them (zero off the patch). */
int bhr_solver_get_source(bhr_solver *s, double *tre, double *tim);
/* The raw samples behind the waveform rows: psi(theta) at the extraction
 * column (psi_re/psi_im[r*M + b], M values per row) on the step of each of
 * the first max_rows rows -- the HighOrder/kern.cu:750-751 column copy on
 * output steps, for projections of the caller's own. */
int bhr_solver_psi_samples(bhr_solver *s, double *psi_re, double *psi_im, int max_rows, int *nrows);

/* Checkpoint and resume (no counterpart in the reference, which rebuilds
 * each solve from scratch): the bytes a checkpoint of this solve needs now
 * (they grow with the waveform rows written), a copy of its resumable
 * state -- the four field planes, the extraction column and its two time
 * integrals, the step and row counters, the timer and the waveform rows so
 * far -- into a caller buffer, and the restore of such a copy into a solve
 * created with the same parameters (and, for a sourced solve, given the
 * same trajectory).  A restored solve continues bit-identically to the one
 * that was checkpointed. */
size_t bhr_solver_checkpoint_size(bhr_solver *s);
int bhr_solver_checkpoint(bhr_solver *s, void *buf, size_t size);
int bhr_solver_restore(bhr_solver *s, const void *buf, size_t size);

/* Advances nsteps steps like bhr_solver_step and reports the device time
 * between CUDA events recorded on the solver stream around them. */
int bhr_solver_time_steps(bhr_solver *s, int nsteps, double *ms);

/* Device stream the solver launches on (a cudaStream_t). */
void *bhr_solver_stream(bhr_solver *s);
/* Times nsteps steps on the solver stream with CUDA events; per-kernel
 * average durations in ms for: source, stage1, stage2, stage3, extract
 * (BHR_RK4: the stage3 slot holds stages 3 and 4 together). */
int bhr_solver_profile(bhr_solver *s, int nsteps, double *avg_ms5, double *total_ms);

/* The particle-only bilinear coefficients of the point-particle source:
 * C[k] multiplies DelR^(i) DelTH^(j) for (i,j) = (0,0) (0,1) (0,2) (1,0)
 * (1,1) (2,0).  Replaces the Maple block of HighOrder/kern.cu:1229-2664. */
int bhr_source_coefficients(const bhr_particle *pt, double a, double mass, double m, double *c_re6,
                            double *c_im6);

/* Spin-weighted spherical harmonic of HighOrder/proj.c:16-35 (s = -2). */
double bhr_swsh(double ell, double m, double theta);

/* Source-free SSP-RK3 steps on a state the caller owns, allocating nothing.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * a framework that reserves the device memory up front and hands out
 * pieces of it, or a latency-critical loop that may not take cudaMalloc's
 * implicit device synchronisation.  `state` is device memory holding the
 * four closed M x N FP64 planes q_re, q_im, p_re, p_im back to back
 * (16-byte aligned); it is advanced nsteps steps in place on `stream` (a
 * cudaStream_t, NULL for the default stream) and closed again on return.
 * p->dt must be > 0.  The two intermediate stages and the coefficient
 * tables live in one fixed file-scope device array of about 11 MB, so
 * grids are limited to N*M <= 131072, N <= 16384, M <= 1024; larger ones
 * are rejected with BHR_INVALID_ARG.  Every GPU that loads the library
 * holds that array until the process exits.  The first call on a device
 * looks up the array's device address and sets the stage kernels'
 * shared-memory size.  Each call waits for its stream to finish and reads
 * a status flag back, so it must not be called while that stream is being
 * captured.  `stream` must belong to p->device; the calling thread's
 * current device is restored on return.  All calls share the array and it
 * keeps the last call's contents (a call with the same grid, spin, m and
 * dt reuses the coefficient tables; the error flag is cleared every call):
 * calls that overlap on the GPU (other streams, other host threads'
 * streams) race. */
int bhr_step_noalloc(const bhr_params *p, double *state, int nsteps, void *stream);

/* ---- Batch engine: many solves per device, advanced together ----------
 * No counterpart in the reference, which runs one body() per process and
 * one process per (trajectory, m) job (HighOrder/main.c:50-55).  The
 * engine queues requests, admits them in arrival order while their device
 * memory fits `hbm_budget_bytes` (one is always admitted when none runs;
 * while the oldest does not fit, later ones that do are admitted ahead of
 * it, at most 64 of them), and advances every running solve with one
 * launch per RK stage (per group of up to 112 solves) over a (solve, tile)
 * work-list.  Requests submitted while others run join at the
 * next bhr_engine_step (continuous batching).  A request's waveform does
 * not depend on the other requests in the batch: it is bit-identical to the
 * same request run alone in an engine, and matches bhr_solver_step's to
 * FP64 rounding. */
typedef struct bhr_engine bhr_engine;

typedef struct bhr_request_info {
  int state;          /* 0 unknown, 1 queued, 2 running, 3 done, 4 failed */
  int status;         /* bhr_status of a failed request */
  int steps_total, steps_done, nrows;
  double submit_s, start_s, finish_s; /* host steady clock, seconds */
} bhr_request_info;

typedef struct bhr_engine_counters {
  int queued, running, finished, tiles;
  long long batch_steps;  /* bhr_engine_step iterations run */
  double point_updates;   /* grid points advanced one step, all solves */
  double device_ms;       /* device time of the batch steps (CUDA events) */
  size_t bytes_in_use, budget;
} bhr_engine_counters;

int bhr_engine_create(int device, size_t hbm_budget_bytes, bhr_engine **out);
void bhr_engine_destroy(bhr_engine *e);
/* Queues a solve; traj_rows (nrows x 10, the .traj columns) may be NULL for
 * a source-free solve.  The request's tile height is fixed at 16 rows, so
 * p->M must be a multiple of 16.  Thread-safe against bhr_engine_step. */
int bhr_engine_submit(bhr_engine *e, const bhr_params *p, const double *traj_rows, int nrows, int64_t *id);
/* Admits what fits, advances all running solves by
 * min(max_steps, fewest steps any of them has left), retires the finished
 * ones; *running = solves still running.  If a bounded device wait of a
 * stage kernel gives up, the running solves' fields are unknown: this and
 * every later call return BHR_TIMEOUT, and the engine is to be destroyed. */
int bhr_engine_step(bhr_engine *e, int max_steps, int *running);
int bhr_engine_poll(bhr_engine *e, int64_t id, bhr_request_info *info);
/* Waveform rows of a finished request (layout of bhr_solver_waveform). */
int bhr_engine_result(bhr_engine *e, int64_t id, double *t, double *h, double *dedt, int max_rows, int *nrows);
int bhr_engine_stats(bhr_engine *e, bhr_engine_counters *st);

/* ---- trajectory generation (GenOT) --------------------------------------
 * Host code (no device work) restating GenOT, the reference's generator of
 * the .traj worldlines the solver reads: an adiabatic inspiral (tabulated,
 * from frequency-domain fluxes), the generalised Ori-Thorne transition and
 * the geodesic plunge, in Mino time (GenOT/ParamWLMino.cc), then that
 * worldline in Boyer-Lindquist time (GenOT/WL_BL.cc).  Units G = c = M = 1. */
typedef struct bhr_genot_params {
  double a;        /* black-hole spin (ParamWLMino argument 1)                */
  double eta;      /* mass ratio (argument 2)                                 */
  double LTi, LTf; /* Ori-Thorne times at which the transition begins and
                      ends (arguments 4, 5)                                   */
  double r_start;  /* radius at which the output starts (argument 6)          */
  double dl;       /* Mino-time step of the output: 0.1 in the reference      */
  int model;       /* E, L, Q through the transition (argument 7): 1 = LSO
                      values plus a constant and a quadratic term, 2 = plus a
                      quadratic and a cubic term                              */
} bhr_genot_params;
/* The Mino-time worldline (GenOT/ParamWLMino.cc:332-531).  insp: n_insp rows
 * of 11 columns, the adiabatic inspiral table (time, Mino time, r,
 * eccentricity, theta_inc in degrees, E, L, Q, and the E, L, Q fluxes, Mino
 * time and fluxes with the mass ratio scaled out; its last row is the last
 * stable orbit).  ot: n_ot rows (T, X) of the Ori-Thorne function, the
 * solution of X'' = -X^2 - T that approaches sqrt(-T) as T -> -infinity.
 * Writes rows (lambda, r, theta_inc, E, L, Q) from r_start until r passes
 * r+ - 0.5 or lambda passes the end of the transition by 100; out = NULL
 * only counts them (*n_out).  transition (4 doubles, may be NULL) receives
 * the Mino times at which the transition begins and ends and r there
 * (the output's lambda runs on the transition's origin).  Inputs the
 * reference exits on (model, LTf past the table, r_start or a Mino time
 * outside the inspiral table) and a negative A or B return
 * BHR_INVALID_ARG. */
int bhr_genot_mino(const bhr_genot_params *p, const double *insp, int n_insp, const double *ot, int n_ot,
                   double *out, int max_rows, int *n_out, double *transition);
typedef struct bhr_genot_bl_params {
  double a;            /* spin (WL_BL argument 1)                             */
  double lambda_start; /* Mino time at which the worldline starts (argument 3) */
  double t_stop;       /* BL time at which it stops (argument 4)              */
  double chi0_deg;     /* initial polar phase chi, cos(theta) =
                          sin(theta_inc) cos(chi) (argument 5)                */
  double phi0_deg;     /* initial axial angle (argument 6)                    */
  double dt;           /* BL time step: 0.001 in the reference                */
} bhr_genot_bl_params;
/* The worldline in BL time (GenOT/WL_BL.cc:7-261): classical RK4 in t for
 * (lambda, chi, phi) over splines of the Mino-time rows (n_mino rows of 6,
 * as bhr_genot_mino writes them; the look-ups use rows 1..n_mino-1, as the
 * reference's do).  Rows t, r, theta, dr/dt, dtheta/dt, dphi/dt, phi, E,
 * L, Q (the .traj columns) for t = 0, dt, ... <= t_stop: every stride-th
 * row to out (when not NULL), every row to the text file path (when not
 * NULL; the reference's "%.12e" format).  *thf_deg and *thdot_pos: theta
 * (degrees) and the sign of dtheta/dlambda at the last row (the reference
 * names the file by them).  With out, path and thf_deg all NULL only
 * *n_out is set (the rows out would receive). */
int bhr_genot_bl(const bhr_genot_bl_params *p, const double *mino, int n_mino, int stride, double *out, int max_rows,
                 int *n_out, double *thf_deg, int *thdot_pos, const char *path);
/* The Ori-Thorne function on T = T0 + k dT, k < rows (X[k]): the solution
 * of X'' = -X^2 - T that approaches sqrt(-T) as T -> -infinity, integrated
 * from its asymptotic series at T_start (< 0, <= T0) by adaptive classical
 * RK4 with step doubling (relative tolerance 1e-13).  Replaces the table
 * GenOT ships (GenOT/OT_X_vs_L.dat, T0 = -40, dT = 0.001, 43411 rows). */
int bhr_genot_ot_table(double T0, double dT, int rows, double T_start, double *X);
/* The reference's .traj file name, a<a>_thi<theta_inc>_thf<theta_f>_<p|n>.traj
 * (GenOT/WL_BL.cc:101-153). */
int bhr_genot_traj_name(double a, double thi0_deg, double thf_deg, int thdot_pos, char *buf, int buflen);

/* The reason for the last failed call made on the calling thread (the
 * string is per thread and valid until that thread's next failing call). */
const char *bhr_last_error_string(void);
/* Device self-check of the bounded waits (no counterpart in the reference):
 * one block waits on a shared-memory barrier that nothing completes; the
 * wait gives up after its iteration limit (about a second) and the kernel
 * returns normally with *device_status = BHR_TIMEOUT, the same path a stage
 * kernel takes when its tile data never arrive.  The device stays usable. */
int bhr_selftest_bounded_wait(int device, int *device_status);
/* Device self-check of the hand-written FP64 reciprocal and square root
 * (Newton-Raphson from the hardware approximations) that the stage and
 * coefficient kernels use (no counterpart in the reference): for the n
 * values x, out[0..n) = the reciprocal, out[n..2n) = CUDA's 1.0 / x,
 * out[2n..3n) = the square root, out[3n..4n) = CUDA's sqrt(x), all computed
 * on the device. */
int bhr_selftest_math(int device, const double *x, int n, double *out);
int bhr_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
