/*
 * teuk_oracle.h -- FP64 CPU oracle for the 2+1 s=-2 Teukolsky evolution.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the oracle: tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it to
 * compare the CUDA path against.  It is never linked into, called by, or
 * shipped with the product library (bh_ringdown_b200).
 *
 * It restates, in plain C with OpenMP over theta rows, the algorithm of the
 * reference TD_GPU_code/HighOrder path (file:line citations are relative to
 * the reference project root):
 *   grid()                 HighOrder/main.c:64-183
 *   kernel_init            HighOrder/kern.cu:84-169
 *   kernel_rhs1/2          HighOrder/kern.cu:171-299, 452-580
 *   kernel_update1/2/3     HighOrder/kern.cu:301-318, 582-620
 *   kernel_boundary1a/1b   HighOrder/kern.cu:320-449
 *   kernel_boundary2a/2b   HighOrder/kern.cu:622-753
 *   reset_sourced/sourced  HighOrder/kern.cu:755-768, 1185-2683 (deposit
 *                          geometry; the particle-only bilinear coefficients
 *                          of the source are supplied by the caller)
 *   body() time loop       HighOrder/body.cu:56-215
 *   swsh/project           HighOrder/proj.c:4-75
 */
#ifndef TEUK_ORACLE_H
#define TEUK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
  int N;            /* radial points (parm.h N)                              */
  int M;            /* theta points  (parm.h M)                              */
  double Xmin;      /* inner grid coordinate (parm.h Xmin)                   */
  double Xmax;      /* outer grid coordinate (parm.h Xmax)                   */
  double mass;      /* BH mass (main.c: mass=1)                              */
  double a;         /* spin (main.c: aa)                                     */
  double m;         /* azimuthal number, a double as in body(mm)            */
  double dt;        /* time step                                             */
  double T;         /* final time (parm.h T)                                 */
  int Fr;           /* output cadence in steps (parm.h Fr)                   */
  int PTSX, PTSY;   /* source patch (parm.h PTSX/PTSY)                       */
  double wr_fac;    /* radial smearing: wr = wr_fac*dx*(1-r+/rp), ref 2.0    */
  double wt_fac;    /* polar smearing:  wt = wt_fac*dtheta, ref 6.0          */
  double out_start; /* waveform rows written when k*dt >= out_start (ref Xmax+200) */
  int ext_col;      /* extraction column (ref N-1)                           */
} orc_params;

/* Particle state for one step, as body.cu:112-124 hands it to sourced(). */
typedef struct orc_particle {
  double rp, tp, phip, E, lz, Q;
  double drdt, d2rdt2, d3rdt3;
  double dthdt, d2thdt2, d3thdt3;
  double dphidt, d2phidt2;
} orc_particle;

/* Bilinear coefficients of the particle source: the six complex numbers
 * C[k] multiplying DelR^(i) * DelTH^(j) for (i,j) in the fixed order
 * (0,0) (0,1) (0,2) (1,0) (1,1) (2,0).  Provided by a caller-supplied
 * function so the oracle carries no copy of any particular evaluator. */
typedef void (*orc_coef_fn)(const orc_particle *p, double a, double mass,
                            double m, double *c_re6, double *c_im6);

typedef struct orc_solver orc_solver;

orc_solver *orc_create(const orc_params *p);
void orc_destroy(orc_solver *s);

/* Grid (main.c:64-183): x_c[N], r_c[N], theta[M]. */
void orc_get_grid(const orc_solver *s, double *x_c, double *r_c, double *theta);
/* Coefficient plane k in order bb,cc,ee,a_re,a_im,d_re,d_im,v_re,v_im. */
void orc_get_coeff(const orc_solver *s, int k, double *out);

void orc_set_state(orc_solver *s, const double *qre, const double *qim,
                   const double *pre, const double *pim);
void orc_get_state(const orc_solver *s, double *qre, double *qim,
                   double *pre, double *pim);
/* Closure of kernel_boundary2a + 2b applied to the main state. */
void orc_apply_closure(orc_solver *s);
/* psi = exp(-(x-c)^2/(2 w^2)) * swsh(l, m, theta) on every point, Pi = 0,
 * followed by the closure (initial data for the source-free configs). */
void orc_init_gaussian(orc_solver *s, double center, double width, double ell);

/* Source planes (tred/timd), each M*N, or NULL to zero them. */
void orc_set_source(orc_solver *s, const double *tre, const double *tim);
void orc_get_source(const orc_solver *s, double *tre, double *tim);
/* reset_sourced + sourced with the bilinear coefficients given. */
void orc_deposit_source(orc_solver *s, const orc_particle *pt,
                        const double *c_re6, const double *c_im6,
                        double timer, double start);

/* One step (body.cu:131-165), current source held fixed: SSP-RK3 as the
 * reference, or classical RK4 after orc_set_integrator(s, 1) (an option the
 * reference does not have; 0 restores SSP-RK3). */
void orc_step(orc_solver *s);
void orc_set_integrator(orc_solver *s, int integrator);
/* kernel_rhs (HighOrder/kern.cu:171-299) of the closure of in4 (four M x N
 * planes) into out4, interior points; between steps only. */
void orc_eval_rhs(orc_solver *s, const double *in4, double *out4);
/* Column ext_col of psi after the last step (kernel_boundary2b copy). */
void orc_get_ext(const orc_solver *s, double *re, double *im);

/* Spin-weighted harmonic and Boole projection (proj.c). qq needs M+1 slots. */
double orc_swsh(double ell, double ml, double the);
double orc_project(double *qq, int M, double l, double m);

/* Full body() loop.  traj: nrows x 10 row-major (.traj columns) or NULL for a
 * source-free run.  coef: bilinear source coefficient provider (needed when
 * traj is given).  Outputs, each sized for max_rows waveform rows:
 *   out_t[r], out_h[r*14 + 2l] = h+ (l=|m|+l), out_h[r*14+2l+1] = hx,
 *   out_dedt[r].  ext_every > 0 stores psi(ext_col, theta) every ext_every
 * steps into ext_re/ext_im (rows of M) up to max_ext rows.
 * Returns the number of waveform rows written, or -1 on error. */
int orc_run(orc_solver *s, const double *traj, int nrows, orc_coef_fn coef,
            int nsteps_limit, double *out_t, double *out_h, double *out_dedt,
            int max_rows, int *out_step, int ext_every, double *ext_re,
            double *ext_im, int max_ext, int *n_ext);

int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
