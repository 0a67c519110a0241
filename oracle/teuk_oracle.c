/*
 * teuk_oracle.c -- FP64 CPU oracle for the 2+1 s=-2 Teukolsky evolution.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle that tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg compare the CUDA path against.  Nothing in
 * the product library links or calls this file.
 *
 * Each function restates one piece of the reference TD_GPU_code/HighOrder
 * path (citations relative to the reference project root).  The reference
 * fixes N, M, Xmin, Xmax at compile time (HighOrder/parm.h:1-13); here they
 * are fields of orc_params.  Layout is the reference's idx(b,a) = N*b + a
 * (HighOrder/parm.h:13): theta rows b, radial columns a contiguous.
 *
 * Deliberate differences from the reference, all outside what its outputs
 * depend on: the source deposit skips columns >= N (the reference has no
 * upper bound and writes past the row, HighOrder/kern.cu:1206); project()
 * gets an M+1 buffer instead of writing one past the array
 * (HighOrder/proj.c:45).
 */
#include "teuk_oracle.h"

#include <complex.h>
#include <stddef.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Constants exactly as the reference spells them. */
#define ORC_PI_PARM 3.14159265358979       /* HighOrder/parm.h:12 (Pi)        */
#define ORC_PIE 3.141592653589793          /* HighOrder/kern.cu:1188 (pie)    */
#define ORC_THIRD 0.33333333333333333      /* HighOrder/kern.cu:46 (third)    */
#define ORC_D1X 0.016666666666667          /* HighOrder/kern.cu:196           */

struct orc_solver {
  orc_params p;
  int N, M;
  double dx, dtheta;
  double *x_c, *r_c, *theta;
  double *coef[9];           /* bb cc ee a_re a_im d_re d_im v_re v_im */
  double *u[4];              /* qre qim pre pim       (reference q*, p*)     */
  double *uc[4];             /* stage arrays          (reference *_c)        */
  int integrator;            /* 0 SSP-RK3 (reference), 1 classical RK4        */
  double *acc[4];            /* RK4 accumulator, allocated on first use       */
  double *rhs[4];
  double *tred, *timd;
  double *ext_re, *ext_im;   /* d_qre_buff / d_qim_buff                      */
};

enum { C_BB, C_CC, C_EE, C_ARE, C_AIM, C_DRE, C_DIM, C_VRE, C_VIM };

static double *zalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ---------------------------------------------------------------------- */
/* grid(): HighOrder/main.c:64-183 (uniform x, theta; Omega layer; Newton
 * inversion of the Kerr tortoise coordinate from the outer end inwards). */
static void orc_grid(orc_solver *s) {
  const int N = s->N, M = s->M;
  const double mass = s->p.mass, aa = s->p.a;
  const double Xmin = s->p.Xmin, Xmax = s->p.Xmax;
  double *tx = zalloc((size_t)N);
  for (int l = 0; l < N; l++) s->x_c[l] = Xmin + (double)l * s->dx;
  for (int m = 0; m < M; m++) s->theta[m] = (double)m * s->dtheta;
  const double rin = Xmin + (Xmax - Xmin) * 0.64;
  const double Rrpt = Xmax + 1e-6;
  for (int l = 0; l < N; l++) {
    double x = s->x_c[l];
    double om = (x < rin) ? 1.0 : 1.0 - pow((x - rin) / (Rrpt - rin), 4);
    tx[l] = x / om;
  }
  const double rp = mass + sqrt(mass * mass - aa * aa);
  const double rm = mass - sqrt(mass * mass - aa * aa);
  if (mass == 0.0) {
    for (int l = 0; l < N; l++) s->r_c[l] = tx[l];
  } else {
    const double tol = 1e-12;
    /* Horizon floor: where r - r+ drops below FP64 resolution the reference
     * iteration takes log(0) and returns NaN.  From the first point whose
     * Newton step lands at or inside r+, this point and every point further
     * in get the next double above r+ instead. */
    const double r_floor = nextafter(rp, INFINITY);
    int floored = 0;
    double r_old = tx[N - 1], r_new = r_old;
    for (int l = N - 1; l >= 0; l--) {
      double diff;
      if (floored) {
        s->r_c[l] = r_floor;
        continue;
      }
      do {
        double drdx = (r_old * r_old + aa * aa - 2.0 * mass * r_old) / (r_old * r_old + aa * aa);
        double x_o;
        if (mass == aa)
          x_o = r_old + 2.0 * aa * log(r_old / aa - 1.0) - 2.0 * aa * aa / (r_old - aa);
        else if (aa == 0.0)
          x_o = r_old + 2.0 * mass * log(r_old / (2.0 * mass) - 1.0);
        else
          x_o = r_old + (rp * rp + aa * aa) / (rp - rm) * log(r_old / rp - 1.0) -
                (rm * rm + aa * aa) / (rp - rm) * log(r_old / rm - 1.0);
        r_new = r_old + (tx[l] - x_o) * drdx;
        if (!(r_new > rp) || !isfinite(r_new)) {
          r_new = r_floor;
          floored = 1;
          break;
        }
        diff = fabs(r_new - r_old) / r_old;
        r_old = r_new;
      } while (diff > tol);
      s->r_c[l] = r_new;
      r_old = r_new;
    }
  }
  free(tx);
}

/* ---------------------------------------------------------------------- */
/* kernel_init: HighOrder/kern.cu:84-169.  Nine real coefficient planes for
 * theta rows 3..M-4 (other rows stay zero); fields zeroed. */
static void orc_coefficients(orc_solver *s) {
  const int N = s->N, M = s->M;
  const double mass = s->p.mass, spin = s->p.a, em = s->p.m;
  const double Xmin = s->p.Xmin, Xmax = s->p.Xmax;
  const double rin = Xmin + (Xmax - Xmin) * 0.64;
  const double Rrpt = Xmax + 1e-6;
  const double a2 = spin * spin, a4 = a2 * a2;
#pragma omp parallel for schedule(static)
  for (int k = 3; k < M - 3; k++) {
    const double y = s->theta[k];
    const double sn = sin(y), cs = cos(y);
    const double cot = 1.0 / tan(y), csc = 1.0 / sin(y);
    for (int j = 0; j < N; j++) {
      const double x = Xmin + (double)j * s->dx;
      double Om, Om1, Om2;
      if (x < rin) {
        Om = 1.0; Om1 = 0.0; Om2 = 0.0;
      } else {
        const double L = Rrpt - rin, L4 = pow(L, 4);
        Om = 1.0 - pow((x - rin) / L, 4);
        Om1 = -4.0 * pow(x - rin, 3) / L4;
        Om2 = -12.0 * pow(x - rin, 2) / L4;
      }
      const double cL = Om - x * Om1;            /* coefL */
      const double eR = Om * s->r_c[j];
      const double eR2 = eR * eR, eR3 = eR2 * eR, eR5 = eR3 * eR2;
      const double Om_2 = Om * Om, Om_3 = Om_2 * Om, Om_4 = Om_2 * Om_2, Om_5 = Om_4 * Om;
      const double cL2 = cL * cL, cL3 = cL2 * cL;
      const double Sg = eR2 + Om_2 * a2;                           /* eR^2+Om^2 a^2 */
      const double Dt = eR2 - 2.0 * eR * mass * Om + Om_2 * a2;    /* Delta-tilde   */
      const double bir = -((2.0 * cL - Om_2) * Sg * Sg) / cL2 + a2 * Dt * sn * sn;
      const double At = (2.0 * (cL - Om_2) * Sg * Sg) / (bir * cL2);
      const double Ar = -((Om_2 * Sg * Sg) / (bir * cL2));
      const double Ayy = -(Dt / bir);
      const double BtR =
          -((Om * (eR3 * (4.0 * cL2 * (eR - 3.0 * mass * Om) + 2.0 * cL * eR2 * Om1 + eR2 * Om * Om2 * x) +
                   2.0 * eR *
                       (cL2 * Om_2 * (5.0 * eR - 4.0 * mass * Om) - 3.0 * cL3 * (eR - 2.0 * mass * Om) +
                        2.0 * cL * eR2 * Om_2 * Om1 + eR2 * Om_3 * Om2 * x) *
                       a2 +
                   (-6.0 * cL3 * Om_2 + 6.0 * cL2 * Om_4 + 2.0 * cL * eR * Om_4 * Om1 + eR * Om_5 * Om2 * x) * a4)) /
            (bir * cL3 * eR));
      const double g1 = 2.0 * Om * Om1 - 2.0 * Om1 * Om1 * x + Om * Om2 * x;
      const double BrR =
          -((Om * (eR5 * g1 + 2.0 * eR3 * Om_2 * g1 * a2 +
                   Om_4 * (6.0 * Om_2 + 2.0 * Om1 * Om1 * x * (-eR + 3.0 * x) +
                           Om * (2.0 * eR * Om1 - 12.0 * Om1 * x + eR * Om2 * x)) *
                       a4 +
                   2.0 * cL2 * eR *
                       (2.0 * eR3 - 6.0 * eR2 * mass * Om + 5.0 * eR * Om_2 * a2 - 4.0 * mass * Om_3 * a2))) /
            (bir * cL3 * eR));
      const double CR = (Dt * (2.0 * eR2 + 6.0 * eR * mass * Om - 6.0 * Om_2 * a2 + 4.0 * eR2 * cot * cot -
                               4.0 * em * eR2 * cot * csc + em * em * eR2 * csc * csc)) /
                        (bir * eR2);
      const double BtI = (2.0 * spin *
                          (em * (-(Om_2 * Sg) + cL * (eR2 + 2.0 * eR * mass * Om + Om_2 * a2)) -
                           2.0 * cL * Dt * cs)) /
                         (bir * cL);
      const double BrI = (-2.0 * em * Om_2 * spin * Sg) / (bir * cL);
      const double CI = (2.0 * em * Om * spin * (eR2 + 2.0 * eR * mass * Om - 3.0 * Om_2 * a2)) / (bir * eR);
      const size_t id = (size_t)N * k + j;
      const double bb = -(At + sqrt(At * At + 4.0 * Ar)) / 2.0;
      s->coef[C_BB][id] = bb;
      s->coef[C_CC][id] = Ayy;
      s->coef[C_EE][id] = At + bb;
      s->coef[C_ARE][id] = -BtR;
      s->coef[C_AIM][id] = -BtI;
      s->coef[C_DRE][id] = BrR - bb * BtR;
      s->coef[C_DIM][id] = BrI - bb * BtI;
      s->coef[C_VRE][id] = -CR;
      s->coef[C_VIM][id] = -CI;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* Stencils of HighOrder/kern.cu:192-261 (6th-order centred first and second
 * derivatives, 9-point Kreiss-Oliger).  f points at the centre, st is the
 * stride between neighbours. */
static inline double d1(const double *f, ptrdiff_t st) {
  return 45.0 * (f[st] - f[-st]) - 9.0 * (f[2 * st] - f[-2 * st]) + (f[3 * st] - f[-3 * st]);
}
static inline double d2(const double *f, ptrdiff_t st) {
  return 2.0 * (f[3 * st] + f[-3 * st]) - 27.0 * (f[2 * st] + f[-2 * st]) +
         270.0 * (f[st] + f[-st]) - 490.0 * f[0];
}
static inline double ko8(const double *f) {
  return (f[4] + f[-4]) - 8.0 * (f[3] + f[-3]) + 28.0 * (f[2] + f[-2]) - 56.0 * (f[1] + f[-1]) + 70.0 * f[0];
}

/* kernel_rhs1 / kernel_rhs2: HighOrder/kern.cu:171-299 and 452-580.  v is the
 * state the RHS is evaluated on (u for stage 1, the *_c arrays after). */
static void orc_rhs(orc_solver *s, double *const v[4]) {
  const int N = s->N, M = s->M;
  const double odx = 1.0 / s->dx, odth = 1.0 / s->dtheta, odt = 1.0 / s->p.dt;
  const double cx = ORC_D1X * odx;
  const double cy = 0.05 * ORC_THIRD * odth;
  const double cyy = 0.05 * ORC_THIRD * ORC_THIRD * odth * odth;
  const double cko = 0.1 * 0.0625 * odt;
  double *const *c = s->coef;
#pragma omp parallel for schedule(static)
  for (int b = 3; b < M - 3; b++) {
    const double ctan = tan(0.5 * ORC_PI_PARM - s->theta[b]);
    for (int a = 3; a < N - 3; a++) {
      const size_t id = (size_t)N * b + a;
      const double dbdx = d1(c[C_BB] + id, 1) * cx;
      const double dre = c[C_DRE][id] - dbdx * c[C_EE][id];
      const double qy_r = d1(v[0] + id, N) * cy, qyy_r = d2(v[0] + id, N) * cyy;
      const double qy_i = d1(v[1] + id, N) * cy, qyy_i = d2(v[1] + id, N) * cyy;
      const double ll_r = qyy_r + ctan * qy_r;
      const double ll_i = qyy_i + ctan * qy_i;
      const double qx_r = d1(v[0] + id, 1) * cx, qx_i = d1(v[1] + id, 1) * cx;
      const double px_r = d1(v[2] + id, 1) * cx, px_i = d1(v[3] + id, 1) * cx;
      double kq_r = 0.0, kq_i = 0.0, kp_r = 0.0, kp_i = 0.0;
      if (a >= 4 && a < N - 4) {
        kq_r = ko8(v[0] + id); kq_i = ko8(v[1] + id);
        kp_r = ko8(v[2] + id); kp_i = ko8(v[3] + id);
      }
      kq_r *= cko; kq_i *= cko; kp_r *= cko; kp_i *= cko;
      const double q_r = v[0][id], q_i = v[1][id], p_r = v[2][id], p_i = v[3][id];
      s->rhs[0][id] = -c[C_BB][id] * qx_r + p_r - kq_r;
      s->rhs[1][id] = -c[C_BB][id] * qx_i + p_i - kq_i;
      s->rhs[2][id] = s->tred[id] + c[C_EE][id] * px_r - kp_r + c[C_CC][id] * ll_r + dre * qx_r -
                      c[C_DIM][id] * qx_i - c[C_ARE][id] * p_r + c[C_AIM][id] * p_i -
                      c[C_VRE][id] * q_r + c[C_VIM][id] * q_i;
      s->rhs[3][id] = s->timd[id] + c[C_EE][id] * px_i - kp_i + c[C_CC][id] * ll_i + dre * qx_i +
                      c[C_DIM][id] * qx_r - c[C_ARE][id] * p_i - c[C_AIM][id] * p_r -
                      c[C_VRE][id] * q_i - c[C_VIM][id] * q_r;
    }
  }
}

/* kernel_update1/2/3: HighOrder/kern.cu:301-318, 582-600, 602-620 (SSP-RK3
 * in Shu-Osher form, interior points only). */
static void orc_update(orc_solver *s, int stage) {
  const int N = s->N, M = s->M;
  const double dt = s->p.dt;
#pragma omp parallel for schedule(static)
  for (int b = 3; b < M - 3; b++)
    for (int a = 3; a < N - 3; a++) {
      const size_t id = (size_t)N * b + a;
      for (int f = 0; f < 4; f++) {
        if (stage == 1)
          s->uc[f][id] = s->u[f][id] + dt * s->rhs[f][id];
        else if (stage == 2)
          s->uc[f][id] = 0.25 * (3.0 * s->u[f][id] + s->uc[f][id] + dt * s->rhs[f][id]);
        else
          s->u[f][id] = ORC_THIRD * (s->u[f][id] + 2.0 * s->uc[f][id] + 2.0 * dt * s->rhs[f][id]);
      }
    }
}

/* kernel_boundary1a/2a: HighOrder/kern.cu:320-409 and 622-711.  Pole rows of
 * columns 3..N-4: even m extrapolates (4 f1 - f2)/3 in the order rows 2, 1,
 * M-3, M-2, 0, M-1; odd m zeroes them. */
static void orc_bnd_poles(orc_solver *s, double *const v[4]) {
  const int N = s->N, M = s->M;
  const int even = (((int)s->p.m) % 2 == 0);
  static const int order[6][3] = {{2, 3, 4}, {1, 2, 3}, {-3, -4, -5}, {-2, -3, -4}, {0, 1, 2}, {-1, -2, -3}};
#pragma omp parallel for schedule(static)
  for (int a = 3; a < N - 3; a++)
    for (int f = 0; f < 4; f++) {
      double *col = v[f] + a;
      for (int k = 0; k < 6; k++) {
        const int r0 = order[k][0] < 0 ? M + order[k][0] : order[k][0];
        const int r1 = order[k][1] < 0 ? M + order[k][1] : order[k][1];
        const int r2 = order[k][2] < 0 ? M + order[k][2] : order[k][2];
        col[(size_t)N * r0] = even ? (4.0 * col[(size_t)N * r1] - col[(size_t)N * r2]) * ORC_THIRD : 0.0;
      }
    }
}

/* kernel_boundary1b/2b: HighOrder/kern.cu:412-449 and 713-753.  Radial end
 * columns of every row: 2 and N-3, then 1 and N-2, then 0 and N-1. */
static void orc_bnd_ends(orc_solver *s, double *const v[4]) {
  const int N = s->N, M = s->M;
#pragma omp parallel for schedule(static)
  for (int b = 0; b < M; b++)
    for (int f = 0; f < 4; f++) {
      double *row = v[f] + (size_t)N * b;
      row[2] = (4.0 * row[3] - row[4]) * ORC_THIRD;
      row[N - 3] = (4.0 * row[N - 4] - row[N - 5]) * ORC_THIRD;
      row[1] = (4.0 * row[2] - row[3]) * ORC_THIRD;
      row[N - 2] = (4.0 * row[N - 3] - row[N - 4]) * ORC_THIRD;
      row[0] = (4.0 * row[1] - row[2]) * ORC_THIRD;
      row[N - 1] = (4.0 * row[N - 2] - row[N - 3]) * ORC_THIRD;
    }
}

static void orc_copy_ext(orc_solver *s) {
  const int N = s->N;
  for (int b = 0; b < s->M; b++) {
    s->ext_re[b] = s->u[0][(size_t)N * b + s->p.ext_col];
    s->ext_im[b] = s->u[1][(size_t)N * b + s->p.ext_col];
  }
}

/* ---------------------------------------------------------------------- */
orc_solver *orc_create(const orc_params *p) {
  if (!p || p->N < 16 || p->M < 10) return NULL;
  orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
  s->p = *p;
  s->N = p->N;
  s->M = p->M;
  if (s->p.ext_col < 0 || s->p.ext_col >= p->N) s->p.ext_col = p->N - 1;
  s->dx = (p->Xmax - p->Xmin) / p->N;   /* main.c:44 */
  s->dtheta = ORC_PI_PARM / p->M;       /* main.c:45 */
  const size_t NM = (size_t)p->N * p->M;
  s->x_c = zalloc((size_t)p->N);
  s->r_c = zalloc((size_t)p->N);
  s->theta = zalloc((size_t)p->M);
  for (int k = 0; k < 9; k++) s->coef[k] = zalloc(NM);
  for (int f = 0; f < 4; f++) {
    s->u[f] = zalloc(NM);
    s->uc[f] = zalloc(NM);
    s->rhs[f] = zalloc(NM);
  }
  s->tred = zalloc(NM);
  s->timd = zalloc(NM);
  s->ext_re = zalloc((size_t)p->M);
  s->ext_im = zalloc((size_t)p->M);
  orc_grid(s);
  orc_coefficients(s);
  return s;
}

void orc_destroy(orc_solver *s) {
  if (!s) return;
  free(s->x_c); free(s->r_c); free(s->theta);
  for (int k = 0; k < 9; k++) free(s->coef[k]);
  for (int f = 0; f < 4; f++) { free(s->u[f]); free(s->uc[f]); free(s->rhs[f]); free(s->acc[f]); }
  free(s->tred); free(s->timd); free(s->ext_re); free(s->ext_im);
  free(s);
}

void orc_get_grid(const orc_solver *s, double *x_c, double *r_c, double *theta) {
  if (x_c) memcpy(x_c, s->x_c, sizeof(double) * s->N);
  if (r_c) memcpy(r_c, s->r_c, sizeof(double) * s->N);
  if (theta) memcpy(theta, s->theta, sizeof(double) * s->M);
}

void orc_get_coeff(const orc_solver *s, int k, double *out) {
  if (k >= 0 && k < 9) memcpy(out, s->coef[k], sizeof(double) * (size_t)s->N * s->M);
}

void orc_set_state(orc_solver *s, const double *qre, const double *qim, const double *pre, const double *pim) {
  const size_t bytes = sizeof(double) * (size_t)s->N * s->M;
  const double *in[4] = {qre, qim, pre, pim};
  for (int f = 0; f < 4; f++) {
    if (in[f]) memcpy(s->u[f], in[f], bytes);
    else memset(s->u[f], 0, bytes);
  }
}

void orc_get_state(const orc_solver *s, double *qre, double *qim, double *pre, double *pim) {
  const size_t bytes = sizeof(double) * (size_t)s->N * s->M;
  double *out[4] = {qre, qim, pre, pim};
  for (int f = 0; f < 4; f++)
    if (out[f]) memcpy(out[f], s->u[f], bytes);
}

void orc_apply_closure(orc_solver *s) {
  orc_bnd_poles(s, s->u);
  orc_bnd_ends(s, s->u);
  orc_copy_ext(s);
}

void orc_init_gaussian(orc_solver *s, double center, double width, double ell) {
  const int N = s->N, M = s->M;
  for (int b = 0; b < M; b++) {
    const double y = orc_swsh(ell, s->p.m, s->theta[b]);
    for (int a = 0; a < N; a++) {
      const double x = s->x_c[a] - center;
      const size_t id = (size_t)N * b + a;
      s->u[0][id] = exp(-x * x / (2.0 * width * width)) * y;
      s->u[1][id] = 0.0;
      s->u[2][id] = 0.0;
      s->u[3][id] = 0.0;
    }
  }
  orc_apply_closure(s);
}

void orc_set_source(orc_solver *s, const double *tre, const double *tim) {
  const size_t bytes = sizeof(double) * (size_t)s->N * s->M;
  if (tre) memcpy(s->tred, tre, bytes); else memset(s->tred, 0, bytes);
  if (tim) memcpy(s->timd, tim, bytes); else memset(s->timd, 0, bytes);
}

void orc_get_source(const orc_solver *s, double *tre, double *tim) {
  const size_t bytes = sizeof(double) * (size_t)s->N * s->M;
  if (tre) memcpy(tre, s->tred, bytes);
  if (tim) memcpy(tim, s->timd, bytes);
}

/* reset_sourced + sourced: HighOrder/kern.cu:755-768 and 1185-1227 (patch
 * placement, Gaussian delta approximants), 2666-2683 (grid-point factors,
 * tilde-phi phase, turn-on window).  The particle-only Maple block is the
 * bilinear form sum_k C[k] DelR^(i_k) DelTH^(j_k). */
void orc_deposit_source(orc_solver *s, const orc_particle *pt, const double *c_re6, const double *c_im6,
                        double timer, double start) {
  const int N = s->N, M = s->M;
  memset(s->tred, 0, sizeof(double) * (size_t)N * M);
  memset(s->timd, 0, sizeof(double) * (size_t)N * M);
  const double a = s->p.a, mass = s->p.mass, mm = s->p.m;
  const double rp = pt->rp, tp = pt->tp;
  const double wt = s->p.wt_fac * s->dtheta;
  const double wp = s->p.wr_fac * s->dx;
  const double rpl = mass + sqrt(mass * mass - a * a);
  const double rm = mass - sqrt(mass * mass - a * a);
  const double wr = wp * (1.0 - rpl / rp);
  const double xp = rp + (rpl * rpl + a * a) / (rpl - rm) * log(rp / rpl - 1.0) -
                    (rm * rm + a * a) / (rpl - rm) * log(rp / rm - 1.0);
  const int ip = (int)((xp - s->p.Xmin) / s->dx);
  const int it = (int)(tp / s->dtheta);
  const double turn = pow(1.0 - exp(-(timer - start) / 25.0), 4);
  const double complex C[6] = {c_re6[0] + I * c_im6[0], c_re6[1] + I * c_im6[1], c_re6[2] + I * c_im6[2],
                               c_re6[3] + I * c_im6[3], c_re6[4] + I * c_im6[4], c_re6[5] + I * c_im6[5]};
  const double g0 = 1.0 / sqrt(2.0 * ORC_PIE);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < s->p.PTSY; j++) {
    const int row = j + it - s->p.PTSY / 2;
    if (!(row > 0 && row < M)) continue;
    const double th = s->theta[row];
    const double st = sin(th), ct = cos(th);
    const double dth = th - tp;
    const double T0 = g0 * exp(-dth * dth / (2.0 * wt * wt)) / wt;
    const double T1 = -dth / (wt * wt) * T0;
    const double T2 = (-1.0 / (wt * wt) + dth * dth / (wt * wt * wt * wt)) * T0;
    for (int k = 0; k < s->p.PTSX; k++) {
      const int col = k + ip - s->p.PTSX / 2;
      if (!(col > 0) || col >= N) continue;
      const double r = s->r_c[col];
      const double dr = r - rp;
      const double R0 = g0 * exp(-dr * dr / (2.0 * wr * wr)) / wr;
      const double R1 = -dr / (wr * wr) * R0;
      const double R2 = (-1.0 / (wr * wr) + dr * dr / (wr * wr * wr * wr)) * R0;
      const double complex t3364 =
          C[0] * R0 * T0 + C[1] * R0 * T1 + C[2] * R0 * T2 + C[3] * R1 * T0 + C[4] * R1 * T1 + C[5] * R2 * T0;
      const double delta = r * r + a * a - 2.0 * mass * r;
      const double cs2 = (r * r + a * a) * (r * r + a * a) - a * a * delta * st * st;
      const double complex rho = -1.0 / (r - a * I * ct);
      const double complex rho4 = rho * rho * rho * rho;
      double complex TT = (r * r + a * a * ct * ct) * t3364 / rho4;
      const double ph = -mm * a / (rpl - rm) * log((r - rpl) / (r - rm));
      TT = TT * (cos(ph) + I * sin(ph));
      TT = TT * turn;
      const size_t id = (size_t)N * row + col;
      s->tred[id] = 8.0 * ORC_PIE * delta * creal(TT) / cs2 / (r * r * r);
      s->timd[id] = 8.0 * ORC_PIE * delta * cimag(TT) / cs2 / (r * r * r);
    }
  }
}

/* Classical RK4 -- an option, not the reference's integrator: the textbook
 * form u + dt/6 (k1 + 2 k2 + 2 k3 + k4) with an accumulator, interior points
 * only, the closure applied to every stage state and to the result as the
 * reference does after each SSP-RK3 stage, the step's source held fixed. */
static void orc_step_rk4(orc_solver *s) {
  const int N = s->N, M = s->M;
  const double dt = s->p.dt;
  const double wk[4] = {dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0};  /* weights of k1..k4 */
  const double hk[3] = {0.5 * dt, 0.5 * dt, dt};                  /* y_{i+1} = u + h_i k_i */
  for (int f = 0; f < 4; f++)
    if (!s->acc[f]) s->acc[f] = zalloc((size_t)N * M);
  for (int st = 0; st < 4; st++) {
    orc_rhs(s, st == 0 ? s->u : s->uc);
#pragma omp parallel for schedule(static)
    for (int b = 3; b < M - 3; b++)
      for (int a = 3; a < N - 3; a++) {
        const size_t id = (size_t)N * b + a;
        for (int f = 0; f < 4; f++) {
          const double k = s->rhs[f][id];
          if (st == 0) s->acc[f][id] = s->u[f][id] + wk[0] * k;
          else if (st < 3) s->acc[f][id] += wk[st] * k;
          if (st < 3) s->uc[f][id] = s->u[f][id] + hk[st] * k;
          else s->u[f][id] = s->acc[f][id] + wk[3] * k;
        }
      }
    double *const *v = st < 3 ? s->uc : s->u;
    orc_bnd_poles(s, v);
    orc_bnd_ends(s, v);
  }
  orc_copy_ext(s);
}

void orc_set_integrator(orc_solver *s, int integrator) { s->integrator = integrator; }

/* kernel_rhs on a given state (four M x N planes, contiguous): the closure
 * is applied to a copy, the right-hand side (current source included) is
 * written for the interior points and zero elsewhere.  Uses the stage
 * arrays as scratch, so only between steps. */
void orc_eval_rhs(orc_solver *s, const double *in4, double *out4) {
  const size_t NM = (size_t)s->N * s->M;
  for (int f = 0; f < 4; f++) {
    memcpy(s->uc[f], in4 + f * NM, NM * sizeof(double));
    memset(s->rhs[f], 0, NM * sizeof(double));
  }
  orc_bnd_poles(s, s->uc);
  orc_bnd_ends(s, s->uc);
  orc_rhs(s, s->uc);
  for (int f = 0; f < 4; f++) memcpy(out4 + f * NM, s->rhs[f], NM * sizeof(double));
}

/* One full step as HighOrder/body.cu:131-165 sequences the kernels. */
void orc_step(orc_solver *s) {
  if (s->integrator == 1) {
    orc_step_rk4(s);
    return;
  }
  orc_rhs(s, s->u);
  orc_update(s, 1);
  orc_bnd_poles(s, s->uc);
  orc_bnd_ends(s, s->uc);
  orc_rhs(s, s->uc);
  orc_update(s, 2);
  orc_bnd_poles(s, s->uc);
  orc_bnd_ends(s, s->uc);
  orc_rhs(s, s->uc);
  orc_update(s, 3);
  orc_bnd_poles(s, s->u);
  orc_bnd_ends(s, s->u);
  orc_copy_ext(s);
}

void orc_get_ext(const orc_solver *s, double *re, double *im) {
  if (re) memcpy(re, s->ext_re, sizeof(double) * s->M);
  if (im) memcpy(im, s->ext_im, sizeof(double) * s->M);
}

/* ---------------------------------------------------------------------- */
/* swsh / fact / project: HighOrder/proj.c:4-75. */
static double orc_fact(double n) {
  double f = 1.0;
  for (double c = 1.0; c <= n; c++) f *= c;
  return f;
}

double orc_swsh(double ell, double ml, double the) {
  double acc = 0.0;
  const double c1 = (ml - 2.0) > 0 ? ml - 2.0 : 0.0;
  const double c2 = ((ell - 2.0) > (ell + ml)) ? ml + ell : ell - 2.0;
  for (double t = c1; t <= c2; t++) {
    double nrm = pow(-1.0, t) * sqrt(orc_fact(ell + ml) * orc_fact(ell - ml) * orc_fact(ell + 2.0) * orc_fact(ell - 2.0));
    nrm = nrm / (orc_fact(ell + ml - t) * orc_fact(ell - 2.0 - t) * orc_fact(t) * orc_fact(t + 2.0 - ml));
    acc += nrm * pow(cos(the / 2.0), 2.0 * ell + ml - 2.0 - 2.0 * t) * pow(sin(the / 2.0), 2.0 * t + 2.0 - ml);
  }
  return sqrt((2.0 * ell + 1.0) / 4.0 / ORC_PI_PARM) * acc;
}

/* Composite Boole rule over theta with 4 pi sin(theta) dtheta swsh weights;
 * qq[M] is set to qq[M-1] first as the reference does. */
double orc_project(double *qq, int M, double l, double m) {
  static const double w[5] = {7.0, 32.0, 12.0, 32.0, 7.0};
  const double dth = ORC_PI_PARM / M;
  double h = 0.0;
  qq[M] = qq[M - 1];
  for (int i = 0; i < M / 4; i++) {
    double th = 4.0 * dth * (double)i;
    for (int k = 0; k < 5; k++) {
      if (k) th += dth;
      h += w[k] * 4.0 * ORC_PI_PARM * qq[4 * i + k] * sin(th) * dth * orc_swsh(l, m, th);
    }
  }
  return 2.0 * h / 45.0;
}

/* ---------------------------------------------------------------------- */
/* body(): HighOrder/body.cu:56-215 for rank 0 of p=1.  The trajectory is an
 * in-memory copy of the .traj rows; a read past the last row leaves the
 * particle variables unchanged, as a failed fscanf does. */
int orc_run(orc_solver *s, const double *traj, int nrows, orc_coef_fn coef, int nsteps_limit, double *out_t,
            double *out_h, double *out_dedt, int max_rows, int *out_step, int ext_every, double *ext_re,
            double *ext_im, int max_ext, int *n_ext) {
  const int N = s->N, M = s->M;
  const double dt = s->p.dt, Xmax = s->p.Xmax, T = s->p.T;
  if (traj && !coef) return -1;
  double timer = (T - Xmax - 200.0) / 1 * 0;
  const double start = timer;
  const double endtime = (T - Xmax - 200.0) / 1 * (0 + 1) + Xmax + 200.0;
  int nt = (int)((endtime - start) / dt);
  if (nsteps_limit >= 0 && nsteps_limit < nt) nt = nsteps_limit;
  const int mabs = abs((int)s->p.m);

  double *iq_r = zalloc((size_t)M), *iq_i = zalloc((size_t)M);
  double *dq_r = zalloc((size_t)M + 1), *dq_i = zalloc((size_t)M + 1);
  double row[10] = {0};
  int cursor = 0;
#define ORC_READ()                                                  \
  do {                                                              \
    if (traj && cursor < nrows) {                                   \
      memcpy(row, traj + (size_t)10 * cursor, sizeof(row));        \
      cursor++;                                                     \
    }                                                               \
  } while (0)
  double rp = 0.0;
  double tmp11 = 0.0, tmp22 = 0.0, tmp33 = 0.0;
  if (traj) {
    ORC_READ();
    do { ORC_READ(); } while (row[0] < timer && cursor < nrows);
    rp = row[1];
  }
  int nrow_out = 0, next = 0;
  for (int k = 0; k < nt; k++) {
    if (traj) {
      const int c0 = cursor;
      ORC_READ();
      ORC_READ();
      if (cursor != c0) rp = row[1];
      rp = rp + 1e-6;
      orc_particle pt;
      memset(&pt, 0, sizeof(pt));
      pt.rp = rp; pt.tp = row[2]; pt.phip = row[6];
      pt.E = row[7]; pt.lz = row[8]; pt.Q = row[9];
      pt.drdt = row[3]; pt.d2rdt2 = (row[3] - tmp11) / dt; pt.d3rdt3 = 0.0;
      pt.dthdt = row[4]; pt.d2thdt2 = (row[4] - tmp22) / dt; pt.d3thdt3 = 0.0;
      pt.dphidt = row[5]; pt.d2phidt2 = (row[5] - tmp33) / dt;
      double cr[6], ci[6];
      coef(&pt, s->p.a, s->p.mass, s->p.m, cr, ci);
      orc_deposit_source(s, &pt, cr, ci, timer, start);
      tmp11 = row[3]; tmp22 = row[4]; tmp33 = row[5];
    } else {
      memset(s->tred, 0, sizeof(double) * (size_t)N * M);
      memset(s->timd, 0, sizeof(double) * (size_t)N * M);
    }
    orc_step(s);
    double dedt = 0.0;
    const double rr = s->r_c[N - 1];
    for (int q = 0; q < M; q++) {
      iq_r[q] = iq_r[q] + s->ext_re[q] * dt;
      iq_i[q] = iq_i[q] + s->ext_im[q] * dt;
      const double psi2 = iq_r[q] * iq_r[q] + iq_i[q] * iq_i[q];
      const double rho2 = rr * rr + pow(s->p.a * cos(s->theta[q]), 2);
      const double dvol = 0.5 * s->dtheta * sin(s->theta[q]) * rr * rr;
      dedt = dedt + psi2 * dvol * pow(rr, 6) / pow(rho2, 4);
      dq_r[q] = dq_r[q] + iq_r[q] * dt;
      dq_i[q] = dq_i[q] + iq_i[q] * dt;
    }
    if (ext_every > 0 && ext_re && (k % ext_every) == 0 && next < max_ext) {
      memcpy(ext_re + (size_t)next * M, s->ext_re, sizeof(double) * M);
      memcpy(ext_im + (size_t)next * M, s->ext_im, sizeof(double) * M);
      next++;
    }
    if (!(k % s->p.Fr) && (k * dt) >= s->p.out_start && nrow_out < max_rows) {
      for (int l = 0; l < 7; l++) {
        out_h[(size_t)nrow_out * 14 + 2 * l] = orc_project(dq_r, M, (double)(l + mabs), s->p.m);
        out_h[(size_t)nrow_out * 14 + 2 * l + 1] = -orc_project(dq_i, M, (double)(l + mabs), s->p.m);
      }
      out_t[nrow_out] = timer - Xmax;
      if (out_dedt) out_dedt[nrow_out] = dedt;
      if (out_step) out_step[nrow_out] = k;
      nrow_out++;
    }
    timer += dt;
  }
#undef ORC_READ
  if (n_ext) *n_ext = next;
  free(iq_r); free(iq_i); free(dq_r); free(dq_i);
  return nrow_out;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
