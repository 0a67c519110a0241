/* body_bhr.c -- body() on top of libbhr.so, in place of body.cu and kern.cu; build as build.sh does:
 *   g++ -O -c main.c proj.c body_bhr.c -I<repo>/include
 *   g++ -o run main.o proj.o body_bhr.o -L<repo>/bh_ringdown_b200 -lbhr -lm */
#include <stdio.h>
#include "bhr.h" /* before parm.h: its macros N, M, Xmin, ... share names with bhr_params fields */
#include "parm.h"

/* parm.h's grid constants, read before their macros are undefined so that
 * the bhr_params fields of the same names can be assigned below. */
static const int kN = N, kM = M, kFr = Fr, kPTSX = PTSX, kPTSY = PTSY;
static const double kXmin = Xmin, kXmax = Xmax, kT = T;
#undef N
#undef M
#undef Xmin
#undef Xmax
#undef T
#undef Fr
#undef PTSX
#undef PTSY

void body(double *r_c, double *theta, double dtheta, double mass, double aa,
          double ss, double mm, double dx, double dt, int p, int my_rank) {
  (void)r_c; (void)theta; (void)dtheta; (void)ss; (void)dx; (void)p;
  bhr_params prm;
  bhr_params_default(&prm);
  prm.N = kN; prm.M = kM; prm.Xmin = kXmin; prm.Xmax = kXmax;   /* parm.h */
  prm.T = kT; prm.Fr = kFr; prm.PTSX = kPTSX; prm.PTSY = kPTSY;
  prm.out_start = kXmax + 200.0;                                /* body.cu:207 */
  prm.mass = mass; prm.a = aa; prm.m = mm; prm.dt = dt;
  prm.device = my_rank % 2;                                     /* body.cu:30 */
  bhr_solver *s = NULL;
  if (bhr_solver_create(&prm, &s) != BHR_OK ||
      bhr_solver_load_trajectory(s, "../Trajectories/a0.0_thi000_thf090.0_n.traj") != BHR_OK ||
      bhr_solver_run(s, ".", "a0.0_thi000_thf090.0_n") != BHR_OK) {
    fprintf(stderr, "bhr: %s\n", bhr_last_error_string());
  }
  bhr_solver_destroy(s);
}
