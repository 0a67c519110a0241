/*
 * ref_driver.cpp -- runs the reference's own HighOrder kernels on CPU cores.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/).  oracle/build_ref.py compiles this
 * file together with the reference's kern.cu (included below through a
 * symlink, with a grid header chosen at build time) plus main.c and proj.c,
 * into oracle/_ref/libref_<tag>.so.  Tests use it to pin the C oracle
 * (oracle/teuk_oracle.c) against the reference itself, and to make the
 * golden fixtures under tests/golden/.
 *
 * The launch configurations follow HighOrder/body.cu:41-51 and the kernel
 * order of one time step follows HighOrder/body.cu:108-165.  The loop over
 * blocks runs under OpenMP; the kernels touch no shared memory.
 */
#include "kern.cu"

#include <cstring>
#include <omp.h>

thread_local emu_dim3 blockIdx;
thread_local emu_dim3 threadIdx;
thread_local emu_dim3 blockDim;

extern "C" {
/* main.c and proj.c are compiled separately; main.c's globals are renamed
 * with an hmc_ prefix at compile time so they do not collide with kern.cu's
 * device scalars of the same names. */
extern double hmc_mass, hmc_aa, hmc_dx, hmc_dtheta;
extern double x_c[N], r_c[N], theta[M];
void grid(void);
double project(double *, double, double);
double swsh(double, double, double);
void hmc_body(double *, double *, double, double, double, double, double, double, double, int, int) {}
}

template <class F>
static void emu_launch(unsigned gx, unsigned gy, unsigned bx, unsigned by, F f, bool parallel = true) {
  const long nblk = (long)gx * (long)gy;
#pragma omp parallel for schedule(static) if (parallel)
  for (long i = 0; i < nblk; i++) {
    blockDim = {bx, by, 1};
    blockIdx = {(unsigned)(i % gx), (unsigned)(i / gx), 0};
    for (unsigned ty = 0; ty < by; ty++)
      for (unsigned tx = 0; tx < bx; tx++) {
        threadIdx = {tx, ty, 0};
        f();
      }
  }
}

static double h_theta[M], h_rc[N];

extern "C" {

int ref_N(void) { return N; }
int ref_M(void) { return M; }
int ref_PTSX(void) { return PTSX; }
int ref_PTSY(void) { return PTSY; }
double ref_Xmin(void) { return Xmin; }
double ref_Xmax(void) { return Xmax; }
void ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

/* main.c grid() with the given mass and spin (main.c:55-63). */
void ref_grid(double mass_in, double aa_in, double *xo, double *ro, double *to) {
  hmc_mass = mass_in;
  hmc_aa = aa_in;
  hmc_dx = (Xmax - Xmin) / N;
  hmc_dtheta = Pi / M;
  grid();
  if (xo) std::memcpy(xo, x_c, sizeof(double) * N);
  if (ro) std::memcpy(ro, r_c, sizeof(double) * N);
  if (to) std::memcpy(to, theta, sizeof(double) * M);
}

/* kernel_init launch of body.cu:53-54 (run serially: every thread of the
 * reference kernel writes the same device scalars). */
void ref_init(double mass_in, double aa_in, double mm_in, double dt_in, const double *th, const double *rc) {
  std::memcpy(h_theta, th, sizeof(h_theta));
  std::memcpy(h_rc, rc, sizeof(h_rc));
  const double dx_in = (Xmax - Xmin) / N, dth_in = Pi / M;
  emu_launch(N / 32, M / 8, 32, 8,
             [&] { kernel_init(dth_in, mass_in, aa_in, -2.0, mm_in, dx_in, dt_in, h_theta, h_rc); }, false);
}

static double *field(int f) {
  switch (f) {
    case 0: return qre;
    case 1: return qim;
    case 2: return pre;
    default: return pim;
  }
}

void ref_set_state(const double *a, const double *b, const double *c, const double *d) {
  const double *in[4] = {a, b, c, d};
  for (int f = 0; f < 4; f++) std::memcpy(field(f), in[f], sizeof(double) * N * M);
}

void ref_get_state(double *a, double *b, double *c, double *d) {
  double *out[4] = {a, b, c, d};
  for (int f = 0; f < 4; f++)
    if (out[f]) std::memcpy(out[f], field(f), sizeof(double) * N * M);
}

void ref_get_coeff(int k, double *out) {
  double *planes[9] = {bb_c, cc_c, ee_c, a_re_c, a_im_c, d_re_c, d_im_c, v_re_c, v_im_c};
  if (k >= 0 && k < 9) std::memcpy(out, planes[k], sizeof(double) * N * M);
}

void ref_set_source(const double *tre, const double *tim) {
  std::memcpy(&tred[0][0], tre, sizeof(double) * N * M);
  std::memcpy(&timd[0][0], tim, sizeof(double) * N * M);
}

void ref_get_source(double *tre, double *tim) {
  std::memcpy(tre, &tred[0][0], sizeof(double) * N * M);
  std::memcpy(tim, &timd[0][0], sizeof(double) * N * M);
}

/* reset_sourced + sourced as body.cu:108 and 122-124 launch them. */
void ref_source(double start, double timer, double rp, double phip, double tp, double E, double lz, double Q,
                double drdt, double d2rdt2, double d3rdt3, double dthdt, double d2thdt2, double d3thdt3,
                double dphidt, double d2phidt2) {
  emu_launch(N / 32, M / 8, 32, 8, [] { reset_sourced(); });
  emu_launch(PTSX / 8, PTSY / 8, 8, 8, [&] {
    sourced(h_theta, start, timer, rp, phip, tp, E, lz, Q, drdt, d2rdt2, d3rdt3, dthdt, d2thdt2, d3thdt3, dphidt,
            d2phidt2, h_rc);
  });
}

/* One time step: the kernel sequence of body.cu:131-165. */
void ref_step(double *ext_re, double *ext_im) {
  static double bre[M], bim[M];
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_rhs1(h_theta, h_rc); });
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_update1(); });
  emu_launch(N / 32, 1, 32, 1, [] { kernel_boundary1a(); });
  emu_launch(M / 8, 1, 8, 1, [] { kernel_boundary1b(); });
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_rhs2(h_theta, h_rc); });
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_update2(); });
  emu_launch(N / 32, 1, 32, 1, [] { kernel_boundary1a(); });
  emu_launch(M / 8, 1, 8, 1, [] { kernel_boundary1b(); });
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_rhs2(h_theta, h_rc); });
  emu_launch(N / 32, M / 8, 32, 8, [] { kernel_update3(); });
  emu_launch(N / 32, 1, 32, 1, [] { kernel_boundary2a(); });
  emu_launch(M / 8, 1, 8, 1, [] { kernel_boundary2b(bre, bim); });
  if (ext_re) std::memcpy(ext_re, bre, sizeof(bre));
  if (ext_im) std::memcpy(ext_im, bim, sizeof(bim));
}

/* kernel_boundary2a + 2b alone, used to close initial data. */
void ref_apply_closure(void) {
  static double bre[M], bim[M];
  emu_launch(N / 32, 1, 32, 1, [] { kernel_boundary2a(); });
  emu_launch(M / 8, 1, 8, 1, [] { kernel_boundary2b(bre, bim); });
}

double ref_project(double *qq, double l, double m) { return project(qq, l, m); }
double ref_swsh(double l, double m, double th) { return swsh(l, m, th); }

}  // extern "C"
