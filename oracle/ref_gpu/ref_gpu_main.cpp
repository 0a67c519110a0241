/*
 * ref_gpu_main.cpp -- runs the reference's own body() on a GPU for one
 * azimuthal mode.
 *
 * TEST INFRASTRUCTURE ONLY (oracle/).  oracle/build_ref.py compiles the
 * reference's HighOrder/body.cu and kern.cu unchanged with nvcc for sm_100a
 * (the grid and final time fixed at compile time by a generated parm.h, as
 * HighOrder/parm.h fixes them), main.c's grid() and proj.c's project()
 * with gcc, and links this driver in place of main()'s m loop
 * (HighOrder/main.c:50-55) into oracle/_ref/refgpu_<tag>.
 *
 *   refgpu_<tag> <workdir> <a> <m> <dt>
 *
 * body() opens ../Trajectories/a0.0_thi000_thf090.0_n.traj relative to
 * the working directory and writes its hm*.dat file there
 * (HighOrder/body.cu:63-78); the driver runs it in <workdir>/run.  Before
 * calling body() it checks every trajectory row against the one bound the
 * reference's source kernel does not check (the patch must end before
 * column N, HighOrder/kern.cu:1204-1206) and refuses to run otherwise.  The
 * radii grid() leaves NaN next to the horizon are floored at the next
 * double above r+, as the library and the oracle do.  Prints one JSON line
 * with the wall-clock seconds of the body() call.
 */
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>

#include "parm.h"

/* main.c (compiled as C++, as HighOrder/build.sh does) with its globals
 * renamed hmc_*: kern.cu's device scalars have the same names. */
extern double hmc_mass, hmc_aa, hmc_ss, hmc_dx, hmc_dtheta, hmc_dt;
extern double x_c[N], r_c[N], theta[M];
void grid(void);
void body(double *, double *, double, double, double, double, double, double, double, int, int);

static int check_trajectory(const std::string &path, double a, double dx) {
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) {
    std::fprintf(stderr, "cannot open %s\n", path.c_str());
    return 1;
  }
  const double rpl = 1.0 + std::sqrt(1.0 - a * a), rm = 1.0 - std::sqrt(1.0 - a * a);
  double v[10];
  long rows = 0;
  int worst = -1 << 30;
  while (std::fscanf(f, "%lf %lf %lf %lf %lf %lf %lf %lf %lf %lf", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6],
                     &v[7], &v[8], &v[9]) == 10) {
    const double rp = v[1];
    const double xp = rp + (rpl * rpl + a * a) / (rpl - rm) * std::log(rp / rpl - 1.0) -
                      (rm * rm + a * a) / (rpl - rm) * std::log(rp / rm - 1.0);
    const int ip = static_cast<int>((xp - Xmin) / dx);
    if (ip > worst) worst = ip;
    rows++;
  }
  std::fclose(f);
  // columns k + ip - PTSX/2 for k < PTSX must stay below N
  if (rows < 2 || worst + PTSX - 1 - PTSX / 2 >= N) {
    std::fprintf(stderr, "trajectory rejected: %ld rows, largest patch column %d (N = %d)\n", rows,
                 worst + PTSX - 1 - PTSX / 2, N);
    return 1;
  }
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s <workdir> <a> <m> <dt>\n", argv[0]);
    return 2;
  }
  const std::string work = argv[1];
  const double a = std::atof(argv[2]), mm = std::atof(argv[3]), dt = std::atof(argv[4]);
  if (!(dt > 0.0) || !(std::fabs(a) < 1.0)) {
    std::fprintf(stderr, "need dt > 0 and |a| < 1 (got a = %s, dt = %s)\n", argv[2], argv[4]);
    return 2;
  }
  hmc_mass = 1.0;
  hmc_aa = a;
  hmc_ss = -2.0;
  hmc_dx = (Xmax - Xmin) / N;
  hmc_dtheta = Pi / M;
  hmc_dt = dt;
  if (check_trajectory(work + "/Trajectories/a0.0_thi000_thf090.0_n.traj", a, hmc_dx)) return 3;
  grid();
  const double rpl = 1.0 + std::sqrt(1.0 - a * a);
  int floored = 0;
  for (int i = 0; i < N; i++)
    if (!(r_c[i] > rpl)) {
      r_c[i] = std::nextafter(rpl, 1e300);
      floored++;
    }
  const std::string run = work + "/run";
  if (chdir(run.c_str()) != 0) {
    std::fprintf(stderr, "cannot enter %s: %s\n", run.c_str(), std::strerror(errno));
    return 4;
  }
  const auto t0 = std::chrono::steady_clock::now();
  body(r_c, theta, hmc_dtheta, hmc_mass, a, -2.0, mm, hmc_dx, dt, 1, 0);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  const double endtime = (T - Xmax - 200.0) / 1 * (0 + 1) + Xmax + 200.0;  // HighOrder/body.cu:58-59
  const int nt = static_cast<int>((endtime - 0.0) / dt);
  std::fflush(stdout);
  std::printf("{\"N\": %d, \"M\": %d, \"T\": %.17g, \"dt\": %.17g, \"nt\": %d, \"seconds\": %.9g, \"floored\": %d}\n", N,
              M, static_cast<double>(T), dt, nt, secs, floored);
  return 0;
}
