// bhr_host.h -- host-side pieces of the solver shared between translation
// units: grid, coefficient factor tables, harmonics, trajectory cursor.
#pragma once

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "bhr.h"

namespace bhr {

// An NVTX range around a host API call (visible in Nsight timelines; a
// no-op when no tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

constexpr double kPiParm = 3.14159265358979;  // HighOrder/parm.h:12

struct Grid {
  int N = 0, M = 0;
  double dx = 0, dtheta = 0, r_plus = 0, r_minus = 0;
  std::vector<double> x_c, r_c, theta;
};

// Grid of HighOrder/main.c:64-183, with a horizon floor where the Newton
// iteration would step to r <= r+ (see grid.cpp).
Grid make_grid(const bhr_params &p);
// The same, into caller arrays (x_c, r_c, tx of N; theta of M); no allocation.
void fill_grid(const bhr_params &p, double *x_c, double *r_c, double *theta, double *tx, double *r_plus,
               double *r_minus);
// Per-column and per-row coefficient factors (layouts of bhr_internal.h).
void make_tables(const bhr_params &p, const Grid &g, std::vector<double> &coltab, std::vector<double> &rowtab);
// The same, into caller arrays (CF_COUNT*N and RF_COUNT*M); no allocation.
void fill_tables(const bhr_params &p, double dx, const double *r_c, const double *theta, double *coltab,
                 double *rowtab);
// Spin-weighted harmonic s=-2 (HighOrder/proj.c:16-35).
double swsh(double ell, double ml, double the);
// Boole-rule projection weights: h_l = sum_b W[l*M + b] * q[b] for
// l = |m| + 0..6 (HighOrder/proj.c:37-75, HighOrder/body.cu:189-202).
void make_projection_weights(const bhr_params &p, const Grid &g, std::vector<double> &w7);
// Weights of dE/dt = sum_b |int psi|^2 * E[b] (HighOrder/body.cu:174-184).
void make_dedt_weights(const bhr_params &p, const Grid &g, std::vector<double> &e);
// Gaussian initial data psi = exp(-(x-c)^2/(2 w^2)) swsh(l, m, theta) is
// separable: the radial factors fa[N] and angular factors gb[M] (both empty
// for zero data); the device forms the interior products (q_im, p_re and
// p_im start at zero; the closure is rebuilt by every reader).
void make_initial_factors(const bhr_params &p, const Grid &g, std::vector<double> &fa, std::vector<double> &gb);
// Reference closure (kernel_boundary2a then 2b) applied on nplanes host planes.
void apply_closure_host(double *planes, int N, int M, bool even_m, int nplanes = 4);

void set_error(const std::string &msg);

}  // namespace bhr
