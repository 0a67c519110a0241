// bhr_grid.cpp -- host set-up of a solve: grid, coefficient factor tables,
// spin-weighted harmonics, projection weights, initial data.
#include <cmath>
#include <cstring>

#include "bhr_host.h"
#include "bhr_internal.h"

namespace bhr {

namespace {
constexpr double kThirdH = 0.33333333333333333;  // HighOrder/kern.cu:46
}

// HighOrder/main.c:64-183.  x_c uniform on [Xmin, Xmax - dx]; theta_b =
// b*dtheta; x~ = x / Omega with the quartic hyperboloidal layer from
// rin = Xmin + 0.64 (Xmax - Xmin); r(x~) by Newton iteration on the Kerr
// tortoise coordinate, marching inwards from the outer point.  Where
// r - r+ falls below FP64 resolution the reference iteration returns NaN;
// from the first point whose step lands at or inside r+ onwards, r is set
// to the next double above r+.
void fill_grid(const bhr_params &p, double *x_c, double *r_c, double *theta, double *tx, double *r_plus,
               double *r_minus) {
  const double dx = (p.Xmax - p.Xmin) / p.N;
  const double dtheta = kPiParm / p.M;
  const double mass = p.mass, aa = p.a;
  for (int l = 0; l < p.N; l++) x_c[l] = p.Xmin + static_cast<double>(l) * dx;
  for (int b = 0; b < p.M; b++) theta[b] = static_cast<double>(b) * dtheta;
  const double rin = p.Xmin + (p.Xmax - p.Xmin) * 0.64;
  const double Rrpt = p.Xmax + 1e-6;
  for (int l = 0; l < p.N; l++) {
    const double x = x_c[l];
    const double om = (x < rin) ? 1.0 : 1.0 - std::pow((x - rin) / (Rrpt - rin), 4);
    tx[l] = x / om;
  }
  const double rp = mass + std::sqrt(mass * mass - aa * aa);
  const double rm = mass - std::sqrt(mass * mass - aa * aa);
  *r_plus = rp;
  *r_minus = rm;
  if (mass == 0.0) {
    for (int l = 0; l < p.N; l++) r_c[l] = tx[l];
    return;
  }
  const double tol = 1e-12;
  const double r_floor = std::nextafter(rp, INFINITY);
  bool floored = false;
  double r_old = tx[p.N - 1], r_new = r_old;
  for (int l = p.N - 1; l >= 0; l--) {
    if (floored) {
      r_c[l] = r_floor;
      continue;
    }
    double diff;
    do {
      const double drdx = (r_old * r_old + aa * aa - 2.0 * mass * r_old) / (r_old * r_old + aa * aa);
      double xo;
      if (mass == aa)
        xo = r_old + 2.0 * aa * std::log(r_old / aa - 1.0) - 2.0 * aa * aa / (r_old - aa);
      else if (aa == 0.0)
        xo = r_old + 2.0 * mass * std::log(r_old / (2.0 * mass) - 1.0);
      else
        xo = r_old + (rp * rp + aa * aa) / (rp - rm) * std::log(r_old / rp - 1.0) -
             (rm * rm + aa * aa) / (rp - rm) * std::log(r_old / rm - 1.0);
      r_new = r_old + (tx[l] - xo) * drdx;
      if (!(r_new > rp) || !std::isfinite(r_new)) {
        r_new = r_floor;
        floored = true;
        break;
      }
      diff = std::fabs(r_new - r_old) / r_old;
      r_old = r_new;
    } while (diff > tol);
    r_c[l] = r_new;
    r_old = r_new;
  }
}

Grid make_grid(const bhr_params &p) {
  Grid g;
  g.N = p.N;
  g.M = p.M;
  g.dx = (p.Xmax - p.Xmin) / p.N;
  g.dtheta = kPiParm / p.M;
  g.x_c.resize(p.N);
  g.r_c.resize(p.N);
  g.theta.resize(p.M);
  std::vector<double> tx(p.N);
  fill_grid(p, g.x_c.data(), g.r_c.data(), g.theta.data(), tx.data(), &g.r_plus, &g.r_minus);
  return g;
}

// Factor tables for the coefficients of HighOrder/kern.cu:113-158.  Every
// coefficient there is (per-column numerator + per-column numerator x
// per-row factor) / bir with bir = B0 + B1 sin^2(theta); the tables hold
// those numerators and the row factors.
void make_tables(const bhr_params &p, const Grid &g, std::vector<double> &coltab, std::vector<double> &rowtab) {
  coltab.assign(static_cast<size_t>(CF_COUNT) * p.N, 0.0);
  rowtab.assign(static_cast<size_t>(RF_COUNT) * p.M, 0.0);
  fill_tables(p, g.dx, g.r_c.data(), g.theta.data(), coltab.data(), rowtab.data());
}

void fill_tables(const bhr_params &p, double dx, const double *r_c, const double *theta, double *coltab,
                 double *rowtab) {
  const int N = p.N, M = p.M;
  for (size_t i = 0; i < static_cast<size_t>(RF_COUNT) * M; i++) rowtab[i] = 0.0;
  const double mass = p.mass, spin = p.a, em = p.m;
  const double rin = p.Xmin + (p.Xmax - p.Xmin) * 0.64;
  const double Rrpt = p.Xmax + 1e-6;
  const double a2 = spin * spin, a4 = a2 * a2;
  for (int j = 0; j < N; j++) {
    const double x = p.Xmin + static_cast<double>(j) * dx;
    double Om = 1.0, O1 = 0.0, O2 = 0.0;
    if (x >= rin) {
      const double L = Rrpt - rin, L4 = std::pow(L, 4);
      Om = 1.0 - std::pow((x - rin) / L, 4);
      O1 = -4.0 * std::pow(x - rin, 3) / L4;
      O2 = -12.0 * std::pow(x - rin, 2) / L4;
    }
    const double cL = Om - x * O1;
    const double eR = Om * r_c[j];
    const double eR2 = eR * eR, eR3 = eR2 * eR, eR5 = eR3 * eR2;
    const double Om2 = Om * Om, Om3 = Om2 * Om, Om4 = Om2 * Om2, Om5 = Om4 * Om;
    const double cL2 = cL * cL, cL3 = cL2 * cL;
    const double Sg = eR2 + Om2 * a2;
    const double Dt = eR2 - 2.0 * eR * mass * Om + Om2 * a2;
    const double xr_num =
        Om * (eR3 * (4.0 * cL2 * (eR - 3.0 * mass * Om) + 2.0 * cL * eR2 * O1 + eR2 * Om * O2 * x) +
              2.0 * eR *
                  (cL2 * Om2 * (5.0 * eR - 4.0 * mass * Om) - 3.0 * cL3 * (eR - 2.0 * mass * Om) +
                   2.0 * cL * eR2 * Om2 * O1 + eR2 * Om3 * O2 * x) *
                  a2 +
              (-6.0 * cL3 * Om2 + 6.0 * cL2 * Om4 + 2.0 * cL * eR * Om4 * O1 + eR * Om5 * O2 * x) * a4);
    const double h1 = 2.0 * Om * O1 - 2.0 * O1 * O1 * x + Om * O2 * x;
    const double yr_num =
        Om * (eR5 * h1 + 2.0 * eR3 * Om2 * h1 * a2 +
              Om4 * (6.0 * Om2 + 2.0 * O1 * O1 * x * (-eR + 3.0 * x) + Om * (2.0 * eR * O1 - 12.0 * O1 * x + eR * O2 * x)) *
                  a4 +
              2.0 * cL2 * eR * (2.0 * eR3 - 6.0 * eR2 * mass * Om + 5.0 * eR * Om2 * a2 - 4.0 * mass * Om3 * a2));
    double *c = coltab;
    c[CF_B0 * N + j] = -((2.0 * cL - Om2) * Sg * Sg) / cL2;
    c[CF_B1 * N + j] = a2 * Dt;
    c[CF_ATN * N + j] = (2.0 * (cL - Om2) * Sg * Sg) / cL2;
    c[CF_ARN * N + j] = -((Om2 * Sg * Sg) / cL2);
    c[CF_CCN * N + j] = -Dt;
    c[CF_XR * N + j] = -(xr_num / (cL3 * eR));
    c[CF_YR * N + j] = -(yr_num / (cL3 * eR));
    c[CF_CR0 * N + j] = Dt * (2.0 * eR2 + 6.0 * eR * mass * Om - 6.0 * Om2 * a2) / eR2;
    c[CF_DT * N + j] = Dt;
    c[CF_CR1 * N + j] = Dt;
    c[CF_BI0 * N + j] = 2.0 * spin * em * (-(Om2 * Sg) + cL * (eR2 + 2.0 * eR * mass * Om + Om2 * a2)) / cL;
    c[CF_BI1 * N + j] = -4.0 * spin * Dt;
    c[CF_BRI * N + j] = (-2.0 * em * Om2 * spin * Sg) / cL;
    c[CF_CIN * N + j] = (2.0 * em * Om * spin * (eR2 + 2.0 * eR * mass * Om - 3.0 * Om2 * a2)) / eR;
  }
  for (int b = 3; b < M - 3; b++) {
    const double y = theta[b];
    const double sn = std::sin(y);
    const double cot = 1.0 / std::tan(y), csc = 1.0 / std::sin(y);
    rowtab[RF_S2 * M + b] = sn * sn;
    rowtab[RF_COS * M + b] = std::cos(y);
    rowtab[RF_G * M + b] = 4.0 * cot * cot - 4.0 * em * cot * csc + em * em * csc * csc;
    rowtab[RF_CTAN * M + b] = std::tan(0.5 * kPiParm - y);
  }
}

// HighOrder/proj.c:8-35: explicit-sum s = -2 harmonic with factorials.
static double fact(double n) {
  double f = 1.0;
  for (double c = 1.0; c <= n; c++) f *= c;
  return f;
}

double swsh(double ell, double ml, double the) {
  double acc = 0.0;
  const double c1 = (ml - 2.0) > 0 ? ml - 2.0 : 0.0;
  const double c2 = ((ell - 2.0) > (ell + ml)) ? ml + ell : ell - 2.0;
  for (double t = c1; t <= c2; t++) {
    double nrm = std::pow(-1.0, t) * std::sqrt(fact(ell + ml) * fact(ell - ml) * fact(ell + 2.0) * fact(ell - 2.0));
    nrm /= fact(ell + ml - t) * fact(ell - 2.0 - t) * fact(t) * fact(t + 2.0 - ml);
    acc += nrm * std::pow(std::cos(the / 2.0), 2.0 * ell + ml - 2.0 - 2.0 * t) *
           std::pow(std::sin(the / 2.0), 2.0 * t + 2.0 - ml);
  }
  return std::sqrt((2.0 * ell + 1.0) / 4.0 / kPiParm) * acc;
}

// Boole weights (7, 32, 12, 32, 7) per panel of four intervals, theta
// accumulated by += dtheta as HighOrder/proj.c:47-72 does; the sample at
// index M aliases M-1 (HighOrder/proj.c:45).  The final 2/45 is folded in.
void make_projection_weights(const bhr_params &p, const Grid &g, std::vector<double> &w7) {
  const int M = p.M;
  w7.assign(static_cast<size_t>(7) * M, 0.0);
  static const double wk[5] = {7.0, 32.0, 12.0, 32.0, 7.0};
  const int mabs = std::abs(static_cast<int>(p.m));
  const double dth = kPiParm / M;
  for (int l = 0; l < 7; l++) {
    const double ell = static_cast<double>(l + mabs);
    for (int i = 0; i < M / 4; i++) {
      double th = 4.0 * dth * static_cast<double>(i);
      for (int k = 0; k < 5; k++) {
        if (k) th += dth;
        int idx = 4 * i + k;
        if (idx == M) idx = M - 1;
        w7[static_cast<size_t>(l) * M + idx] +=
            wk[k] * 4.0 * kPiParm * std::sin(th) * dth * swsh(ell, p.m, th) * (2.0 / 45.0);
      }
    }
  }
}

void make_dedt_weights(const bhr_params &p, const Grid &g, std::vector<double> &e) {
  e.assign(p.M, 0.0);
  const double rr = g.r_c[p.N - 1];
  for (int b = 0; b < p.M; b++) {
    const double rho2 = rr * rr + std::pow(p.a * std::cos(g.theta[b]), 2);
    const double dvol = 0.5 * g.dtheta * std::sin(g.theta[b]) * rr * rr;
    e[b] = dvol * std::pow(rr, 6) / std::pow(rho2, 4);
  }
}

void apply_closure_host(double *planes, int N, int M, bool even_m, int nplanes) {
  const size_t NM = static_cast<size_t>(N) * M;
  for (int f = 0; f < nplanes; f++) {
    double *P = planes + f * NM;
    for (int a = 3; a < N - 3; a++) {
      auto at = [&](int b) -> double & { return P[static_cast<size_t>(b) * N + a]; };
      if (even_m) {
        at(2) = (4.0 * at(3) - at(4)) * kThirdH;
        at(1) = (4.0 * at(2) - at(3)) * kThirdH;
        at(M - 3) = (4.0 * at(M - 4) - at(M - 5)) * kThirdH;
        at(M - 2) = (4.0 * at(M - 3) - at(M - 4)) * kThirdH;
        at(0) = (4.0 * at(1) - at(2)) * kThirdH;
        at(M - 1) = (4.0 * at(M - 2) - at(M - 3)) * kThirdH;
      } else {
        at(0) = at(M - 1) = at(1) = at(2) = at(M - 2) = at(M - 3) = 0.0;
      }
    }
    for (int b = 0; b < M; b++) {
      double *row = P + static_cast<size_t>(b) * N;
      row[2] = (4.0 * row[3] - row[4]) * kThirdH;
      row[N - 3] = (4.0 * row[N - 4] - row[N - 5]) * kThirdH;
      row[1] = (4.0 * row[2] - row[3]) * kThirdH;
      row[N - 2] = (4.0 * row[N - 3] - row[N - 4]) * kThirdH;
      row[0] = (4.0 * row[1] - row[2]) * kThirdH;
      row[N - 1] = (4.0 * row[N - 2] - row[N - 3]) * kThirdH;
    }
  }
}

// Initial data: zero (HighOrder/kern.cu:164-167) or the Gaussian pulse
// psi = exp(-(x-c)^2/(2w^2)) swsh(l, m, theta), Pi = 0, closed by the
// boundary extrapolation so every stored state satisfies the closure.
void make_initial_factors(const bhr_params &p, const Grid &g, std::vector<double> &fa, std::vector<double> &gb) {
  fa.clear();
  gb.clear();
  if (p.init_kind != BHR_INIT_GAUSSIAN) return;
  fa.resize(p.N);
  gb.resize(p.M);
  for (int a = 0; a < p.N; a++) {
    const double x = g.x_c[a] - p.init_center;
    fa[a] = std::exp(-x * x / (2.0 * p.init_width * p.init_width));
  }
  for (int b = 0; b < p.M; b++) gb[b] = swsh(p.init_ell, p.m, g.theta[b]);
}

}  // namespace bhr
