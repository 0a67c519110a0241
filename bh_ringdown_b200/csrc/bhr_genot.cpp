// bhr_genot.cpp -- the trajectory generator, restated from GenOT (host C++,
// no device work).  Two steps, each a C-ABI entry point:
//   bhr_genot_mino  the adiabatic inspiral (tabulated), the generalised
//                   Ori-Thorne transition and the geodesic plunge, sampled
//                   in Mino time (GenOT/ParamWLMino.cc:5-531)
//   bhr_genot_bl    that worldline integrated in Boyer-Lindquist time into
//                   the .traj rows the solver reads (GenOT/WL_BL.cc:7-380)
// Units G = c = M = 1.  theta_inc and theta_f in degrees, theta and phi in
// radians, as in the reference's inputs and outputs.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bhr.h"
#include "bhr_host.h"

using bhr::set_error;

namespace {

constexpr double kDeg = M_PI / 180.0;

// Natural cubic spline through (x[k], y[k]), k = 0..n-1, x increasing.  The
// second derivatives m[k] solve the continuity system
//   h[k-1] m[k-1] + 2 (h[k-1] + h[k]) m[k] + h[k] m[k+1] = 6 (d[k] - d[k-1]),
// d[k] = (y[k+1] - y[k]) / h[k], with m[0] = m[n-1] = 0 (Thomas algorithm).
// On the interval [x[k], x[k+1]], with A = (x[k+1] - t)/h, B = (t - x[k])/h:
//   y(t)  = A y[k] + B y[k+1] + ((A^3 - A) m[k] + (B^3 - B) m[k+1]) h^2 / 6
//   y'(t) = (y[k+1] - y[k]) / h + ((3 B^2 - 1) m[k+1] - (3 A^2 - 1) m[k]) h / 6
// The interval is found by bisection over the knots [lo, n-1] (t outside
// them takes the end interval's cubic), as the reference's look-up does.
class Spline {
 public:
  Spline() = default;
  Spline(const double *x, const double *y, int n, int stride) : x_(n), y_(n), m_(n, 0.0) {
    for (int k = 0; k < n; k++) {
      x_[k] = x[static_cast<size_t>(k) * stride];
      y_[k] = y[static_cast<size_t>(k) * stride];
    }
    if (n < 3) return;
    std::vector<double> cp(n, 0.0), dp(n, 0.0);
    for (int k = 1; k <= n - 2; k++) {
      const double hl = x_[k] - x_[k - 1], hr = x_[k + 1] - x_[k];
      const double rhs = 6.0 * ((y_[k + 1] - y_[k]) / hr - (y_[k] - y_[k - 1]) / hl);
      const double den = 2.0 * (hl + hr) - (k > 1 ? hl * cp[k - 1] : 0.0);
      cp[k] = hr / den;
      dp[k] = (rhs - (k > 1 ? hl * dp[k - 1] : 0.0)) / den;
    }
    m_[n - 2] = dp[n - 2];
    for (int k = n - 3; k >= 1; k--) m_[k] = dp[k] - cp[k] * m_[k + 1];
  }
  int size() const { return static_cast<int>(x_.size()); }
  double x(int k) const { return x_[k]; }
  double y(int k) const { return y_[k]; }
  // Value at t; search over knots [lo, n-1].
  double value(double t, int lo = 0) const {
    const int k = bracket(t, lo);
    const double h = x_[k + 1] - x_[k];
    const double A = (x_[k + 1] - t) / h, B = (t - x_[k]) / h;
    return A * y_[k] + B * y_[k + 1] + ((A * A * A - A) * m_[k] + (B * B * B - B) * m_[k + 1]) * (h * h) / 6.0;
  }
  // First derivative at t; search over knots [lo, n-1].
  double deriv(double t, int lo = 0) const {
    const int k = bracket(t, lo);
    const double h = x_[k + 1] - x_[k];
    const double A = (x_[k + 1] - t) / h, B = (t - x_[k]) / h;
    return (y_[k + 1] - y_[k]) / h + ((3.0 * B * B - 1.0) * m_[k + 1] - (3.0 * A * A - 1.0) * m_[k]) * h / 6.0;
  }

 private:
  int bracket(double t, int lo) const {
    int hi = size() - 1;
    while (hi - lo > 1) {
      const int mid = (hi + lo) >> 1;
      if (x_[mid] > t) hi = mid;
      else lo = mid;
    }
    return lo;
  }
  std::vector<double> x_, y_, m_;
};

// Kerr radial potential R(r) = [E (r^2 + a^2) - a L]^2 - Delta [r^2 + (L - a E)^2 + Q]
// and the derivatives of it the transition and the plunge use.
double delta(double r, double a) { return r * r - 2.0 * r + a * a; }
// dR/dr
double dR_dr(double r, double a, double E, double L, double Q) {
  const double lme = L - a * E, r2a2 = r * r + a * a;
  return -2.0 * r * (r2a2 - 2.0 * r) - 2.0 * (r - 1.0) * (r * r + Q + lme * lme) + 4.0 * E * r * (E * r2a2 - a * L);
}

// theta_inc (degrees) of a geodesic with E, L, Q: from the turning point
// z_- = cos(theta_min)^2 of the polar potential (GenOT/ParamWLMino.cc:606-621).
double theta_inc(double a, double E, double L, double Q) {
  const double A = a * a * (1.0 - E * E);
  const double B = -L * L - Q - A;
  const double qq = -0.5 * (B - std::sqrt(B * B - 4.0 * A * Q));
  const double thm = std::acos(std::sqrt(Q / qq)) * 180.0 / M_PI;
  return L > 0.0 ? 90.0 - thm : 90.0 + thm;
}

// The adiabatic inspiral: splines in Mino time of r, theta_inc, E, L, Q and
// of dE/dlambda, dL/dlambda, dQ/dlambda (GenOT/ParamWLMino.cc:5-195).  The
// table holds Mino time and fluxes with the mass ratio eta scaled out;
// Mino time is put back as l = (l~ - l~0)/eta + l~0.
struct Inspiral {
  std::vector<double> l;
  Spline r, thi, E, L, Q, dE, dL, dQ;
  double l0 = 0, l1 = 0;
  int last = 0;
  std::vector<double> col(const double *rows, int n, int c, double sign = 1.0) const {
    std::vector<double> v(n);
    for (int i = 0; i < n; i++) v[i] = sign * rows[static_cast<size_t>(i) * 11 + c];
    return v;
  }
  Inspiral(const double *rows, int n, double eta) : l(n) {
    for (int i = 0; i < n; i++) {
      const double lt = rows[static_cast<size_t>(i) * 11 + 1];
      l[i] = i == 0 ? lt : (lt - l[0]) / eta + l[0];
    }
    auto mk = [&](int c, double sign) {
      const std::vector<double> v = col(rows, n, c, sign);
      return Spline(l.data(), v.data(), n, 1);
    };
    r = mk(2, 1.0);
    thi = mk(4, 1.0);
    E = mk(5, 1.0);
    L = mk(6, 1.0);
    Q = mk(7, 1.0);
    dE = mk(8, -1.0);  // the table holds the fluxes, -dE/dl~
    dL = mk(9, -1.0);
    dQ = mk(10, -1.0);
    l0 = l[0];
    l1 = l[n - 1];
    last = n - 1;
  }
  bool in_range(double lam) const { return lam >= l0 && lam <= l1; }
  // lambda at which r(lambda) = rr, by bisection to relative width 1e-14
  // (r decreases along the inspiral).
  double lambda_at(double rr) const {
    double lo = l0, hi = l1;
    for (int it = 0; it < 400 && std::fabs(2.0 * (hi - lo) / (hi + lo)) > 1e-14; it++) {
      const double mid = 0.5 * (hi + lo);
      if (r.value(mid) < rr) hi = mid;
      else lo = mid;
    }
    return 0.5 * (lo + hi);
  }
};

// The generalised Ori-Thorne transition (GenOT/ParamWLMino.cc:197-300).
// With A = -R'''/4 and B = -(1/2) sum_C (d^2 R/dC dr) dC/dlambda at the LSO
// (C = E, L, Q; fluxes per eta-scaled Mino time), r - r_lso obeys
// d^2 R/dl^2 = -A R^2 - eta B l, whose scaled form d^2 X/dT^2 = -X^2 - T is
// the universal table X(T): l = T (eta A B)^(-1/5),
// r = r_lso + X (eta B)^(2/5) A^(-3/5).  E, L, Q run from their LSO values
// with slope eta dC/dl, plus corrections that join them to the inspiral at
// l_Ti with matching value and slope: model 1 adds a constant and a
// quadratic term, model 2 a quadratic and a cubic one.
struct Transition {
  Spline X;
  double a = 0, eta = 0, A = 0, B = 0;
  double s = 0, s_inv = 0;  // (eta A B)^(1/5) and (eta A B)^(-1/5)
  double r_lso = 0, C_lso[3] = {0, 0, 0}, dC_lso[3] = {0, 0, 0};
  int model = 2;
  double c0[3] = {0, 0, 0}, c2[3] = {0, 0, 0}, c3[3] = {0, 0, 0};

  double r_of(double l) const { return r_lso + X.value(l * s) * std::pow(eta * B, 0.4) * std::pow(A, -0.6); }
  // dr/dl; the table look-up of the derivative starts its search at knot 1
  // (GenOT/ParamWLMino.cc:565-589).
  double drdl_of(double l) const { return X.deriv(l * s, 1) * std::pow(eta * B, 0.6) * std::pow(A, -0.4); }
  // E, L or Q (c = 0, 1, 2) at l
  double C_of(int c, double l) const {
    if (model == 1) return c0[c] + C_lso[c] + l * (eta * dC_lso[c] + l * 0.5 * c2[c]);
    return C_lso[c] + l * (eta * dC_lso[c] + l * (0.5 * c2[c] + (l / 6.0) * c3[c]));
  }
  // Join to the inspiral's value CI and slope dCI (per eta-scaled Mino time) at lTi.
  void join(int c, double lTi, double CI, double dCI) {
    const double C = C_lso[c], dC = dC_lso[c];
    if (model == 1) {
      c2[c] = eta * (dCI - dC) / lTi;
      c0[c] = 0.5 * (2.0 * (CI - C) - lTi * eta * (dC + dCI));
    } else {
      c2[c] = -2.0 * (3.0 * C - 3.0 * CI + (2.0 * dC + dCI) * eta * lTi) / (lTi * lTi);
      c3[c] = 6.0 * (2.0 * C - 2.0 * CI + (dC + dCI) * eta * lTi) / (lTi * lTi * lTi);
    }
  }
};

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

// Column c of n rows of `width` doubles strictly increases (the splines'
// knots; the reference stops on a repeated knot).
bool increasing(const double *rows, int n, int width, int c) {
  for (int i = 1; i < n; i++)
    if (!(rows[static_cast<size_t>(i) * width + c] > rows[static_cast<size_t>(i - 1) * width + c])) return false;
  return true;
}

// The three BL-time derivatives of the worldline with respect to Mino time
// (GenOT/WL_BL.cc:340-380): dt/dlambda, dphi/dt and dchi/dlambda, where
// cos(theta) = sin(theta_inc) cos(chi).
double dt_dl(double a, double r, double th, double E, double L) {
  const double r2a2 = r * r + a * a, st = std::sin(th), dl = delta(r, a);
  return E * (r2a2 * r2a2 / dl - a * a * st * st) - 2.0 * a * r * L / dl;
}
double dphi_dt(double a, double r, double th, double E, double L) {
  const double st = std::sin(th), dl = delta(r, a);
  const double num = a * (2.0 * E * r - a * L) + L * dl / (st * st);
  const double den = a * a * a * a * E - 2.0 * a * L * r + 2.0 * a * a * E * r * r + E * r * r * r * r -
                     a * a * E * dl * st * st;
  return num / den;
}
double dchi_dl(double a, double chi, double thi, double E, double L, double Q) {
  const double A = a * a * (1.0 - E * E);
  const double B = -L * L - Q - A;
  const double zm = std::sin(thi * kDeg);
  const double zsq = zm * zm * std::cos(chi) * std::cos(chi);
  const double bzp = 0.5 * (-B + std::sqrt(B * B - 4.0 * A * Q));
  return std::sqrt(bzp - A * zsq);
}

}  // namespace

extern "C" {

int bhr_genot_mino(const bhr_genot_params *p, const double *insp, int n_insp, const double *ot, int n_ot,
                   double *out, int max_rows, int *n_out, double *transition) {
  if (n_out) *n_out = 0;
  if (!p || !insp || !ot || !n_out || n_insp < 4 || n_ot < 4)
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: null argument or too few table rows");
  if (p->model != 1 && p->model != 2) return fail(BHR_INVALID_ARG, "bhr_genot_mino: model must be 1 or 2");
  if (!(p->eta > 0.0) || !(p->dl > 0.0) || !(std::fabs(p->a) < 1.0))
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: need eta > 0, dl > 0, |a| < 1");
  if (!increasing(insp, n_insp, 11, 1) || !increasing(ot, n_ot, 2, 0))
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: Mino time of the inspiral table and T of the Ori-Thorne table "
                                 "must increase");
  const double a = p->a, eta = p->eta;
  const Inspiral I(insp, n_insp, eta);
  // LSO: the inspiral table's last row
  const int e = I.last;
  Transition T;
  T.X = Spline(ot, ot + 1, n_ot, 2);
  T.a = a;
  T.eta = eta;
  T.model = p->model;
  T.r_lso = I.r.y(e);
  const double E = I.E.y(e), Lz = I.L.y(e), Q = I.Q.y(e), r = T.r_lso;
  T.C_lso[0] = E;
  T.C_lso[1] = Lz;
  T.C_lso[2] = Q;
  T.dC_lso[0] = I.dE.y(e);
  T.dC_lso[1] = I.dL.y(e);
  T.dC_lso[2] = I.dQ.y(e);
  // R''' and the mixed derivatives d^2 R / dC dr at the LSO
  const double R3 = 12.0 + 24.0 * (E * E - 1.0) * r;
  const double RE = -4.0 * a * Lz + 8.0 * E * r * r * r + 4.0 * a * a * E * (1.0 + r);
  const double RL = -4.0 * (a * E + Lz * (r - 1.0));
  const double RQ = 2.0 * (1.0 - r);
  T.A = -0.25 * R3;
  T.B = -0.5 * (RE * T.dC_lso[0] + RL * T.dC_lso[1] + RQ * T.dC_lso[2]);
  if (!(T.A > 0.0) || !(T.B > 0.0))
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: A = -R'''/4 and B at the LSO must be positive");
  T.s = std::pow(eta * T.A * T.B, 0.2);
  T.s_inv = std::pow(eta * T.A * T.B, -0.2);
  const double lTi = p->LTi * T.s_inv;
  if (p->LTf > ot[static_cast<size_t>(n_ot - 1) * 2])
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: LTf is beyond the transition table");
  const double lTf = p->LTf * T.s_inv;
  // Match the inspiral to the transition where r = r_trans(lTi); inspiral
  // Mino time then runs on the transition's origin (l = 0 near its middle).
  const double rTi = T.r_of(lTi);
  const double off = I.lambda_at(rTi) - lTi;
  if (!I.in_range(lTi + off))
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: the transition start is outside the inspiral table");
  const Spline *IC[3] = {&I.E, &I.L, &I.Q};
  const Spline *ID[3] = {&I.dE, &I.dL, &I.dQ};
  for (int c = 0; c < 3; c++) T.join(c, lTi, IC[c]->value(lTi + off), ID[c]->value(lTi + off));
  const double Ep = T.C_of(0, lTf), Lp = T.C_of(1, lTf), Qp = T.C_of(2, lTf);  // the plunge's constants
  if (transition) {
    transition[0] = lTi;
    transition[1] = lTf;
    transition[2] = rTi;
    transition[3] = T.r_of(lTf);
  }
  if (I.r.y(0) < p->r_start)
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: r_start is outside the inspiral table");
  const double lstart = I.lambda_at(p->r_start) - off;
  const double lend = lTf + 100.0, dl = p->dl, r_stop = 1.0 + std::sqrt((1.0 - a) * (1.0 + a)) - 0.5;
  if (!((lend - lstart) / dl < 2e8))
    return fail(BHR_INVALID_ARG, "bhr_genot_mino: more than 2e8 rows (eta too small or dl too fine)");
  double rh = 0, vh = 0, thih = 0, eh = 0, lh = 0, qh = 0;
  bool in_trans = false;
  int n = 0;
  for (double l = lstart; l <= lend; l += dl) {
    if (l < lTi) {
      const double li = l + off;
      if (!I.in_range(li)) return fail(BHR_INVALID_ARG, "bhr_genot_mino: Mino time outside the inspiral table");
      rh = I.r.value(li);
      thih = I.thi.value(li);
      eh = I.E.value(li);
      lh = I.L.value(li);
      qh = I.Q.value(li);
    } else if (l > lTi && l < lTf) {
      rh = T.r_of(l);
      vh = T.drdl_of(l);
      eh = T.C_of(0, l);
      lh = T.C_of(1, l);
      qh = T.C_of(2, l);
      thih = theta_inc(a, eh, lh, qh);
      in_trans = true;
    } else {
      // plunge: one classical RK4 step of r'' = R'(r)/2 with the
      // constants at lTf, from the previous sample (E, L, Q and theta_inc
      // stay at their last transition values in the rows)
      if (!in_trans) return fail(BHR_INVALID_ARG, "bhr_genot_mino: the plunge must follow a transition sample");
      auto acc = [&](double rr) { return 0.5 * dR_dr(rr, a, Ep, Lp, Qp); };
      const double dr1 = vh * dl, dv1 = acc(rh) * dl;
      const double dr2 = (vh + 0.5 * dv1) * dl, dv2 = acc(rh + 0.5 * dr1) * dl;
      const double dr3 = (vh + 0.5 * dv2) * dl, dv3 = acc(rh + 0.5 * dr2) * dl;
      const double dr4 = (vh + dv3) * dl, dv4 = acc(rh + dr3) * dl;
      rh += dr1 / 6.0 + dr2 / 3.0 + dr3 / 3.0 + dr4 / 6.0;
      vh += dv1 / 6.0 + dv2 / 3.0 + dv3 / 3.0 + dv4 / 6.0;
    }
    if (out) {
      if (n >= max_rows) {
        *n_out = n + 1;
        return fail(BHR_INVALID_ARG, "bhr_genot_mino: more rows than max_rows");
      }
      double *o = out + static_cast<size_t>(n) * 6;
      o[0] = l;
      o[1] = rh;
      o[2] = thih;
      o[3] = eh;
      o[4] = lh;
      o[5] = qh;
    }
    n++;
    if (rh < r_stop) break;
  }
  *n_out = n;
  return BHR_OK;
}

int bhr_genot_bl(const bhr_genot_bl_params *p, const double *mino, int n_mino, int stride, double *out, int max_rows,
                 int *n_out, double *thf_deg, int *thdot_pos, const char *path) {
  if (n_out) *n_out = 0;
  if (!p || !mino || !n_out || n_mino < 4 || stride < 1)
    return fail(BHR_INVALID_ARG, "bhr_genot_bl: null argument, too few rows or stride < 1");
  if (!(p->dt > 0.0) || !(std::fabs(p->a) < 1.0)) return fail(BHR_INVALID_ARG, "bhr_genot_bl: need dt > 0, |a| < 1");
  if (!increasing(mino + 6, n_mino - 1, 6, 0))
    return fail(BHR_INVALID_ARG, "bhr_genot_bl: the worldline's Mino time must increase");
  if (!(p->t_stop / p->dt < 2e8)) return fail(BHR_INVALID_ARG, "bhr_genot_bl: more than 2e8 rows");
  // rows of BL time: t = 0, dt, 2 dt, ... (accumulated) while t <= t_stop
  int nrows = 0;
  for (double t = 0.0; t <= p->t_stop; t += p->dt) nrows++;
  const int nkeep = (nrows + stride - 1) / stride;
  if (!out && !path && !thf_deg) {  // count only
    *n_out = nkeep;
    return BHR_OK;
  }
  if (out && nkeep > max_rows) {
    *n_out = nkeep;
    return fail(BHR_INVALID_ARG, "bhr_genot_bl: more rows than max_rows");
  }
  FILE *f = nullptr;
  if (path) {
    f = std::fopen(path, "w");
    if (!f) return fail(BHR_IO_ERROR, std::string("bhr_genot_bl: cannot open ") + path);
  }
  // The worldline's splines are over rows 1..n-1 (the reference's look-ups
  // start at its second row; GenOT/WL_BL.cc:55-60).
  const double *m1 = mino + 6;
  const int n = n_mino - 1;
  const Spline R(m1, m1 + 1, n, 6), TI(m1, m1 + 2, n, 6), SE(m1, m1 + 3, n, 6), SL(m1, m1 + 4, n, 6),
      SQ(m1, m1 + 5, n, 6);
  const double a = p->a, dt = p->dt;
  double l = p->lambda_start, chi = p->chi0_deg * kDeg, phi = p->phi0_deg * kDeg;
  double thh = 0.0, dthdl = 0.0;
  int row = 0, kept = 0;
  // the increments over dt of (lambda, chi, phi) from the rates at Mino
  // time ll and phase cc: dt / (dt/dlambda), dt (dchi/dlambda) / (dt/dlambda), dt dphi/dt
  auto step = [&](double ll, double cc, double &kl, double &kc, double &kp) {
    const double rr = R.value(ll), ti = TI.value(ll), e = SE.value(ll), lz = SL.value(ll), q = SQ.value(ll);
    const double th = std::acos(std::sin(ti * kDeg) * std::cos(cc));
    const double tl = dt_dl(a, rr, th, e, lz);
    kl = dt / tl;
    kc = dt * dchi_dl(a, cc, ti, e, lz, q) / tl;
    kp = dt * dphi_dt(a, rr, th, e, lz);
  };
  for (double t = 0.0; t <= p->t_stop; t += dt, row++) {
    // the worldline here
    const double rh = R.value(l), drdl = R.deriv(l), ti = TI.value(l);
    const double ch = std::sin(ti * kDeg) * std::cos(chi);
    thh = std::acos(ch);
    const double eh = SE.value(l), lh = SL.value(l), qh = SQ.value(l);
    const double tl = dt_dl(a, rh, thh, eh, lh);
    const double cl = dchi_dl(a, chi, ti, eh, lh, qh);
    const double ph = dphi_dt(a, rh, thh, eh, lh);
    dthdl = std::sin(ti * kDeg) * std::sin(chi) * cl / std::sqrt(1.0 - ch * ch);
    const double v[10] = {t, rh, thh, drdl / tl, dthdl / tl, ph, phi, eh, lh, qh};
    if (f)
      std::fprintf(f, "%.12e %.12e %.12e %.12e %.12e %.12e %.12e %.12e %.12e %.12e\n", v[0], v[1], v[2], v[3], v[4],
                   v[5], v[6], v[7], v[8], v[9]);
    if (out && row % stride == 0) std::memcpy(out + static_cast<size_t>(kept++) * 10, v, sizeof(v));
    // classical RK4 in t for (lambda, chi, phi)
    const double k1l = dt / tl, k1c = dt * cl / tl, k1p = dt * ph;
    double k2l, k2c, k2p, k3l, k3c, k3p, k4l, k4c, k4p;
    step(l + 0.5 * k1l, chi + 0.5 * k1c, k2l, k2c, k2p);
    step(l + 0.5 * k2l, chi + 0.5 * k2c, k3l, k3c, k3p);
    step(l + k3l, chi + k3c, k4l, k4c, k4p);
    l += k1l / 6.0 + k2l / 3.0 + k3l / 3.0 + k4l / 6.0;
    chi += k1c / 6.0 + k2c / 3.0 + k3c / 3.0 + k4c / 6.0;
    phi += k1p / 6.0 + k2p / 3.0 + k3p / 3.0 + k4p / 6.0;
  }
  if (f && std::fclose(f) != 0) return fail(BHR_IO_ERROR, std::string("bhr_genot_bl: writing ") + path + " failed");
  *n_out = out ? kept : nkeep;
  if (thf_deg) *thf_deg = thh / kDeg;
  if (thdot_pos) *thdot_pos = dthdl > 0.0 ? 1 : 0;
  return BHR_OK;
}

int bhr_genot_ot_table(double T0, double dT, int rows, double T_start, double *X) {
  if (!X || rows < 1 || !(dT > 0.0) || !(T_start < 0.0) || !(T_start <= T0))
    return fail(BHR_INVALID_ARG, "bhr_genot_ot_table: need rows >= 1, dT > 0 and T_start <= T0, T_start < 0");
  // X'' = -X^2 - T as (X, V); start on the asymptotic series
  // X = u^(1/2) + u^(-2)/8 - (49/128) u^(-9/2), u = -T (order by order in u^(-5/2))
  const double u = -T_start;
  double y[2] = {std::sqrt(u) + 0.125 / (u * u) - 49.0 / 128.0 * std::pow(u, -4.5),
                 -(0.5 / std::sqrt(u) - 0.25 / (u * u * u) + 49.0 / 128.0 * 4.5 * std::pow(u, -5.5))};
  auto rk4 = [](double t, const double *y0, double h, double *y1) {
    auto f = [](double tt, const double *yy, double *d) {
      d[0] = yy[1];
      d[1] = -yy[0] * yy[0] - tt;
    };
    double k1[2], k2[2], k3[2], k4[2], w[2];
    f(t, y0, k1);
    for (int i = 0; i < 2; i++) w[i] = y0[i] + 0.5 * h * k1[i];
    f(t + 0.5 * h, w, k2);
    for (int i = 0; i < 2; i++) w[i] = y0[i] + 0.5 * h * k2[i];
    f(t + 0.5 * h, w, k3);
    for (int i = 0; i < 2; i++) w[i] = y0[i] + h * k3[i];
    f(t + h, w, k4);
    for (int i = 0; i < 2; i++) y1[i] = y0[i] + h / 6.0 * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
  };
  // Adaptive classical RK4 with step doubling (a step against two half
  // steps, their difference / 15 as the error, the Richardson-extrapolated
  // result kept), landing exactly on each table point.
  const double rtol = 1e-13, atol = 1e-13;
  double t = T_start, h = 1e-3;
  long long steps = 0;
  for (int k = 0; k < rows; k++) {
    const double target = T0 + dT * k;
    while (t < target) {
      if (++steps > 200000000LL) return fail(BHR_INVALID_ARG, "bhr_genot_ot_table: step limit (blow-up?)");
      const double hh = std::min(h, target - t);
      double y1[2], yh[2], y2[2];
      rk4(t, y, hh, y1);
      rk4(t, y, 0.5 * hh, yh);
      rk4(t + 0.5 * hh, yh, 0.5 * hh, y2);
      double err = 0.0;
      for (int i = 0; i < 2; i++) err = std::max(err, std::fabs(y2[i] - y1[i]) / 15.0 / (atol + rtol * std::fabs(y2[i])));
      if (!std::isfinite(err)) return fail(BHR_INVALID_ARG, "bhr_genot_ot_table: the solution is not finite there");
      if (err <= 1.0) {
        for (int i = 0; i < 2; i++) y[i] = y2[i] + (y2[i] - y1[i]) / 15.0;
        t = (hh == target - t) ? target : t + hh;
        h = hh * std::min(4.0, 0.9 * std::pow(std::max(err, 1e-10), -0.2));
      } else {
        h = hh * std::max(0.1, 0.9 * std::pow(err, -0.25));
      }
    }
    X[k] = y[0];
  }
  return BHR_OK;
}

int bhr_genot_traj_name(double a, double thi0_deg, double thf_deg, int thdot_pos, char *buf, int buflen) {
  if (!buf || buflen < 1) return fail(BHR_INVALID_ARG, "bhr_genot_traj_name: no buffer");
  // a, theta_inc of the first row (truncated) with zeros to three digits,
  // theta_f with one decimal and zeros to five characters, chosen by the
  // value before rounding; "p" or "n" for the sign of dtheta/dlambda at the
  // end (GenOT/WL_BL.cc:101-153)
  const int thi = static_cast<int>(thi0_deg);
  const char *tz = thi < 10 ? "00" : thi < 100 ? "0" : "";
  const char *fz = thf_deg < 10 ? "00" : thf_deg < 100 ? "0" : "";
  const int w = thf_deg < 10 ? 2 : thf_deg < 100 ? 3 : 4;
  const int k = std::snprintf(buf, static_cast<size_t>(buflen), "a%2.1f_thi%s%d_thf%s%*.1f_%s.traj", a, tz, thi, fz, w,
                              thf_deg, thdot_pos ? "p" : "n");
  if (k < 0 || k >= buflen) return fail(BHR_INVALID_ARG, "bhr_genot_traj_name: buffer too small");
  return BHR_OK;
}

}  // extern "C"
