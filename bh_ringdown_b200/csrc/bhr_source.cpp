// bhr_source.cpp -- particle-only coefficients of the point-particle source.
//
// The reference evaluates a Maple-generated expression per grid point and
// per step (HighOrder/kern.cu:1229-2664).  That expression depends only on
// the particle's state; grid points enter through the Gaussian delta
// approximants alone, bilinearly.  This file evaluates the six complex
// coefficients of that bilinear form once per step, from this project's own
// derivation of the s=-2 Teukolsky source (gen_source.py, which documents
// the formula and conventions and writes bhr_source_gen.inc).
#include <cmath>
#include <complex>

#include "bhr.h"
#include "bhr_host.h"

namespace {

using cplx = std::complex<double>;
const cplx I_(0.0, 1.0);

template <class T>
inline T ipow(T b, int n) {
  const bool neg = n < 0;
  unsigned e = static_cast<unsigned>(neg ? -n : n);
  T r = T(1.0), p = b;
  while (e) {
    if (e & 1u) r *= p;
    p *= p;
    e >>= 1u;
  }
  return neg ? T(1.0) / r : r;
}

void eval_coefficients(double rp, double tp, double E, double lz, double drdt, double d2rdt2, double d3rdt3,
                       double dthdt, double d2thdt2, double d3thdt3, double dphidt, double d2phidt2, double a,
                       double mass, double m, double nmu, cplx *C) {
  using std::cos;
  using std::sin;
#include "bhr_source_gen.inc"
}

}  // namespace

extern "C" int bhr_source_coefficients(const bhr_particle *pt, double a, double mass, double m, double *c_re6,
                                       double *c_im6) {
  if (!pt || !c_re6 || !c_im6) {
    bhr::set_error("null argument");
    return BHR_INVALID_ARG;
  }
  const double rplus = mass + std::sqrt(mass * mass - a * a);
  if (!(pt->rp > rplus) || !(std::sin(pt->tp) != 0.0) || !std::isfinite(pt->rp) || !std::isfinite(pt->tp)) {
    bhr::set_error("particle must sit outside the horizon and off the poles");
    return BHR_INVALID_ARG;
  }
  cplx C[6];
  eval_coefficients(pt->rp, pt->tp, pt->E, pt->lz, pt->drdt, pt->d2rdt2, pt->d3rdt3, pt->dthdt, pt->d2thdt2,
                    pt->d3thdt3, pt->dphidt, pt->d2phidt2, a, mass, m, 1.0, C);
  // Mode factor of delta(phi - phip): exp(-i m phip) / (2 pi).
  const double ph = -m * pt->phip;
  const cplx mode = cplx(std::cos(ph), std::sin(ph)) / (2.0 * 3.141592653589793);
  for (int k = 0; k < 6; k++) {
    const cplx v = C[k] * mode;
    if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) {
      bhr::set_error("non-finite source coefficient");
      return BHR_NAN_DETECTED;
    }
    c_re6[k] = v.real();
    c_im6[k] = v.imag();
  }
  return BHR_OK;
}
