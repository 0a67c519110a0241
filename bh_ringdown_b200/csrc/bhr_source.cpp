// bhr_source.cpp -- particle-only coefficients of the point-particle source.
#include "bhr.h"
#include "bhr_host.h"

extern "C" int bhr_source_coefficients(const bhr_particle *pt, double a, double mass, double m, double *c_re6,
                                       double *c_im6) {
  (void)pt; (void)a; (void)mass; (void)m; (void)c_re6; (void)c_im6;
  bhr::set_error("particle source coefficients are not built into this library yet");
  return BHR_INVALID_ARG;
}
