/* TEST INFRASTRUCTURE: exposes plibm's exp/pow and the system libm's for the
 * accuracy tests (tests/test_plibm.py). */
#include <math.h>
#include <stdint.h>
#include "../../openifs_b200/csrc/plibm.h"

static double ulp_diff(double a, double b) {
  if (a == b) return 0.0;
  if (!(a == a) || !(b == b)) return 1e300;
  return fabs(a - b) / (nextafter(fabs(b), INFINITY) - fabs(b));
}
/* mode 0: exp(x[i]); mode 1: pow(x[i], y[i]).  Writes plibm and libm results
 * and returns the largest ulp distance between them. */
double plibm_check(int mode, const double *x, const double *y, long n, double *out_p, double *out_l) {
  double worst = 0.0;
  for (long i = 0; i < n; ++i) {
    double a = mode == 0 ? plibm_exp(x[i]) : plibm_pow(x[i], y[i]);
    double b = mode == 0 ? exp(x[i]) : pow(x[i], y[i]);
    if (out_p) out_p[i] = a;
    if (out_l) out_l[i] = b;
    double d = ulp_diff(a, b);
    if (d > worst) worst = d;
  }
  return worst;
}
