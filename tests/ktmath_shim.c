/* Test shim: exports ktmath.h's functions with C linkage so the CPU tests can
 * check their accuracy against mpmath and their agreement with the device
 * build.  Built by tests/conftest.py with -ffp-contract=off. */
#include "../kerrtracecpp2_b200/csrc/ktmath.h"

double kts_sin(double x) { return ktm_sin(x); }
double kts_cos(double x) { return ktm_cos(x); }
double kts_exp(double x) { return ktm_exp(x); }
double kts_log(double x) { return ktm_log(x); }
double kts_log10(double x) { return ktm_log10(x); }
double kts_pow(double x, double y) { return ktm_pow(x, y); }
double kts_cbrt(double x) { return ktm_cbrt(x); }
double kts_atan2(double y, double x) { return ktm_atan2(y, x); }
double kts_acos(double x) { return ktm_acos(x); }
double kts_atan(double x) { return ktm_atan(x); }
double kts_asin(double x) { return ktm_asin(x); }
double kts_hypot(double x, double y) { return ktm_hypot(x, y); }
void kts_div3_n(const double* x, double* q, long n) {
  for (long i = 0; i < n; ++i) q[i] = ktm_div3(x[i]);
}
