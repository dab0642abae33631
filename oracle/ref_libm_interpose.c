/* ref_libm_interpose.c -- TEST INFRASTRUCTURE (oracle).
 *
 * Linked into the *strict* build of the reference renderer only.  It defines
 * the libm entry points the reference's hot path calls (knds_metric.hpp,
 * geodesic.hpp, camera.hpp, ray_bundle.hpp, main.cpp:329-434, 1306-1866) with
 * hidden visibility, so inside that shared object the reference's own code
 * binds to the renderer's deterministic libm (ktmath.h) instead of glibc's.
 * The reference source is not modified: this is symbol interposition at link
 * time.  Nothing outside the strict oracle library sees these symbols. */
#include <complex.h>

#include "../kerrtracecpp2_b200/csrc/ktmath.h"

#define KT_HIDDEN __attribute__((visibility("hidden")))

KT_HIDDEN double sin(double x) { return ktm_sin(x); }
KT_HIDDEN double cos(double x) { return ktm_cos(x); }
KT_HIDDEN double pow(double x, double y) { return ktm_pow(x, y); }
KT_HIDDEN double exp(double x) { return ktm_exp(x); }
KT_HIDDEN double log(double x) { return ktm_log(x); }
KT_HIDDEN double log10(double x) { return ktm_log10(x); }
KT_HIDDEN double cbrt(double x) { return ktm_cbrt(x); }
KT_HIDDEN double atan2(double y, double x) { return ktm_atan2(y, x); }
KT_HIDDEN double acos(double x) { return ktm_acos(x); }
/* the elliptic-closed solver (main.cpp:705-1301): std::asin, std::atan and
 * std::abs of a std::complex<double> (cabs) */
KT_HIDDEN double asin(double x) { return ktm_asin(x); }
KT_HIDDEN double atan(double x) { return ktm_atan(x); }
KT_HIDDEN double hypot(double x, double y) { return ktm_hypot(x, y); }
KT_HIDDEN double cabs(double complex z) { return ktm_hypot(creal(z), cimag(z)); }
