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

/* ktm_div_rcp against the division on n pseudo-random (a, b) pairs
 * (xorshift64*, seed): mode 0 uniform exponents over the guarded range and
 * beyond (|x| in [2^-300, 2^300), either sign, zeros and powers of two
 * mixed in), mode 1 the renderer's range (mantissas uniform, |x| in
 * [2^-40, 2^60)).  Returns the number of quotients whose bits differ. */
static uint64_t kts_next(uint64_t* s) {
  *s ^= *s >> 12;
  *s ^= *s << 25;
  *s ^= *s >> 27;
  return *s * 2685821657736338717ULL;
}
static double kts_draw(uint64_t* s, int lo, int hi) {
  const uint64_t u = kts_next(s);
  const uint64_t man = u & 0xfffffffffffffULL;
  const int span = hi - lo;
  const int ex = lo + (int)((kts_next(s) >> 11) % (uint64_t)span);
  uint64_t bits = ((uint64_t)(ex + 1023) << 52) | man;
  if ((u >> 52) & 1) bits |= 0x8000000000000000ULL;
  if (((u >> 53) & 63) == 0) bits &= 0xfff0000000000000ULL;  /* a power of two */
  double x;
  memcpy(&x, &bits, 8);
  if (((u >> 59) & 31) == 0 && lo < 0) x = 0.0;
  return x;
}
long kts_div_rcp_check(uint64_t seed, long n, int mode) {
  uint64_t s = seed | 1;
  long bad = 0;
  const int lo = mode == 0 ? -300 : -40, hi = mode == 0 ? 300 : 60;
  for (long i = 0; i < n; ++i) {
    const double a = kts_draw(&s, lo, hi), b = kts_draw(&s, lo, hi);
    if (b == 0.0) continue;
    const double q = ktm_div_rcp(a, b, ktm_rcp(b));
    const double w = a / b;
    uint64_t qb, wb;
    memcpy(&qb, &q, 8);
    memcpy(&wb, &w, 8);
    bad += (qb != wb) && !(q != q && w != w);
  }
  return bad;
}
