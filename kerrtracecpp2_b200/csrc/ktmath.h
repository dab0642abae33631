/*
 * ktmath.h -- the renderer's own deterministic binary64 math library.
 *
 * Why it exists: the geodesic right-hand side differentiates the Hamiltonian
 * by central finite differences (relative step 1e-5..1e-6), which amplifies a
 * one-ulp difference in sin/cos/pow by ~1e5, and the accept/reject step
 * controller turns that into a different step sequence.  Results that agree
 * to 1e-9 between the CPU reference and the GPU are therefore only possible
 * when both evaluate *bit-identical* transcendentals.  CUDA's and glibc's
 * libm differ in the last bit, so this header provides one implementation,
 * compiled from the same source for the host (gcc, -ffp-contract=off) and the
 * device (nvcc, --fmad=false), and interposed into the strict build of the
 * reference (its calls to sin, cos, pow, exp, log, log10, cbrt, atan2, acos
 * resolve to these).
 *
 * Methods (all published, coefficients generated by gen_ktmath_consts.py):
 *   sin/cos : Cody-Waite reduction by pi/2 with a three-part split, the
 *             reduced argument kept as a double-double, Taylor polynomials
 *             on |r| <= pi/4 (Horner, fma).
 *   exp     : reduction by ln 2 (32-bit high part), Taylor polynomial on
 *             |r| <= ln2/2, exact scaling by 2^k built from bits.
 *   log     : x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *             s = (m-1)/(m+1) carried as a double-double, series in s^2.
 *   pow     : exp(y * log|x|) with log and the product kept in
 *             double-double, C99 Annex F special cases.
 *   cbrt    : Newton iteration on [1,8) with a double-double final residual.
 *   atan2   : octant folding, table of atan(i/8) in double-double and the
 *             addition formula atan z = atan c + atan((z-c)/(1+zc)), series.
 *   acos    : 2 atan2(sqrt(1-x), sqrt(1+x)).
 * Accuracy (tests/test_ktmath.py checks it against mpmath): sin, cos, exp,
 * log, log10, pow, cbrt <= 1 ulp; atan2 <= 2 ulp; acos <= 2 ulp on the
 * sampled domains.  sin/cos are accurate for |x| < 2^26 and deterministic
 * (but not accurate) beyond.
 *
 * Every function uses only +, -, *, /, sqrt, fma, rint, fabs, floor, fmod
 * and bit manipulation, each of which is correctly rounded (or exact) on both
 * x86-64 (SSE2/FMA) and sm_100a, so host and device results are identical.
 */
#ifndef KTMATH_H
#define KTMATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>
#include "ktmath_consts.h"

#if defined(__CUDACC__)
#define KTM_FN static __host__ __device__ inline
#else
#define KTM_FN static inline
#endif

KTM_FN uint64_t ktm_bits(double x) {
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
}
KTM_FN double ktm_from_bits(uint64_t u) {
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
}
KTM_FN double ktm_inf(void) { return ktm_from_bits(0x7ff0000000000000ULL); }
KTM_FN double ktm_nan(void) { return ktm_from_bits(0x7ff8000000000000ULL); }
KTM_FN int ktm_isnan(double x) { return x != x; }
KTM_FN int ktm_isinf(double x) { return fabs(x) == ktm_inf(); }

/* 2^n for n in [-1022, 1023], exact. */
KTM_FN double ktm_pow2i(int n) { return ktm_from_bits((uint64_t)(n + 1023) << 52); }

/* x * 2^n for any n in [-2100, 2100]; one IEEE rounding at most (subnormals). */
KTM_FN double ktm_scale(double x, int n) {
  if (n > 1023) {
    x *= ktm_pow2i(1023);
    n -= 1023;
    if (n > 1023) n = 1023;
    return x * ktm_pow2i(n);
  }
  if (n < -1022) {
    x *= ktm_pow2i(-1022 + 54);
    n += 1022 - 54;
    if (n < -1022) {
      x *= ktm_pow2i(-1022);
      n += 1022;
      if (n < -1022) n = -1022;
    }
    return x * ktm_pow2i(n);
  }
  return x * ktm_pow2i(n);
}

/* ---------------------------------------------------------------- sin/cos */

/* Reduced-argument kernels for r = rh + rl, |rh| <= pi/4 (+ a few ulp),
 * |rl| <= ulp(rh): sin(rh+rl) ~ sin(rh) + rl cos(rh), cos ~ cos(rh) - rl sin(rh). */
KTM_FN double ktm_sin_kernel(double rh, double rl) {
  const double c[9] = KTM_SIN_COEFFS;
  const double z = rh * rh;
  double p = c[8];
  p = fma(p, z, c[7]);
  p = fma(p, z, c[6]);
  p = fma(p, z, c[5]);
  p = fma(p, z, c[4]);
  p = fma(p, z, c[3]);
  p = fma(p, z, c[2]);
  p = fma(p, z, c[1]);
  p = fma(p, z, c[0]);
  return rh + fma(rh * z, p, fma(-0.5 * z, rl, rl));
}

KTM_FN double ktm_cos_kernel(double rh, double rl) {
  const double c[9] = KTM_COS_COEFFS;
  const double z = rh * rh;
  const double zlo = fma(rh, rh, -z);
  double p = c[8];
  p = fma(p, z, c[7]);
  p = fma(p, z, c[6]);
  p = fma(p, z, c[5]);
  p = fma(p, z, c[4]);
  p = fma(p, z, c[3]);
  p = fma(p, z, c[2]);
  p = fma(p, z, c[1]);
  p = fma(p, z, c[0]);
  const double hz = 0.5 * z;
  const double w = 1.0 - hz;
  const double tail = fma(z * z, p, fma(-rh, rl, ((1.0 - w) - hz) - 0.5 * zlo));
  return w + tail;
}

/* Reduce x by pi/2: returns r = *rh + *rl with |r| <= pi/4 (approximately)
 * and the quadrant in *q (0..3).  Inf/NaN give NaN. */
KTM_FN void ktm_rem_pio2(double x, double* rh, double* rl, int* q) {
  const double ax = fabs(x);
  if (!(ax <= 0x1p26)) {
    if (ktm_isnan(x) || ktm_isinf(x)) {
      *q = 0;
      *rh = x - x;
      *rl = 0.0;
      return;
    }
    /* Deterministic coarse reduction for huge arguments (not accurate). */
    x = fmod(x, 4.0 * KTM_PIO2_1);
  }
  if (fabs(x) < KTM_PIO4_HI) {
    *q = 0;
    *rh = x;
    *rl = 0.0;
    return;
  }
  const double k = rint(x * KTM_2_OVER_PI);
  const double r1 = fma(-k, KTM_PIO2_1, x);  /* exact for |x| <= 2^26 */
  const double t = k * KTM_PIO2_2;
  const double tl = fma(k, KTM_PIO2_2, -t);
  const double h = r1 - t;
  const double l = (((r1 - h) - t) - tl) - k * KTM_PIO2_3;
  const double hh = h + l;
  *rh = hh;
  *rl = (h - hh) + l;
  *q = (int)((int64_t)k & 3);
}

KTM_FN void ktm_sincos(double x, double* s, double* c) {
  if (fabs(x) < 0x1p-27) {
    *s = x;
    *c = 1.0;
    return;
  }
  int q;
  double rh, rl;
  ktm_rem_pio2(x, &rh, &rl, &q);
  const double sr = ktm_sin_kernel(rh, rl);
  const double cr = ktm_cos_kernel(rh, rl);
  switch (q) {
    case 0: *s = sr;  *c = cr;  break;
    case 1: *s = cr;  *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
  }
}

KTM_FN double ktm_sin(double x) {
  double s, c;
  ktm_sincos(x, &s, &c);
  return s;
}

KTM_FN double ktm_cos(double x) {
  double s, c;
  ktm_sincos(x, &s, &c);
  return c;
}

/* ------------------------------------------------------------- x / 3 */

/* x / b for a small odd constant b, the correctly rounded IEEE quotient, in
 * three operations instead of a division (ktm_div3: the metric's Lambda/3
 * terms).  Method: one correction step of P. Markstein (IBM J. Res. Dev.
 * 34(1), 1990) applied to q0 = RN(x y), y = RN(1/b), for which
 * |1 - b y| = 2^-54 (b = 3; it is 2^-56 for b = 15):
 *   |x y - x/b| = (x/b) |1 - b y| < ulp(x/b)/2, so |q0 - x/b| < ulp(x/b);
 *   r = x - b q0 is then a small multiple of ulp(q0), exact in one fma;
 *   q0 + r y = x/b + (1 - b y)(q0 - x/b) is within 2^-54 ulp of x/b,
 * while x/b in units of its ulp is an integer over the odd b, at least
 * 1/(2b) ulp from any rounding midpoint; so RN(q0 + r y) = RN(x/b).  Zero,
 * subnormal, near-overflow, Inf and NaN arguments take the division. */
KTM_FN double ktm_div_odd(double x, double b, double y) {
  const uint32_t e = (uint32_t)(ktm_bits(x) >> 52) & 0x7ffu;
  if (e - 64u >= 1936u) return x / b;
  const double q0 = x * y;
  return fma(fma(-b, q0, x), y, q0);
}
KTM_FN double ktm_div3(double x) { return ktm_div_odd(x, 3.0, 0x1.5555555555555p-2); }


/* -------------------------------------------------------------------- exp */

/* exp(hi + lo) where |lo| <= ulp(hi). */
KTM_FN double ktm_exp_dd(double hi, double lo) {
  if (ktm_isnan(hi)) return hi;
  if (hi > 709.8) return ktm_inf();
  if (hi < -745.2) return 0.0;
  const double c[13] = KTM_EXP_COEFFS;
  const double k = rint(hi * KTM_INV_LN2);
  double r = fma(-k, KTM_LN2_HI, hi);
  r = fma(-k, KTM_LN2_LO, r);
  r = r + lo;
  double p = c[12];
  p = fma(p, r, c[11]);
  p = fma(p, r, c[10]);
  p = fma(p, r, c[9]);
  p = fma(p, r, c[8]);
  p = fma(p, r, c[7]);
  p = fma(p, r, c[6]);
  p = fma(p, r, c[5]);
  p = fma(p, r, c[4]);
  p = fma(p, r, c[3]);
  p = fma(p, r, c[2]);
  p = fma(p, r, c[1]);
  p = fma(p, r, c[0]);
  const double e = 1.0 + fma(r * r, p, r);
  return ktm_scale(e, (int)k);
}

KTM_FN double ktm_exp(double x) { return ktm_exp_dd(x, 0.0); }

/* -------------------------------------------------------------------- log */

/* log(x) as a double-double for finite x > 0. */
KTM_FN void ktm_log_dd(double x, double* out_hi, double* out_lo) {
  const double lc[12] = KTM_LOG_COEFFS;
  int e = 0;
  if (x < 0x1p-1022) {
    x *= 0x1p54;
    e = -54;
  }
  uint64_t u = ktm_bits(x);
  e += (int)((u >> 52) & 0x7ff) - 1023;
  u = (u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m = ktm_from_bits(u);
  if (m > 2.0 * KTM_SQRT2_OVER_2) {
    m *= 0.5;
    e += 1;
  }
  const double f = m - 1.0;                 /* exact (Sterbenz) */
  const double den = 2.0 + f;
  const double den_lo = (2.0 - den) + f;    /* Fast2Sum, |f| < 2 */
  const double s = f / den;
  double rem = fma(-s, den, f);
  rem = rem - s * den_lo;
  const double s_lo = rem / den;
  const double z = s * s;
  double p = lc[11];
  p = fma(p, z, lc[10]);
  p = fma(p, z, lc[9]);
  p = fma(p, z, lc[8]);
  p = fma(p, z, lc[7]);
  p = fma(p, z, lc[6]);
  p = fma(p, z, lc[5]);
  p = fma(p, z, lc[4]);
  p = fma(p, z, lc[3]);
  p = fma(p, z, lc[2]);
  p = fma(p, z, lc[1]);
  p = fma(p, z, lc[0]);
  const double t_hi = 2.0 * s;
  const double t_lo = fma(z * s, p, 2.0 * s_lo);
  const double de = (double)e;
  const double a_hi = de * KTM_LN2_HI;      /* exact: 32-bit constant */
  const double a_lo = de * KTM_LN2_LO;
  /* TwoSum(a_hi, t_hi) */
  const double sum = a_hi + t_hi;
  const double bb = sum - a_hi;
  const double err = (a_hi - (sum - bb)) + (t_hi - bb);
  const double lo = err + (t_lo + a_lo);
  const double hi = sum + lo;
  *out_hi = hi;
  *out_lo = (sum - hi) + lo;
}

KTM_FN double ktm_log(double x) {
  if (ktm_isnan(x)) return x;
  if (x < 0.0) return ktm_nan();
  if (x == 0.0) return -ktm_inf();
  if (ktm_isinf(x)) return x;
  double h, l;
  ktm_log_dd(x, &h, &l);
  return h;
}

KTM_FN double ktm_log10(double x) {
  if (ktm_isnan(x)) return x;
  if (x < 0.0) return ktm_nan();
  if (x == 0.0) return -ktm_inf();
  if (ktm_isinf(x)) return x;
  double h, l;
  ktm_log_dd(x, &h, &l);
  const double p = h * KTM_INV_LN10_HI;
  const double pe = fma(h, KTM_INV_LN10_HI, -p);
  return p + (pe + fma(h, KTM_INV_LN10_LO, l * KTM_INV_LN10_HI));
}

/* -------------------------------------------------------------------- pow */

KTM_FN double ktm_pow(double x, double y) {
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  if (ktm_isnan(x) || ktm_isnan(y)) return x + y;
  const double ax = fabs(x);
  /* y_kind: 0 = not an integer, 1 = odd integer, 2 = even integer */
  int y_kind = 0;
  if (fabs(y) >= 0x1p53) {
    y_kind = ktm_isinf(y) ? 0 : 2;
  } else if (floor(y) == y) {
    y_kind = (fmod(y, 2.0) != 0.0) ? 1 : 2;
  }
  if (ktm_isinf(y)) {
    if (ax == 1.0) return 1.0;
    return ((ax > 1.0) == (y > 0.0)) ? ktm_inf() : 0.0;
  }
  if (x == 0.0) {
    const int neg = (ktm_bits(x) >> 63) != 0;
    if (y < 0.0) return (y_kind == 1 && neg) ? -ktm_inf() : ktm_inf();
    return (y_kind == 1 && neg) ? -0.0 : 0.0;
  }
  if (ktm_isinf(x)) {
    if (x > 0.0) return (y > 0.0) ? ktm_inf() : 0.0;
    if (y > 0.0) return (y_kind == 1) ? -ktm_inf() : ktm_inf();
    return (y_kind == 1) ? -0.0 : 0.0;
  }
  if (x < 0.0 && y_kind == 0) return ktm_nan();
  double lh, ll;
  ktm_log_dd(ax, &lh, &ll);
  const double ph = y * lh;
  const double pl = fma(y, lh, -ph) + y * ll;
  double r = ktm_exp_dd(ph, pl);
  if (x < 0.0 && y_kind == 1) r = -r;
  return r;
}

/* ------------------------------------------------------------------- cbrt */

KTM_FN double ktm_cbrt(double x) {
  if (x == 0.0 || ktm_isnan(x) || ktm_isinf(x)) return x;
  const int neg = x < 0.0;
  double a = fabs(x);
  int e = 0;
  if (a < 0x1p-1022) {
    a *= 0x1p54;
    e = -54;
  }
  uint64_t u = ktm_bits(a);
  e += (int)((u >> 52) & 0x7ff) - 1023;
  u = (u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m = ktm_from_bits(u); /* [1,2) */
  int q = e / 3;
  int rr = e - 3 * q;
  if (rr < 0) {
    rr += 3;
    q -= 1;
  }
  if (rr == 1) m *= 2.0;
  else if (rr == 2) m *= 4.0; /* m in [1,8), a = m 2^(3q) */
  /* Newton on y^3 = m from a linear start (error < 0.35 on [1,8)). */
  double y = 0.7 + 0.19 * m - 0.0085 * m * m;
  for (int i = 0; i < 6; ++i) y = y - (y * y * y - m) / (3.0 * y * y);
  /* final step with the residual y^3 - m evaluated in double-double */
  const double y2 = y * y;
  const double y2l = fma(y, y, -y2);
  const double y3 = y2 * y;
  const double y3l = fma(y2, y, -y3) + y2l * y;
  const double res = (y3 - m) + y3l;
  y = y - res / (3.0 * y2);
  y = ktm_scale(y, q);
  return neg ? -y : y;
}

/* ------------------------------------------------------------- atan2/acos */

/* atan(z + zl) for z in [0, 1], |zl| <= ulp(z), as (hi, lo). */
KTM_FN void ktm_atan01(double z, double zl, double* hi, double* lo) {
  const double th[9] = KTM_ATAN_TAB_HI;
  const double tl[9] = KTM_ATAN_TAB_LO;
  const double ac[9] = KTM_ATAN_COEFFS;
  int i = (int)(z * 8.0 + 0.5);
  if (i > 8) i = 8;
  const double c = 0.125 * (double)i;
  const double num = z - c;                 /* exact (Sterbenz) */
  const double den = fma(z, c, 1.0);
  const double t = num / den;
  const double t_lo = fma(-t, den, num) / den;
  const double t2 = t * t;
  double p = ac[8];
  p = fma(p, t2, ac[7]);
  p = fma(p, t2, ac[6]);
  p = fma(p, t2, ac[5]);
  p = fma(p, t2, ac[4]);
  p = fma(p, t2, ac[3]);
  p = fma(p, t2, ac[2]);
  p = fma(p, t2, ac[1]);
  p = fma(p, t2, ac[0]);
  /* zl enters through d atan/dz = 1/(1+z^2) */
  const double corr = t_lo + zl / fma(z, z, 1.0);
  const double at = t + fma(t * t2, p, corr);
  *hi = th[i];
  *lo = tl[i] + at;
}

KTM_FN double ktm_atan2(double y, double x) {
  if (ktm_isnan(x) || ktm_isnan(y)) return x + y;
  const int yneg = (ktm_bits(y) >> 63) != 0;
  const int xneg = (ktm_bits(x) >> 63) != 0;
  double res;
  if (y == 0.0) {
    res = xneg ? KTM_PI_HI : 0.0;
    return yneg ? -res : res;
  }
  if (x == 0.0) {
    res = KTM_PIO2_HI;
    return yneg ? -res : res;
  }
  const double ax = fabs(x), ay = fabs(y);
  if (ktm_isinf(ax) || ktm_isinf(ay)) {
    if (ktm_isinf(ax) && ktm_isinf(ay)) {
      res = xneg ? 3.0 * KTM_PIO4_HI : KTM_PIO4_HI;
    } else if (ktm_isinf(ax)) {
      res = xneg ? KTM_PI_HI : 0.0;
    } else {
      res = KTM_PIO2_HI;
    }
    return yneg ? -res : res;
  }
  double hi, lo;
  if (ay <= ax) {
    const double z = ay / ax;
    ktm_atan01(z, fma(-z, ax, ay) / ax, &hi, &lo);
  } else {
    double h2, l2;
    const double z = ax / ay;
    ktm_atan01(z, fma(-z, ay, ax) / ay, &h2, &l2);
    hi = KTM_PIO2_HI - h2;
    lo = (KTM_PIO2_HI - hi - h2) + (KTM_PIO2_LO - l2);
  }
  if (xneg) {
    const double h3 = KTM_PI_HI - hi;
    lo = (KTM_PI_HI - h3 - hi) + (KTM_PI_LO - lo);
    hi = h3;
  }
  res = hi + lo;
  return yneg ? -res : res;
}

KTM_FN double ktm_acos(double x) {
  if (ktm_isnan(x)) return x;
  if (fabs(x) > 1.0) return ktm_nan();
  return 2.0 * ktm_atan2(sqrt(1.0 - x), sqrt(1.0 + x));
}

/* atan(x) = atan2(x, 1): |x| <= 1 reduces to atan01(|x|) exactly. */
KTM_FN double ktm_atan(double x) { return ktm_atan2(x, 1.0); }

/* asin(x) = atan2(x, sqrt((1 - x)(1 + x))); 1 - x is exact for x >= 1/2. */
KTM_FN double ktm_asin(double x) {
  if (ktm_isnan(x)) return x;
  if (fabs(x) > 1.0) return ktm_nan();
  return ktm_atan2(x, sqrt((1.0 - x) * (1.0 + x)));
}

/* hypot(x, y) = sqrt(x^2 + y^2) without overflow or underflow: both scaled
 * by a power of two that brings the larger into [1, 2), the sum of squares
 * in double-double, one Newton correction of its square root. */
KTM_FN double ktm_hypot(double x, double y) {
  double a = fabs(x), b = fabs(y);
  if (ktm_isinf(a) || ktm_isinf(b)) return ktm_inf();
  if (ktm_isnan(a) || ktm_isnan(b)) return a + b;
  if (a < b) {
    const double t = a;
    a = b;
    b = t;
  }
  if (b == 0.0) return a;
  const int e = (int)((ktm_bits(a) >> 52) & 0x7ff) - 1023;
  const int k = e < -1000 ? -1000 : e;  /* subnormal a: a moderate scale is enough */
  a = ktm_scale(a, -k);
  b = ktm_scale(b, -k);
  const double h = a * a, hl = fma(a, a, -h);
  const double q = b * b, ql = fma(b, b, -q);
  const double s = h + q;
  const double sl = ((h - s) + q) + (hl + ql);
  double r = sqrt(s);
  r = r + (fma(-r, r, s) + sl) / (2.0 * r);
  return ktm_scale(r, k);
}

#endif /* KTMATH_H */
