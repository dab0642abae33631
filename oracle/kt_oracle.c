/* kt_oracle.c -- TEST INFRASTRUCTURE: CPU oracle of the geodesic path.
 *
 * Plain-C restatement of the reference renderer's per-pixel path.  Every
 * function names the reference lines it follows (paths relative to the
 * reference project root).  Expressions keep the reference's association
 * order, e.g. `a*b*c` is written (a*b)*c, because the parity bar is bit
 * equality.  Must be compiled with -ffp-contract=off.  Transcendentals come
 * from ktmath.h (the renderer's deterministic libm), exactly as in the strict
 * reference build; sqrt, division, fabs, floor and fmod are IEEE-exact
 * everywhere.  Not product code: see kt_oracle.h. */
#include "kt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../kerrtracecpp2_b200/csrc/ktmath.h"

#define ORC_PI 3.14159265358979323846 /* M_PI */

/* std::max / std::min / the clamp template (main.cpp:62-64), NaN semantics
 * included: max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a. */
static double omax(double a, double b) { return (a < b) ? b : a; }
static double omin(double a, double b) { return (b < a) ? b : a; }
static double oclamp(double v, double lo, double hi) { return v < lo ? lo : v > hi ? hi : v; }
static int oisfinite(double x) { return !ktm_isnan(x) && !ktm_isinf(x); }

typedef struct { double M, a, Q, L; } Metric;

/* ------------------------------------------------------------------ BL metric
 * knds_metric.hpp:45-132 */
static double m_sigma(const Metric* g, double r, double th) {
  const double ct = ktm_cos(th);
  return r * r + ((g->a * g->a) * ct) * ct;
}
static double m_delta_r(const Metric* g, double r) {
  return (((r * r + g->a * g->a) * (1.0 - ((g->L * r) * r) / 3.0)) - (2.0 * g->M) * r) + g->Q * g->Q;
}
static double m_delta_th(const Metric* g, double th) {
  const double ct = ktm_cos(th);
  return 1.0 + ((((g->L * g->a) * g->a) * ct) * ct) / 3.0;
}
static double m_xi(const Metric* g) { return 1.0 + ((g->L * g->a) * g->a) / 3.0; }

/* covariant_BL, knds_metric.hpp:71-88 */
static void m_cov_bl(const Metric* g, double r, double th, double G[4][4]) {
  const double sig = m_sigma(g, r, th);
  const double dr = m_delta_r(g, r);
  const double dth = m_delta_th(g, th);
  const double xi2 = m_xi(g) * m_xi(g);
  const double st = ktm_sin(th);
  const double st2 = st * st;
  const double a = g->a;
  const double r2a2 = r * r + a * a;
  const double pre = sig * xi2;
  memset(G, 0, 16 * sizeof(double));
  G[0][0] = (-dr + ((dth * a) * a) * st2) / pre;
  G[0][3] = G[3][0] = ((a * st2) * (dr - dth * r2a2)) / pre;
  G[1][1] = sig / dr;
  G[2][2] = sig / dth;
  G[3][3] = (st2 * ((dth * r2a2) * r2a2 - ((dr * a) * a) * st2)) / pre;
}

/* contravariant_BL, knds_metric.hpp:99-117 */
static void m_con_bl(const Metric* g, double r, double th, double G[4][4]) {
  const double sig = m_sigma(g, r, th);
  const double dr = m_delta_r(g, r);
  const double dth = m_delta_th(g, th);
  const double xi2 = m_xi(g) * m_xi(g);
  const double st = ktm_sin(th);
  const double st2 = st * st;
  const double a = g->a;
  const double r2a2 = r * r + a * a;
  const double pre = (sig * dr) * dth;
  memset(G, 0, 16 * sizeof(double));
  G[0][0] = ((-xi2) * ((dth * r2a2) * r2a2 - ((dr * a) * a) * st2)) / pre;
  G[0][3] = G[3][0] = ((a * xi2) * (dr - dth * r2a2)) / pre;
  G[1][1] = dr / sig;
  G[2][2] = dth / sig;
  if (st2 > 1e-14) G[3][3] = (xi2 * (dr - ((dth * a) * a) * st2)) / (pre * st2);
}

/* hamiltonian, knds_metric.hpp:122-132 */
static double m_ham(const Metric* g, double r, double th, double pr, double pth, double pt,
                    double pphi) {
  double G[4][4];
  m_con_bl(g, r, th, G);
  return 0.5 * (((((G[0][0] * pt) * pt + ((2.0 * G[0][3]) * pt) * pphi) + (G[1][1] * pr) * pr) +
                 (G[2][2] * pth) * pth) + (G[3][3] * pphi) * pphi);
}

/* ------------------------------------------------------------------ KS metric
 * knds_metric.hpp:150-230, ingoing (main.cpp:1312 KS_INGOING = true) */
static double m_r_ks(double X, double Y, double Z, double a) {
  const double R2 = (X * X + Y * Y) + Z * Z;
  const double a2 = a * a;
  const double b = R2 - a2;
  return sqrt(0.5 * (b + sqrt(b * b + ((4.0 * a2) * Z) * Z)));
}

static void m_con_ks(const Metric* g, double X, double Y, double Z, double G[4][4]) {
  const double a = g->a;
  const double r = m_r_ks(X, Y, Z, a);
  const double rho2 = r * r + (((a * a) * Z) * Z) / (r * r);
  const double H = ((2.0 * g->M) * r - g->Q * g->Q) / rho2;
  const double r2a2 = r * r + a * a;
  const double sa = 1.0 * a;
  const double l[4] = {1.0, (r * X + sa * Y) / r2a2, (r * Y - sa * X) / r2a2, Z / r};
  const double lU[4] = {-l[0], l[1], l[2], l[3]};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) G[i][j] = 0.0;
  G[0][0] = -1.0;
  G[1][1] = 1.0;
  G[2][2] = 1.0;
  G[3][3] = 1.0;
  for (int mu = 0; mu < 4; ++mu)
    for (int nu = 0; nu < 4; ++nu) G[mu][nu] -= (H * lU[mu]) * lU[nu];
}

static double m_ham_ks(const Metric* g, double X, double Y, double Z, const double p[4]) {
  double G[4][4];
  m_con_ks(g, X, Y, Z, G);
  double H = 0.0;
  for (int mu = 0; mu < 4; ++mu)
    for (int nu = 0; nu < 4; ++nu) H += (G[mu][nu] * p[mu]) * p[nu];
  return 0.5 * H;
}

/* BL_to_KS_spatial, knds_metric.hpp:368-387 */
static void m_bl_to_ks(double r, double th, double ph, double a, double* X, double* Y, double* Z) {
  const double st = ktm_sin(th), ct = ktm_cos(th);
  const double sf = ktm_sin(ph), cf = ktm_cos(ph);
  *X = st * (r * cf - a * sf);
  *Y = st * (r * sf + a * cf);
  *Z = r * ct;
}

/* KS_to_BL_spatial, knds_metric.hpp:390-411 (the first atan2 values are
 * overwritten there and never observed). */
static void m_ks_to_bl(double X, double Y, double Z, double a, double* r, double* th, double* ph) {
  *r = m_r_ks(X, Y, Z, a);
  const double rr = *r;
  const double Zr = Z / rr;
  *th = ktm_acos(Zr < -1.0 ? -1.0 : Zr > 1.0 ? 1.0 : Zr);
  const double st_val = sqrt(omax(1.0 - (Z * Z) / (rr * rr), 0.0));
  const double r2a2 = rr * rr + a * a;
  if (st_val > 1e-10) {
    const double cf = (X * rr + Y * a) / (st_val * r2a2);
    const double sf = (Y * rr - X * a) / (st_val * r2a2);
    *ph = ktm_atan2(sf, cf);
  } else {
    *ph = 0.0;
  }
}

/* ---------------------------------------------------------- horizon / ISCO */

/* r_horizon, knds_metric.hpp:237-315 */
static double orc_bisect(const Metric* g, double lo, double hi) {
  double flo = m_delta_r(g, lo), fhi = m_delta_r(g, hi);
  (void)fhi;
  if (!oisfinite(flo) || !oisfinite(fhi)) return ktm_nan();
  for (int i = 0; i < 160; ++i) {
    const double mid = 0.5 * (lo + hi);
    const double fmid = m_delta_r(g, mid);
    if (!oisfinite(fmid)) break;
    if ((flo > 0.0 && fmid < 0.0) || (flo < 0.0 && fmid > 0.0)) {
      hi = mid;
      fhi = fmid;
    } else {
      lo = mid;
      flo = fmid;
    }
  }
  return 0.5 * (lo + hi);
}

static void orc_push_root(double* roots, int* n, double rr) {
  if (!oisfinite(rr) || rr <= 0.0) return;
  for (int i = 0; i < *n; ++i) {
    /* std::max({1.0, |roots[i]|, |rr|}) */
    double rel = 1.0;
    if (rel < fabs(roots[i])) rel = fabs(roots[i]);
    if (rel < fabs(rr)) rel = fabs(rr);
    if (fabs(roots[i] - rr) <= 1e-8 * rel) return;
  }
  if (*n < 16) roots[(*n)++] = rr;
}

static int cmp_double(const void* x, const void* y) {
  const double a = *(const double*)x, b = *(const double*)y;
  return (a < b) ? -1 : (a > b) ? 1 : 0;
}

static double m_r_horizon(const Metric* g) {
  const double M = g->M, a = g->a, Q = g->Q, L = g->L;
  if (fabs(L) < 1e-15) {
    const double disc = (M * M - a * a) - Q * Q;
    return M + sqrt(omax(disc, 0.0));
  }
  const double scale = omax(fabs(M), 1.0);
  const double rmin = omax(1e-6 * scale, 1e-9);
  double rmax;
  if (L > 0.0)
    rmax = omax(20.0 * scale, 1.25 * sqrt(3.0 / L));
  else
    rmax = (200.0 * scale + 20.0 * fabs(a)) + 20.0 * fabs(Q);
  if (!(rmax > rmin)) rmax = rmin * 10.0;
  double roots[16];
  int nroots = 0;
  const int samples = 20000;
  const double log_span = ktm_log(rmax / rmin);
  double prev_r = rmin;
  double prev_f = m_delta_r(g, prev_r);
  for (int i = 1; i <= samples; ++i) {
    const double t = (double)i / (double)samples;
    const double r = rmin * ktm_exp(log_span * t);
    const double f = m_delta_r(g, r);
    if (oisfinite(prev_f) && oisfinite(f)) {
      if (prev_f == 0.0) orc_push_root(roots, &nroots, prev_r);
      if (f == 0.0) orc_push_root(roots, &nroots, r);
      if ((prev_f > 0.0 && f < 0.0) || (prev_f < 0.0 && f > 0.0))
        orc_push_root(roots, &nroots, orc_bisect(g, prev_r, r));
    }
    prev_r = r;
    prev_f = f;
  }
  if (nroots == 0) {
    const double disc = (M * M - a * a) - Q * Q;
    return M + sqrt(omax(disc, 0.0));
  }
  qsort(roots, (size_t)nroots, sizeof(double), cmp_double);
  if (L > 0.0 && nroots >= 2) return roots[nroots - 2];
  return roots[nroots - 1];
}

/* keplerian_omega, knds_metric.hpp:354-363 */
static double m_kepler(const Metric* g, double r) {
  const double s = (g->a < 0.0) ? 1.0 : -1.0;
  const double Meff = (g->M - (g->Q * g->Q) / (2.0 * r)) + (((g->L * g->a) * r) * r) / 3.0;
  const double sq = sqrt(omax(Meff, 0.0));
  const double den = r * sqrt(r) + (s * g->a) * sq;
  if (fabs(den) < 1e-14) return 0.0;
  return (s * sq) / den;
}

/* r_isco, knds_metric.hpp:318-349 */
static double m_l_circ(const Metric* g, double rr) {
  const double Om = m_kepler(g, rr);
  double G[4][4];
  m_cov_bl(g, rr, ORC_PI / 2.0, G);
  const double N2 = -((G[0][0] + (2.0 * G[0][3]) * Om) + (G[3][3] * Om) * Om);
  if (N2 <= 0.0) return -1e30;
  const double ut = 1.0 / sqrt(N2);
  return -(G[3][0] + G[3][3] * Om) * ut;
}

static double m_r_isco(const Metric* g) {
  const double M = g->M, a = g->a;
  if (fabs(g->L) < 1e-15 && fabs(g->Q) < 1e-15) {
    if (fabs(a) < 1e-10) return 6.0 * M;
    const double ap = a / M;
    const double z1 = 1.0 + ktm_cbrt(1.0 - ap * ap) * (ktm_cbrt(1.0 + ap) + ktm_cbrt(1.0 - ap));
    const double z2 = sqrt((3.0 * ap) * ap + z1 * z1);
    return M * ((3.0 + z2) - sqrt((3.0 - z1) * ((3.0 + z1) + 2.0 * z2)));
  }
  const double rh = m_r_horizon(g);
  double r = rh * 1.05;
  const double dr = 1e-4 * M;
  double L_prev = m_l_circ(g, r);
  for (; r < 30.0 * M; r += dr) {
    const double L = m_l_circ(g, r + dr);
    if (L < L_prev && L_prev > 0.0) return r;
    L_prev = L;
  }
  return r;
}

double orc_r_horizon(double M, double a, double Q, double L) {
  const Metric g = {M, a, Q, L};
  return m_r_horizon(&g);
}
double orc_r_isco(double M, double a, double Q, double L) {
  const Metric g = {M, a, Q, L};
  return m_r_isco(&g);
}

/* ------------------------------------------------------------------ camera
 * camera.hpp:38-145 */
typedef struct { double r, th, ph, pr, pth, pt, pphi; } Geo; /* GeodesicState */

typedef struct {
  double r_obs, theta_obs, phi_obs, fov_h;
  int W, H;
} Cam;

static Geo cam_angle_ray(const Cam* c, double alpha, double beta, const Metric* g) {
  const double r0 = c->r_obs, th0 = c->theta_obs;
  double G[4][4];
  m_cov_bl(g, r0, th0, G);
  const double ca = ktm_cos(alpha), sa = ktm_sin(alpha);
  const double cb = ktm_cos(beta), sb = ktm_sin(beta);
  const double gtt = G[0][0], gtphi = G[0][3], grr = G[1][1], gthth = G[2][2], gphph = G[3][3];
  const double sqrt_grr = sqrt(fabs(grr));
  const double sqrt_gthth = sqrt(fabs(gthth));
  const double denom_phi = gphph - (gtphi * gtphi) / gtt;
  const int tetrad_ok = (gtt < -1e-14) && oisfinite(denom_phi) && (denom_phi > 1e-14) &&
                        oisfinite(sqrt_grr) && (sqrt_grr > 1e-14) && oisfinite(sqrt_gthth) &&
                        (sqrt_gthth > 1e-14);
  double pUt = 1.0;
  double pUr = ((-ca) * cb) / omax(sqrt_grr, 1e-14);
  double pUth = (-sb) / omax(sqrt_gthth, 1e-14);
  double pUphi = ((-sa) * cb) / sqrt(omax(fabs(gphph), 1e-14));
  if (tetrad_ok) {
    const double ut = 1.0 / sqrt(-gtt);
    const double ephi_p = 1.0 / sqrt(denom_phi);
    const double ephi_t = ((-gtphi) / gtt) * ephi_p;
    const double n_r = (-ca) * cb;
    const double n_th = -sb;
    const double n_ph = (-sa) * cb;
    pUt = ut + n_ph * ephi_t;
    pUr = n_r / sqrt_grr;
    pUth = n_th / sqrt_gthth;
    pUphi = n_ph * ephi_p;
  }
  double pt = gtt * pUt + gtphi * pUphi;
  const double pr = grr * pUr;
  const double pth = gthth * pUth;
  const double pphi = gtphi * pUt + gphph * pUphi;
  double U[4][4];
  m_con_bl(g, r0, th0, U);
  const double A = U[0][0];
  const double B = (2.0 * U[0][3]) * pphi;
  const double C = ((U[1][1] * pr) * pr + (U[2][2] * pth) * pth) + (U[3][3] * pphi) * pphi;
  const double disc = B * B - (4.0 * A) * C;
  if (disc >= 0.0 && fabs(A) > 1e-15) {
    const double sq = sqrt(disc);
    const double pt1 = (-B - sq) / (2.0 * A);
    const double pt2 = (-B + sq) / (2.0 * A);
    pt = (pt1 < 0.0) ? pt1 : pt2;
    if (pt > 0.0) pt = omin(pt1, pt2);
  }
  Geo s = {r0, th0, c->phi_obs, pr, pth, pt, pphi};
  return s;
}

static void cam_pixel_angles(const Cam* c, int px, int py, double offx, double offy,
                             double* alpha, double* beta) {
  const int span = (c->W > 1) ? (c->W - 1) : 1;
  const double x = (double)px + offx;
  const double y = (double)py + offy;
  *alpha = (c->fov_h * (x - 0.5 * (double)(c->W - 1))) / (double)span;
  *beta = (c->fov_h * (0.5 * (double)(c->H - 1) - y)) / (double)span;
}

/* ------------------------------------------------------------- integrators
 * geodesic.hpp:40-431 */
static double dphi_vel(const Metric* g, double r, double th, double pt, double pphi) {
  double U[4][4];
  m_con_bl(g, r, th, U);
  return U[3][0] * pt + U[3][3] * pphi;
}

static double clamp01(double x) {
  if (x < 0.0) return 0.0;
  if (x > 1.0) return 1.0;
  return x;
}

static double hermite(double y0, double y1, double dy0, double dy1, double h, double alpha) {
  alpha = clamp01(alpha);
  const double a2 = alpha * alpha;
  const double a3 = a2 * alpha;
  const double h00 = (2.0 * a3 - 3.0 * a2) + 1.0;
  const double h10 = (a3 - 2.0 * a2) + alpha;
  const double h01 = -2.0 * a3 + 3.0 * a2;
  const double h11 = a3 - a2;
  return ((h00 * y0 + h10 * (h * dy0)) + h01 * y1) + h11 * (h * dy1);
}

static int sign_change(double f0, double f1) {
  return ((f0 <= 0.0 && f1 >= 0.0) || (f0 >= 0.0 && f1 <= 0.0));
}

/* first_event_alpha_hermite, geodesic.hpp:98-140, bins = iterations = 8 */
static int first_event(double y0, double y1, double dy0, double dy1, double h, double target,
                       double* alpha_out) {
  const int bins = 8, iterations = 8;
  const double f_eps = 1e-12;
  double a0 = 0.0;
  double f0 = y0 - target;
  if (fabs(f0) <= f_eps) {
    *alpha_out = 0.0;
    return 1;
  }
  for (int i = 1; i <= bins; ++i) {
    const double a1 = (double)i / (double)bins;
    const double f1 = (i == bins) ? (y1 - target) : (hermite(y0, y1, dy0, dy1, h, a1) - target);
    if (fabs(f1) <= f_eps) {
      *alpha_out = a1;
      return 1;
    }
    if (sign_change(f0, f1)) {
      double lo = a0, hi = a1;
      for (int k = 0; k < iterations; ++k) {
        const double mid = 0.5 * (lo + hi);
        const double fm = hermite(y0, y1, dy0, dy1, h, mid) - target;
        if (sign_change(f0, fm))
          hi = mid;
        else
          lo = mid;
      }
      *alpha_out = 0.5 * (lo + hi);
      return 1;
    }
    a0 = a1;
    f0 = f1;
  }
  return 0;
}

/* geodesic_rhs, geodesic.hpp:143-166 */
static void geo_rhs(const Metric* g, double r, double th, double pr, double pth, double pt,
                    double pphi, double* dr, double* dth, double* dpr, double* dpth) {
  double U[4][4];
  m_con_bl(g, r, th, U);
  *dr = U[1][1] * pr;
  *dth = U[2][2] * pth;
  const double eps_r = 1e-5 * omax(fabs(r), 0.01);
  const double eps_th = 1e-6;
  *dpr = -(m_ham(g, r + eps_r, th, pr, pth, pt, pphi) - m_ham(g, r - eps_r, th, pr, pth, pt, pphi)) /
         (2.0 * eps_r);
  *dpth = -(m_ham(g, r, th + eps_th, pr, pth, pt, pphi) - m_ham(g, r, th - eps_th, pr, pth, pt, pphi)) /
          (2.0 * eps_th);
}

/* rk4_step, geodesic.hpp:169-194 */
static void rk4_step(const Metric* g, Geo* s, double dlam) {
  double dr1, dth1, dpr1, dpth1, dr2, dth2, dpr2, dpth2, dr3, dth3, dpr3, dpth3, dr4, dth4, dpr4,
      dpth4;
  const double r = s->r, th = s->th, pr = s->pr, pth = s->pth, pt = s->pt, pp = s->pphi;
  const double hd = 0.5 * dlam;
  geo_rhs(g, r, th, pr, pth, pt, pp, &dr1, &dth1, &dpr1, &dpth1);
  geo_rhs(g, r + hd * dr1, th + hd * dth1, pr + hd * dpr1, pth + hd * dpth1, pt, pp, &dr2, &dth2,
          &dpr2, &dpth2);
  geo_rhs(g, r + hd * dr2, th + hd * dth2, pr + hd * dpr2, pth + hd * dpth2, pt, pp, &dr3, &dth3,
          &dpr3, &dpth3);
  geo_rhs(g, r + dlam * dr3, th + dlam * dth3, pr + dlam * dpr3, pth + dlam * dpth3, pt, pp, &dr4,
          &dth4, &dpr4, &dpth4);
  const double dp1 = dphi_vel(g, r, th, pt, pp);
  const double dp2 = dphi_vel(g, r + hd * dr1, th + hd * dth1, pt, pp);
  const double dp3 = dphi_vel(g, r + hd * dr2, th + hd * dth2, pt, pp);
  const double dp4 = dphi_vel(g, r + dlam * dr3, th + dlam * dth3, pt, pp);
  const double w = dlam / 6.0;
  s->r += w * (((dr1 + 2.0 * dr2) + 2.0 * dr3) + dr4);
  s->th += w * (((dth1 + 2.0 * dth2) + 2.0 * dth3) + dth4);
  s->ph += w * (((dp1 + 2.0 * dp2) + 2.0 * dp3) + dp4);
  s->pr += w * (((dpr1 + 2.0 * dpr2) + 2.0 * dpr3) + dpr4);
  s->pth += w * (((dpth1 + 2.0 * dpth2) + 2.0 * dpth3) + dpth4);
}

/* Step-size update shared by every step-doubling controller
 * (geodesic.hpp:226-256, main.cpp:1507-1527, ray_bundle.hpp:235-262). */
static int doubling_update(double err, double tol, double* dlam) {
  if (!oisfinite(err)) {
    *dlam = (oisfinite(*dlam) && *dlam > 1e-10) ? *dlam * 0.5 : 1e-6;
    if (*dlam < 1e-10) *dlam = 1e-10;
    return -1;
  }
  const int accepted = (err < tol || *dlam < 1e-10);
  if (accepted) {
    const double scale = (err > 1e-14) ? 0.9 * ktm_pow(tol / err, 0.2) : 4.0;
    double hnew = *dlam * scale;
    if (!oisfinite(hnew)) hnew = *dlam;
    *dlam = hnew;
    if (*dlam > 100.0) *dlam = 100.0;
    if (*dlam < 1e-10) *dlam = 1e-10;
  } else {
    const double half = *dlam * 0.5;
    double hnew = (*dlam * 0.9) * ktm_pow(tol / err, 0.25);
    if (!oisfinite(hnew)) hnew = half;
    *dlam = hnew;
    if (*dlam > half) *dlam = half;
    if (*dlam < 1e-10) *dlam = 1e-10;
  }
  return accepted;
}

/* rk4_adaptive, geodesic.hpp:204-257 */
static int rk4_adaptive(const Metric* g, Geo* s, double* dlam, double tol) {
  const Geo s0 = *s;
  Geo sA = s0;
  rk4_step(g, &sA, *dlam);
  Geo sB = s0;
  rk4_step(g, &sB, 0.5 * *dlam);
  rk4_step(g, &sB, 0.5 * *dlam);
  const double e0 = sA.r - sB.r, e1 = sA.th - sB.th, e2 = sA.pr - sB.pr, e3 = sA.pth - sB.pth;
  const double err = sqrt(((e0 * e0 + e1 * e1) + e2 * e2) + e3 * e3) / 15.0;
  const int acc = doubling_update(err, tol, dlam);
  *s = (acc == 1) ? sB : s0;
  return acc == 1;
}

/* DOPRI5, geodesic.hpp:262-414 */
typedef struct { double v[4]; } Vec4;

static void eval_rhs(const Metric* g, const Geo* s, Vec4* k) {
  geo_rhs(g, s->r, s->th, s->pr, s->pth, s->pt, s->pphi, &k->v[0], &k->v[1], &k->v[2], &k->v[3]);
}

static Geo advance(const Geo* s0, double h, const Vec4* ks, const double* w, int nk) {
  Geo s = *s0;
  for (int i = 0; i < nk; ++i) {
    s.r += (h * w[i]) * ks[i].v[0];
    s.th += (h * w[i]) * ks[i].v[1];
    s.pr += (h * w[i]) * ks[i].v[2];
    s.pth += (h * w[i]) * ks[i].v[3];
  }
  return s;
}

static int dopri5_adaptive(const Metric* g, Geo* s, double* h, Vec4* fsal, double tol) {
  Vec4 k[7];
  if (!ktm_isnan(fsal->v[0]))
    k[0] = *fsal;
  else
    eval_rhs(g, s, &k[0]);
  static const double a2[1] = {1.0 / 5.0};
  static const double a3[2] = {3.0 / 40.0, 9.0 / 40.0};
  static const double a4[3] = {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0};
  static const double a5[4] = {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0};
  static const double a6[5] = {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0,
                               -5103.0 / 18656.0};
  static const double b5[6] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0,
                               11.0 / 84.0};
  static const double b4[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0,
                               -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
  Geo st = advance(s, *h, k, a2, 1);
  eval_rhs(g, &st, &k[1]);
  st = advance(s, *h, k, a3, 2);
  eval_rhs(g, &st, &k[2]);
  st = advance(s, *h, k, a4, 3);
  eval_rhs(g, &st, &k[3]);
  st = advance(s, *h, k, a5, 4);
  eval_rhs(g, &st, &k[4]);
  st = advance(s, *h, k, a6, 5);
  eval_rhs(g, &st, &k[5]);
  const Geo y5 = advance(s, *h, k, b5, 6);
  eval_rhs(g, &y5, &k[6]);
  const Geo y4 = advance(s, *h, k, b4, 7);
  const double dy[4] = {y5.r - y4.r, y5.th - y4.th, y5.pr - y4.pr, y5.pth - y4.pth};
  const double ref[4] = {s->r, s->th, s->pr, s->pth};
  double err2 = 0.0;
  for (int i = 0; i < 4; ++i) {
    const double ratio = dy[i] / (tol * (1.0 + fabs(ref[i])));
    err2 += ratio * ratio;
  }
  const double err = sqrt(err2 / 4.0);
  if (!oisfinite(err)) {
    *h = (oisfinite(*h) && *h > 1e-10) ? *h * 0.5 : 1e-6;
    if (*h < 1e-10) *h = 1e-10;
    fsal->v[0] = ktm_nan();
    return 0;
  }
  const int accepted = (err <= 1.0 || *h < 1e-10);
  if (accepted) {
    *s = y5;
    *fsal = k[6];
    const double fac = (err > 1e-12) ? 0.9 * ktm_pow(1.0 / err, 0.2) : 4.0;
    double hnew = *h * fac;
    if (!oisfinite(hnew)) hnew = *h;
    if (hnew > 100.0) hnew = 100.0;
    if (hnew < 1e-10) hnew = 1e-10;
    *h = hnew;
  } else {
    double hnew = (*h * 0.9) * ktm_pow(1.0 / err, 0.25);
    if (!oisfinite(hnew)) hnew = *h * 0.5;
    *h = omax(hnew, 1e-10);
    fsal->v[0] = ktm_nan();
  }
  return accepted;
}

/* ---------------------------------------------------------------- results */
typedef struct {
  uint8_t outcome;
  double r, redshift, magnif, phi_disk, theta_esc, phi_esc;
  uint32_t steps, attempts;
} Ray;

/* TraceResult{out, r, redshift, phi_disk, theta_esc, phi_esc} (main.cpp:187-191) */
static Ray ray_result(int outcome, double r, double red, double phi_disk, double th_esc,
                      double ph_esc) {
  Ray o;
  o.outcome = (uint8_t)outcome;
  o.r = r;
  o.redshift = red;
  o.magnif = 1.0;
  o.phi_disk = phi_disk;
  o.theta_esc = th_esc;
  o.phi_esc = ph_esc;
  o.steps = o.attempts = 0;
  return o;
}

/* disk_redshift, main.cpp:329-341 */
static double disk_redshift(const Metric* g, double r, double pt, double pphi) {
  const double Om = m_kepler(g, r);
  const double b = (-pphi) / (-pt);
  double G[4][4];
  m_cov_bl(g, r, ORC_PI / 2.0, G);
  const double d2 = -((G[0][0] + (2.0 * G[0][3]) * Om) + (G[3][3] * Om) * Om);
  if (d2 <= 0.0) return 1.0;
  const double dv = fabs(1.0 - Om * b);
  if (dv < 1e-8) return 20.0;
  const double red = sqrt(d2) / dv;
  return oisfinite(red) ? red : 1.0;
}

typedef struct {
  Metric g;
  Cam cam;
  int chart, intg, bundles;
  int solver; /* effective RaySolverMode: KT_SOLVER_STANDARD or KT_SOLVER_SEMI_ANALYTIC */
  int max_steps;
  double step_init, tol;
  double r_in, r_out, r_esc, rh;
  double offx, offy;
} Frame;

enum { EV_NONE, EV_DISK, EV_HORIZON, EV_ESCAPE };

/* trace_single, main.cpp:343-434 */
static Ray trace_single(const Frame* f, Geo s) {
  const Metric* g = &f->g;
  const double rh_cut = f->rh * 1.03;
  double dlam = omax(f->step_init, 1e-10);
  Vec4 fsal;
  fsal.v[0] = fsal.v[1] = fsal.v[2] = fsal.v[3] = ktm_nan();
  const int max_steps = f->max_steps < 1 ? 1 : f->max_steps;
  uint32_t att = 0;
  for (int it = 0; it < max_steps; ++it) {
    const Geo sp = s;
    double step_used = dlam;
    int rejects = 0;
    for (;;) {
      step_used = dlam;
      ++att;
      const int acc = (f->intg == KT_DOPRI5) ? dopri5_adaptive(g, &s, &dlam, &fsal, f->tol)
                                             : rk4_adaptive(g, &s, &dlam, f->tol);
      if (acc) break;
      if (!oisfinite(dlam) || ++rejects > 64) {
        Ray o = ray_result(KT_OUT_ESCAPED, s.r, 1.0, s.th, s.ph, 0.0);
        o.steps = (uint32_t)it;
        o.attempts = att;
        return o;
      }
    }
    double best_alpha = 2.0;
    int ev = EV_NONE;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    const double q0 = sp.th - ORC_PI / 2.0;
    const double q1 = s.th - ORC_PI / 2.0;
    if (sign_change(q0, q1) || (omin(fabs(q0), fabs(q1)) < 0.35)) {
      double dr0, dth0, dpr0, dpth0, dr1, dth1, dpr1, dpth1;
      geo_rhs(g, sp.r, sp.th, sp.pr, sp.pth, sp.pt, sp.pphi, &dr0, &dth0, &dpr0, &dpth0);
      geo_rhs(g, s.r, s.th, s.pr, s.pth, s.pt, s.pphi, &dr1, &dth1, &dpr1, &dpth1);
      double alpha = 0.0;
      if (first_event(sp.th, s.th, dth0, dth1, step_used, ORC_PI / 2.0, &alpha)) {
        const double r_hit = hermite(sp.r, s.r, dr0, dr1, step_used, alpha);
        if (r_hit >= f->r_in && r_hit <= f->r_out) {
          disk_r = r_hit;
          disk_red = oclamp(disk_redshift(g, r_hit, s.pt, s.pphi), 0.0, 20.0);
          disk_phi = sp.ph + alpha * (s.ph - sp.ph);
          best_alpha = alpha;
          ev = EV_DISK;
        }
      }
    }
    if (s.r <= rh_cut) {
      const double denom_h = sp.r - s.r;
      double alpha_h = (fabs(denom_h) > 1e-12) ? ((sp.r - rh_cut) / denom_h) : 0.0;
      alpha_h = oclamp(alpha_h, 0.0, 1.0);
      if (alpha_h < best_alpha) {
        best_alpha = alpha_h;
        ev = EV_HORIZON;
      }
    }
    if (s.r >= f->r_esc) {
      const double denom_e = s.r - sp.r;
      double alpha_e = (fabs(denom_e) > 1e-12) ? ((f->r_esc - sp.r) / denom_e) : 1.0;
      alpha_e = oclamp(alpha_e, 0.0, 1.0);
      if (alpha_e < best_alpha) {
        best_alpha = alpha_e;
        ev = EV_ESCAPE;
      }
    }
    Ray o;
    if (ev == EV_DISK) {
      o = ray_result(KT_OUT_DISK, disk_r, disk_red, disk_phi, 0.0, 0.0);
    } else if (ev == EV_HORIZON) {
      o = ray_result(KT_OUT_HORIZON, sp.r + best_alpha * (s.r - sp.r), 0.0, 0.0, 0.0, 0.0);
    } else if (ev == EV_ESCAPE) {
      const double th_esc = sp.th + best_alpha * (s.th - sp.th);
      const double ph_esc = sp.ph + best_alpha * (s.ph - sp.ph);
      o = ray_result(KT_OUT_ESCAPED, f->r_esc, 1.0, th_esc, ph_esc, 0.0);
    } else {
      continue;
    }
    o.steps = (uint32_t)it + 1;
    o.attempts = att;
    return o;
  }
  Ray o = ray_result(KT_OUT_ESCAPED, s.r, 1.0, s.th, s.ph, 0.0);
  o.steps = (uint32_t)max_steps;
  o.attempts = att;
  return o;
}

/* --------------------------------------------- separable Kerr tracer
 * The semi-analytic solver (main.cpp:436-703): Kerr only (Q = Lambda = 0),
 * BL chart.  The first integrals E = -p_t, L_z = p_phi and Carter's Q_c
 * reduce the ray to (r, theta, phi) with the radial and polar potentials
 * R(r), Theta(theta) and the branch signs of dr and dtheta; RK4 step
 * doubling on those three.  Any failure restarts the ray on the standard
 * BL tracer with RK4 step doubling. */
typedef struct { double M, a, E, Lz, Qc; } SepC;           /* SeparableKerrConsts */
typedef struct { double r, th, ph; int sr, sth; } SepS;     /* SeparableState */

/* init_separable_consts, main.cpp:454-468 */
static int sep_init(const Geo* s, const Metric* g, SepC* c) {
  if (fabs(g->Q) > 1e-15 || fabs(g->L) > 1e-15) return 0;
  c->M = g->M;
  c->a = g->a;
  c->E = -s->pt;
  c->Lz = s->pphi;
  if (!(oisfinite(c->E) && oisfinite(c->Lz) && c->E > 0.0)) return 0;
  const double st = ktm_sin(s->th), ct = ktm_cos(s->th);
  const double st2 = omax(st * st, 1e-14);
  c->Qc = s->pth * s->pth + (ct * ct) * ((c->Lz * c->Lz) / st2 - ((c->a * c->a) * c->E) * c->E);
  return oisfinite(c->Qc);
}

/* kerr_sep_delta, kerr_sep_R, kerr_sep_Theta (main.cpp:470-486) */
static double sep_delta(const SepC* c, double r) { return (r * r - (2.0 * c->M) * r) + c->a * c->a; }

static double sep_R(const SepC* c, double r) {
  const double P = c->E * (r * r + c->a * c->a) - c->a * c->Lz;
  const double u = c->Lz - c->a * c->E;
  const double K = c->Qc + u * u;
  return P * P - sep_delta(c, r) * K;
}

static double sep_Theta(const SepC* c, double th) {
  const double st = ktm_sin(th), ct = ktm_cos(th);
  const double st2 = omax(st * st, 1e-14);
  return c->Qc - (ct * ct) * ((c->Lz * c->Lz) / st2 - ((c->a * c->a) * c->E) * c->E);
}

/* kerr_sep_rhs, main.cpp:488-504 */
static int sep_rhs(const SepC* c, const SepS* s, double* dr, double* dth, double* dph) {
  const double st = ktm_sin(s->th), ct = ktm_cos(s->th);
  const double st2 = omax(st * st, 1e-14);
  const double sig = omax(s->r * s->r + ((c->a * c->a) * ct) * ct, 1e-14);
  const double del = sep_delta(c, s->r);
  const double P = c->E * (s->r * s->r + c->a * c->a) - c->a * c->Lz;
  const double R = sep_R(c, s->r);
  const double T = sep_Theta(c, s->th);
  *dr = ((s->sr >= 0) ? 1.0 : -1.0) * sqrt(omax(R, 0.0)) / sig;
  *dth = ((s->sth >= 0) ? 1.0 : -1.0) * sqrt(omax(T, 0.0)) / sig;
  *dph = (c->Lz / st2 + c->a * (P / omax(del, 1e-14) - c->E)) / sig;
  return oisfinite(*dr) && oisfinite(*dth) && oisfinite(*dph);
}

/* rk4_step_separable_kerr, main.cpp:506-537 */
static int sep_rk4(const SepC* c, SepS* s, double h) {
  double r1, t1, p1, r2, t2, p2, r3, t3, p3, r4, t4, p4;
  const SepS s0 = *s;
  SepS q = s0;
  if (!sep_rhs(c, &s0, &r1, &t1, &p1)) return 0;
  q.r = s0.r + (0.5 * h) * r1;
  q.th = s0.th + (0.5 * h) * t1;
  q.ph = s0.ph + (0.5 * h) * p1;
  if (!sep_rhs(c, &q, &r2, &t2, &p2)) return 0;
  q.r = s0.r + (0.5 * h) * r2;
  q.th = s0.th + (0.5 * h) * t2;
  q.ph = s0.ph + (0.5 * h) * p2;
  if (!sep_rhs(c, &q, &r3, &t3, &p3)) return 0;
  q.r = s0.r + h * r3;
  q.th = s0.th + h * t3;
  q.ph = s0.ph + h * p3;
  if (!sep_rhs(c, &q, &r4, &t4, &p4)) return 0;
  const double w = h / 6.0;
  s->r += w * (((r1 + 2.0 * r2) + 2.0 * r3) + r4);
  s->th += w * (((t1 + 2.0 * t2) + 2.0 * t3) + t4);
  s->ph += w * (((p1 + 2.0 * p2) + 2.0 * p3) + p4);
  return oisfinite(s->r) && oisfinite(s->th) && oisfinite(s->ph);
}

/* rk4_adaptive_separable_kerr, main.cpp:539-576: 1 accepted, 0 rejected */
static int sep_adaptive(const SepC* c, SepS* s, double* h, double tol) {
  SepS A = *s, B = *s;
  if (!sep_rk4(c, &A, *h) || !sep_rk4(c, &B, 0.5 * *h) || !sep_rk4(c, &B, 0.5 * *h)) {
    *h = omax(*h * 0.5, 1e-10);
    return 0;
  }
  const double e0 = A.r - B.r, e1 = A.th - B.th, e2 = A.ph - B.ph;
  const double err = sqrt((e0 * e0 + e1 * e1) + e2 * e2) / 15.0;
  if (!oisfinite(err)) {
    *h = omax(*h * 0.5, 1e-10);
    return 0;
  }
  if (err < tol || *h < 1e-10) {
    *s = B;
    const double sc = (err > 1e-14) ? 0.9 * ktm_pow(tol / err, 0.2) : 4.0;
    *h = oclamp(*h * sc, 1e-10, 100.0);
    return 1;
  }
  *h = omax((*h * 0.9) * ktm_pow(tol / err, 0.25), 1e-10);
  return 0;
}

/* trace_single_separable_kerr, main.cpp:578-703.  The standard tracer it
 * falls back to always integrates with RK4 step doubling. */
static Ray trace_separable(const Frame* f, const Geo* sbl) {
  Frame fb = *f;
  fb.intg = KT_RK4_DOUBLING;
  SepC c;
  if (!sep_init(sbl, &f->g, &c)) return trace_single(&fb, *sbl);
  double dr0, dth0, dpr0, dpth0;
  geo_rhs(&f->g, sbl->r, sbl->th, sbl->pr, sbl->pth, sbl->pt, sbl->pphi, &dr0, &dth0, &dpr0, &dpth0);
  SepS s = {sbl->r, sbl->th, sbl->ph, dr0 >= 0.0 ? 1 : -1, dth0 >= 0.0 ? 1 : -1};
  const double rh_cut = f->rh * 1.03;
  double h = omax(f->step_init, 1e-10);
  double prevR = sep_R(&c, s.r), prevT = sep_Theta(&c, s.th);
  const int max_steps = f->max_steps < 1 ? 1 : f->max_steps;
  uint32_t att = 0;
  for (int it = 0; it < max_steps; ++it) {
    const SepS sp = s;
    double step_used = h;
    int rejects = 0;
    for (;;) {
      step_used = h;
      ++att;
      if (sep_adaptive(&c, &s, &h, f->tol)) break;
      if (!oisfinite(h) || ++rejects > 64) return trace_single(&fb, *sbl);
    }
    if (s.th < 0.0) {
      s.th = -s.th;
      s.sth = -s.sth;
    } else if (s.th > ORC_PI) {
      s.th = 2.0 * ORC_PI - s.th;
      s.sth = -s.sth;
    }
    const double Rn = sep_R(&c, s.r), Tn = sep_Theta(&c, s.th);
    if (Rn <= 1e-9 && prevR > 1e-9) s.sr = -s.sr;
    if (Tn <= 1e-11 && prevT > 1e-11) s.sth = -s.sth;

    double best_alpha = 2.0;
    int ev = EV_NONE;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    const double q0 = sp.th - ORC_PI / 2.0;
    const double q1 = s.th - ORC_PI / 2.0;
    if (sign_change(q0, q1) || (omin(fabs(q0), fabs(q1)) < 0.35)) {
      double a0, b0, c0, a1, b1, c1;
      if (!sep_rhs(&c, &sp, &a0, &b0, &c0) || !sep_rhs(&c, &s, &a1, &b1, &c1))
        return trace_single(&fb, *sbl);
      double alpha = 0.0;
      if (first_event(sp.th, s.th, b0, b1, step_used, ORC_PI / 2.0, &alpha)) {
        const double r_hit = hermite(sp.r, s.r, a0, a1, step_used, alpha);
        if (r_hit >= f->r_in && r_hit <= f->r_out) {
          disk_r = r_hit;
          disk_red = oclamp(disk_redshift(&f->g, r_hit, sbl->pt, sbl->pphi), 0.0, 20.0);
          disk_phi = sp.ph + alpha * (s.ph - sp.ph);
          best_alpha = alpha;
          ev = EV_DISK;
        }
      }
    }
    if (s.r <= rh_cut) {
      const double denom_h = sp.r - s.r;
      double alpha_h = (fabs(denom_h) > 1e-12) ? ((sp.r - rh_cut) / denom_h) : 0.0;
      alpha_h = oclamp(alpha_h, 0.0, 1.0);
      if (alpha_h < best_alpha) {
        best_alpha = alpha_h;
        ev = EV_HORIZON;
      }
    }
    if (s.r >= f->r_esc) {
      const double denom_e = s.r - sp.r;
      double alpha_e = (fabs(denom_e) > 1e-12) ? ((f->r_esc - sp.r) / denom_e) : 1.0;
      alpha_e = oclamp(alpha_e, 0.0, 1.0);
      if (alpha_e < best_alpha) {
        best_alpha = alpha_e;
        ev = EV_ESCAPE;
      }
    }
    Ray o;
    if (ev == EV_DISK) {
      o = ray_result(KT_OUT_DISK, disk_r, disk_red, disk_phi, 0.0, 0.0);
    } else if (ev == EV_HORIZON) {
      o = ray_result(KT_OUT_HORIZON, sp.r + best_alpha * (s.r - sp.r), 0.0, 0.0, 0.0, 0.0);
    } else if (ev == EV_ESCAPE) {
      const double th_esc = sp.th + best_alpha * (s.th - sp.th);
      const double ph_esc = sp.ph + best_alpha * (s.ph - sp.ph);
      o = ray_result(KT_OUT_ESCAPED, f->r_esc, 1.0, th_esc, ph_esc, 0.0);
    } else {
      prevR = Rn;
      prevT = Tn;
      continue;
    }
    o.steps = (uint32_t)it + 1;
    o.attempts = att;
    return o;
  }
  Ray o = ray_result(KT_OUT_ESCAPED, s.r, 1.0, s.th, s.ph, 0.0);
  o.steps = (uint32_t)max_steps;
  o.attempts = att;
  return o;
}

/* ------------------------------------------------------------- KS tracer
 * main.cpp:1306-1660 */
typedef struct { double X, Y, Z, pX, pY, pZ, pT; } KS;

static int solve_3x3(const double Ain[3][3], const double bin[3], double x[3]) {
  double A[3][4];
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) A[i][j] = Ain[i][j];
    A[i][3] = bin[i];
  }
  for (int col = 0; col < 3; ++col) {
    int piv = col;
    double best = fabs(A[piv][col]);
    for (int r = col + 1; r < 3; ++r) {
      const double v = fabs(A[r][col]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (best < 1e-14) return 0;
    if (piv != col) {
      for (int k = col; k < 4; ++k) {
        const double t = A[col][k];
        A[col][k] = A[piv][k];
        A[piv][k] = t;
      }
    }
    const double inv = 1.0 / A[col][col];
    for (int k = col; k < 4; ++k) A[col][k] *= inv;
    for (int r = 0; r < 3; ++r) {
      if (r == col) continue;
      const double fr = A[r][col];
      for (int k = col; k < 4; ++k) A[r][k] -= fr * A[col][k];
    }
  }
  x[0] = A[0][3];
  x[1] = A[1][3];
  x[2] = A[2][3];
  return 1;
}

static void jacobian_bl_to_ks(double r, double th, double ph, double a, double J[3][3]) {
  const double er = 1e-6 * (fabs(r) + 1.0);
  const double eth = 1e-6;
  const double eph = 1e-6;
  double p[6][3];
  m_bl_to_ks(r + er, th, ph, a, &p[0][0], &p[0][1], &p[0][2]);
  m_bl_to_ks(r - er, th, ph, a, &p[1][0], &p[1][1], &p[1][2]);
  m_bl_to_ks(r, th + eth, ph, a, &p[2][0], &p[2][1], &p[2][2]);
  m_bl_to_ks(r, th - eth, ph, a, &p[3][0], &p[3][1], &p[3][2]);
  m_bl_to_ks(r, th, ph + eph, a, &p[4][0], &p[4][1], &p[4][2]);
  m_bl_to_ks(r, th, ph - eph, a, &p[5][0], &p[5][1], &p[5][2]);
  for (int i = 0; i < 3; ++i) {
    J[i][0] = (p[0][i] - p[1][i]) / (2.0 * er);
    J[i][1] = (p[2][i] - p[3][i]) / (2.0 * eth);
    J[i][2] = (p[4][i] - p[5][i]) / (2.0 * eph);
  }
}

static int init_ks_state(const Frame* f, const Geo* sb, KS* k) {
  const Metric* g = &f->g;
  if (fabs(g->L) > 1e-15) return 0;
  m_bl_to_ks(sb->r, sb->th, sb->ph, g->a, &k->X, &k->Y, &k->Z);
  double J[3][3], A3[3][3];
  jacobian_bl_to_ks(sb->r, sb->th, sb->ph, g->a, J);
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) A3[j][i] = J[i][j];
  const double b3[3] = {sb->pr, sb->pth, sb->pphi};
  double x3[3];
  if (!solve_3x3(A3, b3, x3)) return 0;
  k->pX = x3[0];
  k->pY = x3[1];
  k->pZ = x3[2];
  double U[4][4];
  m_con_ks(g, k->X, k->Y, k->Z, U);
  const double A = U[0][0];
  const double B = 2.0 * ((U[0][1] * k->pX + U[0][2] * k->pY) + U[0][3] * k->pZ);
  const double C = (((((U[1][1] * k->pX) * k->pX + (U[2][2] * k->pY) * k->pY) + (U[3][3] * k->pZ) * k->pZ) +
                     ((2.0 * U[1][2]) * k->pX) * k->pY) +
                    ((2.0 * U[1][3]) * k->pX) * k->pZ) +
                   ((2.0 * U[2][3]) * k->pY) * k->pZ;
  const double disc = B * B - (4.0 * A) * C;
  if (disc < 0.0 || fabs(A) < 1e-15) return 0;
  const double sq = sqrt(disc);
  const double pT1 = (-B - sq) / (2.0 * A);
  const double pT2 = (-B + sq) / (2.0 * A);
  k->pT = (pT1 < 0.0) ? pT1 : pT2;
  if (k->pT > 0.0) k->pT = omin(pT1, pT2);
  return oisfinite(k->pT);
}

static void rhs_ks(const Metric* g, const KS* s, double d[6]) {
  double U[4][4];
  m_con_ks(g, s->X, s->Y, s->Z, U);
  d[0] = ((U[1][0] * s->pT + U[1][1] * s->pX) + U[1][2] * s->pY) + U[1][3] * s->pZ;
  d[1] = ((U[2][0] * s->pT + U[2][1] * s->pX) + U[2][2] * s->pY) + U[2][3] * s->pZ;
  d[2] = ((U[3][0] * s->pT + U[3][1] * s->pX) + U[3][2] * s->pY) + U[3][3] * s->pZ;
  const double p[4] = {s->pT, s->pX, s->pY, s->pZ};
  const double eX = 1e-5 * (fabs(s->X) + 0.1);
  const double eY = 1e-5 * (fabs(s->Y) + 0.1);
  const double eZ = 1e-5 * (fabs(s->Z) + 0.1);
  d[3] = -(m_ham_ks(g, s->X + eX, s->Y, s->Z, p) - m_ham_ks(g, s->X - eX, s->Y, s->Z, p)) / (2.0 * eX);
  d[4] = -(m_ham_ks(g, s->X, s->Y + eY, s->Z, p) - m_ham_ks(g, s->X, s->Y - eY, s->Z, p)) / (2.0 * eY);
  d[5] = -(m_ham_ks(g, s->X, s->Y, s->Z + eZ, p) - m_ham_ks(g, s->X, s->Y, s->Z - eZ, p)) / (2.0 * eZ);
}

static KS ks_axpy(const KS* s0, double f, const double d[6]) {
  KS s = {s0->X + f * d[0], s0->Y + f * d[1], s0->Z + f * d[2],
          s0->pX + f * d[3], s0->pY + f * d[4], s0->pZ + f * d[5], s0->pT};
  return s;
}

static void rk4_step_ks(const Metric* g, KS* s, double dlam) {
  double k1[6], k2[6], k3[6], k4[6];
  const KS s0 = *s;
  rhs_ks(g, &s0, k1);
  const KS s2 = ks_axpy(&s0, 0.5 * dlam, k1);
  rhs_ks(g, &s2, k2);
  const KS s3 = ks_axpy(&s0, 0.5 * dlam, k2);
  rhs_ks(g, &s3, k3);
  const KS s4 = ks_axpy(&s0, dlam, k3);
  rhs_ks(g, &s4, k4);
  const double w = dlam / 6.0;
  double* v[6] = {&s->X, &s->Y, &s->Z, &s->pX, &s->pY, &s->pZ};
  for (int i = 0; i < 6; ++i) *v[i] += w * (((k1[i] + 2.0 * k2[i]) + 2.0 * k3[i]) + k4[i]);
}

static int rk4_adaptive_ks(const Metric* g, KS* s, double* dlam, double tol) {
  const KS s0 = *s;
  KS sA = s0;
  rk4_step_ks(g, &sA, *dlam);
  KS sB = s0;
  rk4_step_ks(g, &sB, 0.5 * *dlam);
  rk4_step_ks(g, &sB, 0.5 * *dlam);
  const double e0 = sA.X - sB.X, e1 = sA.Y - sB.Y, e2 = sA.Z - sB.Z;
  const double e3 = sA.pX - sB.pX, e4 = sA.pY - sB.pY, e5 = sA.pZ - sB.pZ;
  const double err = sqrt(((((e0 * e0 + e1 * e1) + e2 * e2) + e3 * e3) + e4 * e4) + e5 * e5) / 15.0;
  const int acc = doubling_update(err, tol, dlam);
  *s = (acc == 1) ? sB : s0;
  return acc == 1;
}

static void ks_covector_to_bl(double r, double th, double ph, double a, double pX, double pY,
                              double pZ, double pbl[3]) {
  double J[3][3];
  jacobian_bl_to_ks(r, th, ph, a, J);
  const double pxyz[3] = {pX, pY, pZ};
  for (int j = 0; j < 3; ++j) {
    pbl[j] = 0.0;
    for (int i = 0; i < 3; ++i) pbl[j] += J[i][j] * pxyz[i];
  }
}

static Ray trace_single_ks(const Frame* f, const Geo* sbl) {
  const Metric* g = &f->g;
  KS s;
  if (!init_ks_state(f, sbl, &s)) return trace_single(f, *sbl);
  const double rh_cut = f->rh * 1.03;
  double dlam = omax(f->step_init, 1e-10);
  double prev_r = m_r_ks(s.X, s.Y, s.Z, g->a);
  const int max_steps = f->max_steps < 1 ? 1 : f->max_steps;
  uint32_t att = 0;
  for (int it = 0; it < max_steps; ++it) {
    const KS sp = s;
    double step_used = dlam;
    int rejects = 0;
    for (;;) {
      step_used = dlam;
      ++att;
      if (rk4_adaptive_ks(g, &s, &dlam, f->tol)) break;
      if (!oisfinite(dlam) || ++rejects > 64) {
        double rt, tt, pt;
        m_ks_to_bl(s.X, s.Y, s.Z, g->a, &rt, &tt, &pt);
        Ray o = ray_result(KT_OUT_ESCAPED, rt, 1.0, tt, pt, 0.0);
        o.steps = (uint32_t)it;
        o.attempts = att;
        return o;
      }
    }
    const double r_now = m_r_ks(s.X, s.Y, s.Z, g->a);
    double best_alpha = 2.0;
    int ev = EV_NONE;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    if (sign_change(sp.Z, s.Z) || (omin(fabs(sp.Z), fabs(s.Z)) < 0.35)) {
      double d0[6], d1[6];
      rhs_ks(g, &sp, d0);
      rhs_ks(g, &s, d1);
      double alpha = 0.0;
      int hit = first_event(sp.Z, s.Z, d0[2], d1[2], step_used, 0.0, &alpha);
      if (!hit && sign_change(sp.Z, s.Z)) {
        const double denom = sp.Z - s.Z;
        alpha = (fabs(denom) > 1e-12) ? (sp.Z / denom) : 0.5;
        alpha = oclamp(alpha, 0.0, 1.0);
        hit = 1;
      }
      if (hit) {
        const double Xh = hermite(sp.X, s.X, d0[0], d1[0], step_used, alpha);
        const double Yh = hermite(sp.Y, s.Y, d0[1], d1[1], step_used, alpha);
        const double Zh = hermite(sp.Z, s.Z, d0[2], d1[2], step_used, alpha);
        const double pXh = hermite(sp.pX, s.pX, d0[3], d1[3], step_used, alpha);
        const double pYh = hermite(sp.pY, s.pY, d0[4], d1[4], step_used, alpha);
        const double pZh = hermite(sp.pZ, s.pZ, d0[5], d1[5], step_used, alpha);
        const double pTh = sp.pT;
        double r_hit, th_hit, ph_hit;
        m_ks_to_bl(Xh, Yh, Zh, g->a, &r_hit, &th_hit, &ph_hit);
        if (r_hit >= f->r_in && r_hit <= f->r_out) {
          double pbl[3];
          ks_covector_to_bl(r_hit, th_hit, ph_hit, g->a, pXh, pYh, pZh, pbl);
          disk_r = r_hit;
          disk_red = oclamp(disk_redshift(g, r_hit, pTh, pbl[2]), 0.0, 20.0);
          disk_phi = ph_hit;
          best_alpha = alpha;
          ev = EV_DISK;
        }
      }
    }
    if (r_now <= rh_cut) {
      const double denom_h = prev_r - r_now;
      double alpha_h = (fabs(denom_h) > 1e-12) ? ((prev_r - rh_cut) / denom_h) : 0.0;
      alpha_h = oclamp(alpha_h, 0.0, 1.0);
      if (alpha_h < best_alpha) {
        best_alpha = alpha_h;
        ev = EV_HORIZON;
      }
    }
    if (r_now >= f->r_esc) {
      const double denom_e = r_now - prev_r;
      double alpha_e = (fabs(denom_e) > 1e-12) ? ((f->r_esc - prev_r) / denom_e) : 1.0;
      alpha_e = oclamp(alpha_e, 0.0, 1.0);
      if (alpha_e < best_alpha) {
        best_alpha = alpha_e;
        ev = EV_ESCAPE;
      }
    }
    if (ev != EV_NONE) {
      Ray o;
      if (ev == EV_DISK) {
        o = ray_result(KT_OUT_DISK, disk_r, disk_red, disk_phi, 0.0, 0.0);
      } else if (ev == EV_HORIZON) {
        o = ray_result(KT_OUT_HORIZON, prev_r + best_alpha * (r_now - prev_r), 0.0, 0.0, 0.0, 0.0);
      } else {
        const double Xe = sp.X + best_alpha * (s.X - sp.X);
        const double Ye = sp.Y + best_alpha * (s.Y - sp.Y);
        const double Ze = sp.Z + best_alpha * (s.Z - sp.Z);
        double re, te, pe;
        m_ks_to_bl(Xe, Ye, Ze, g->a, &re, &te, &pe);
        o = ray_result(KT_OUT_ESCAPED, re, 1.0, te, pe, 0.0);
      }
      o.steps = (uint32_t)it + 1;
      o.attempts = att;
      return o;
    }
    prev_r = r_now;
  }
  double re, te, pe;
  m_ks_to_bl(s.X, s.Y, s.Z, g->a, &re, &te, &pe);
  Ray o = ray_result(KT_OUT_ESCAPED, re, 1.0, te, pe, 0.0);
  o.steps = (uint32_t)max_steps;
  o.attempts = att;
  return o;
}

/* ------------------------------------------------------ elliptic-closed
 * trace_single_elliptic_closed (main.cpp:705-1295): for a Kerr ray, the
 * Mino time of its first equator crossing (closed form, Jacobi cn) and its
 * radius there from the roots of the radial quartic (Jacobi inversion in
 * one of three root configurations), Carlson R_F for the elliptic
 * integrals.  Only a crossing inside the disk is used, and only when the
 * standard tracer of the frame's chart does not end the ray at the horizon;
 * every other ray is the standard tracer's.  Complex products and quotients
 * by the textbook formulas (the reference's -ffast-math arithmetic), |z| by
 * hypot. */
typedef struct { double re, im; } Cx;
static Cx cx(double re, double im) { Cx z = {re, im}; return z; }
static Cx cx_add(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
static Cx cx_sub(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
static Cx cx_mul(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static Cx cx_div(Cx a, Cx b) {
  const double t = b.re * b.re + b.im * b.im;
  return cx((a.re * b.re + a.im * b.im) / t, (a.im * b.re - a.re * b.im) / t);
}
static double cx_abs(Cx a) { return ktm_hypot(a.re, a.im); }

/* carlson_rf, main.cpp:706-742 */
static double carlson_rf(double x, double y, double z) {
  if (!(x >= 0.0 && y >= 0.0 && z >= 0.0)) return ktm_nan();
  if (!oisfinite(x) || !oisfinite(y) || !oisfinite(z)) return ktm_nan();
  double xn = x, yn = y, zn = z;
  for (int it = 0; it < 64; ++it) {
    const double mu = ((xn + yn) + zn) / 3.0;
    if (!(mu > 0.0) || !oisfinite(mu)) return ktm_nan();
    const double X = 1.0 - xn / mu, Y = 1.0 - yn / mu, Z = 1.0 - zn / mu;
    const double eps = omax(omax(fabs(X), fabs(Y)), fabs(Z));
    if (eps < 1e-10) {
      const double E2 = X * Y - Z * Z;
      const double E3 = (X * Y) * Z;
      const double corr = (((1.0 - E2 / 10.0) + E3 / 14.0) + (E2 * E2) / 24.0) - ((3.0 * E2) * E3) / 44.0;
      return corr / sqrt(mu);
    }
    const double sx = sqrt(xn), sy = sqrt(yn), sz = sqrt(zn);
    const double lam = (sx * sy + sx * sz) + sy * sz;
    xn = 0.25 * (xn + lam);
    yn = 0.25 * (yn + lam);
    zn = 0.25 * (zn + lam);
  }
  return ktm_nan();
}

/* ellint_F_incomplete, ellint_K_complete (main.cpp:744-757) */
static double ell_F(double phi, double m) {
  const double sn = ktm_sin(phi), cs = ktm_cos(phi);
  const double x = cs * cs;
  const double y = 1.0 - (m * sn) * sn;
  if (y <= 0.0) return ktm_nan();
  return sn * carlson_rf(x, y, 1.0);
}

static double ell_K(double m) {
  if (!(m >= 0.0 && m < 1.0)) return ktm_nan();
  return carlson_rf(0.0, 1.0 - m, 1.0);
}

/* jacobi_sn2_from_u, main.cpp:759-777 */
static double jac_sn2(double u, double m, double Kc) {
  if (!(m >= 0.0 && m < 1.0) || !(Kc > 0.0) || !oisfinite(u)) return ktm_nan();
  double ur = fmod(u, 2.0 * Kc);
  if (ur < 0.0) ur += 2.0 * Kc;
  if (ur > Kc) ur = 2.0 * Kc - ur;
  double lo = 0.0, hi = 0.5 * ORC_PI;
  for (int it = 0; it < 64; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double Fm = ell_F(mid, m);
    if (!oisfinite(Fm)) return ktm_nan();
    if (Fm < ur)
      lo = mid;
    else
      hi = mid;
  }
  const double sn = ktm_sin(0.5 * (lo + hi));
  return sn * sn;
}

/* quartic_roots_monic_complex (main.cpp:779-812): Durand-Kerner from four
 * points on the circle of radius 1 + max |b_i|. */
static void quartic_roots(const double b[4], Cx z[4]) {
  double rad = fabs(b[0]);
  for (int i = 1; i < 4; ++i) rad = omax(rad, fabs(b[i]));
  rad = 1.0 + rad;
  const double PI_ = 3.141592653589793238462643383279502884;
  for (int i = 0; i < 4; ++i) {
    const double a = (0.5 * (double)i) * PI_;
    z[i] = cx(rad * ktm_cos(a), rad * ktm_sin(a));
  }
  for (int it = 0; it < 160; ++it) {
    double max_delta = 0.0;
    Cx zn[4];
    for (int i = 0; i < 4; ++i) {
      Cx den = cx(1.0, 0.0);
      for (int j = 0; j < 4; ++j)
        if (i != j) den = cx_mul(den, cx_sub(z[i], z[j]));
      if (cx_abs(den) < 1e-20) den = cx(1e-20, 0.0);
      /* (((z + b0) z + b1) z + b2) z + b3 */
      Cx p = cx_add(z[i], cx(b[0], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[1], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[2], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[3], 0.0));
      const Cx delta = cx_div(p, den);
      zn[i] = cx_sub(z[i], delta);
      max_delta = omax(max_delta, cx_abs(delta));
    }
    for (int i = 0; i < 4; ++i) z[i] = zn[i];
    if (max_delta < 1e-13) break;
  }
}

/* jacobi_sn_cn_from_u, main.cpp:834-876 */
static int jac_sn_cn(double u, double m, double Kc, double* sn, double* cn) {
  *sn = *cn = ktm_nan();
  if (!(m >= 0.0 && m < 1.0) || !(Kc > 0.0) || !oisfinite(u)) return 0;
  const double twoK = 2.0 * Kc;
  long long n = (long long)floor(u / twoK);
  double ur = u - (double)n * twoK;
  if (ur < 0.0) {
    ur += twoK;
    --n;
  }
  const int second = ur > Kc;
  const double target = second ? (twoK - ur) : ur;
  double lo = 0.0, hi = 0.5 * ORC_PI;
  for (int it = 0; it < 72; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double Fm = ell_F(mid, m);
    if (!oisfinite(Fm)) return 0;
    if (Fm < target)
      lo = mid;
    else
      hi = mid;
  }
  const double amp = 0.5 * (lo + hi);
  double s_ = ktm_sin(amp), c_ = ktm_cos(amp);
  if (second) c_ = -c_;
  if ((n & 1LL) != 0) {
    s_ = -s_;
    c_ = -c_;
  }
  *sn = s_;
  *cn = c_;
  return oisfinite(s_) && oisfinite(c_);
}

/* jacobi_sc_from_u, main.cpp:878-885 */
static int jac_sc(double u, double m, double Kc, double* sc) {
  double sn, cn;
  *sc = ktm_nan();
  if (!jac_sn_cn(u, m, Kc, &sn, &cn)) return 0;
  if (fabs(cn) < 1e-14) return 0;
  *sc = sn / cn;
  return oisfinite(*sc);
}

enum { RAD_REAL4 = 0, RAD_REAL2 = 1, RAD_COMPLEX4 = 2 };
typedef struct {
  int kind;
  double r1, r2, r3, r4;
  double m, Kc, omega, X0;
  int phase_sign, tau_sign;
  double A, B, r_lo, r_hi;
  double a2, b1, g0;
} RadMap; /* EllipticRadialMap, main.cpp:893-916 */

/* elliptic_radial_r_from_phase, main.cpp:918-956 */
static double rad_r(const RadMap* mp, double X) {
  if (mp->kind == RAD_REAL4) {
    const double sn2 = jac_sn2(X, mp->m, mp->Kc);
    if (!oisfinite(sn2)) return ktm_nan();
    const double r24 = mp->r2 - mp->r4, r14 = mp->r1 - mp->r4;
    const double den = r24 - r14 * sn2;
    if (fabs(den) < 1e-14) return ktm_nan();
    return (mp->r1 * r24 - (mp->r2 * r14) * sn2) / den;
  }
  if (mp->kind == RAD_REAL2) {
    double sn, cn;
    if (!jac_sn_cn(X, mp->m, mp->Kc, &sn, &cn)) return ktm_nan();
    const double num = (mp->B * mp->r_hi - mp->A * mp->r_lo) + (mp->B * mp->r_hi + mp->A * mp->r_lo) * cn;
    const double den = (mp->B - mp->A) + (mp->B + mp->A) * cn;
    if (fabs(den) < 1e-14) return ktm_nan();
    return num / den;
  }
  double sc;
  if (!jac_sc(X, mp->m, mp->Kc, &sc)) return ktm_nan();
  const double den = 1.0 + mp->g0 * sc;
  if (fabs(den) < 1e-14) return ktm_nan();
  return -mp->a2 * ((mp->g0 - sc) / den) - mp->b1;
}

/* align_initial_radial_sign (main.cpp:981-1000) */
static void rad_align(RadMap* mp, double dr0, int flip_phase, int flip_tau) {
  if (fabs(dr0) < 1e-14) return;
  const double probe = 1e-6;
  const double Xp = (double)mp->phase_sign * mp->X0 + ((double)mp->tau_sign * mp->omega) * probe;
  const double Xm = (double)mp->phase_sign * mp->X0 - ((double)mp->tau_sign * mp->omega) * probe;
  const double rp = rad_r(mp, Xp), rm = rad_r(mp, Xm);
  if (!oisfinite(rp) || !oisfinite(rm)) return;
  if ((dr0 >= 0.0) == (rp >= rm)) return;
  if (flip_phase) mp->phase_sign = -mp->phase_sign;
  if (flip_tau) mp->tau_sign = -mp->tau_sign;
}

static void sort_desc(double* v, int n) {
  for (int i = 1; i < n; ++i)
    for (int j = i; j > 0 && v[j] > v[j - 1]; --j) {
      const double t = v[j];
      v[j] = v[j - 1];
      v[j - 1] = t;
    }
}

/* init_elliptic_radial_map, main.cpp:958-1168 */
static int rad_init(const SepC* c, double r0, double dr0, RadMap* out) {
  const double u = c->Lz - c->a * c->E;
  const double Kpot = c->Qc + u * u;
  const double A0 = (c->E * c->a) * c->a - c->a * c->Lz;
  const double c4 = c->E * c->E;
  if (!(c4 > 1e-18)) return 0;
  const double c2 = (2.0 * c->E) * A0 - Kpot;
  const double c1 = (2.0 * c->M) * Kpot;
  const double c0 = A0 * A0 - (c->a * c->a) * Kpot;
  const double b[4] = {0.0, c2 / c4, c1 / c4, c0 / c4};
  Cx z[4];
  quartic_roots(b, z);
  double rr[4];
  Cx cr[4];
  int nr = 0, nc = 0;
  for (int i = 0; i < 4; ++i) {
    if (!oisfinite(z[i].re) || !oisfinite(z[i].im)) return 0;
    const double tol = 1e-7 * omax(1.0, fabs(z[i].re));
    if (fabs(z[i].im) <= tol)
      rr[nr++] = z[i].re;
    else
      cr[nc++] = z[i];
  }
  memset(out, 0, sizeof *out);
  out->phase_sign = out->tau_sign = 1;
  if (nr == 4) {
    sort_desc(rr, 4);
    out->kind = RAD_REAL4;
    out->r1 = rr[0];
    out->r2 = rr[1];
    out->r3 = rr[2];
    out->r4 = rr[3];
    const double den_omega = (out->r1 - out->r3) * (out->r2 - out->r4);
    if (!(den_omega > 0.0)) return 0;
    out->omega = 0.5 * sqrt(den_omega);
    const double k_num = (out->r2 - out->r3) * (out->r1 - out->r4);
    const double k_den = (out->r2 - out->r4) * (out->r1 - out->r3);
    if (!(k_den > 0.0)) return 0;
    out->m = k_num / k_den;
    if (!(out->m >= 0.0 && out->m < 1.0)) return 0;
    out->Kc = ell_K(out->m);
    if (!oisfinite(out->Kc) || !(out->Kc > 0.0)) return 0;
    const double den_obs = r0 - out->r2, den_root = out->r1 - out->r4;
    if (fabs(den_obs) < 1e-14 || fabs(den_root) < 1e-14) return 0;
    const double u0_raw = ((r0 - out->r1) / den_obs) * ((out->r2 - out->r4) / den_root);
    if (!oisfinite(u0_raw)) return 0;
    if (u0_raw < -1e-6 || u0_raw > 1.0 + 1e-6) return 0;
    const double u0 = oclamp(u0_raw, 0.0, 1.0);
    out->X0 = ell_F(ktm_asin(sqrt(u0)), out->m);
    if (!oisfinite(out->X0)) return 0;
    const int case1 = (r0 >= out->r3 && r0 <= out->r2);
    const int alpha = case1 ? -1 : 1;
    const int nu_r = (dr0 >= 0.0) ? 1 : -1;
    out->phase_sign = alpha * nu_r;
    out->tau_sign = 1;
    rad_align(out, dr0, 1, 0);
    return 1;
  }
  if (nr == 2 && nc == 2) {
    const double r1 = omin(rr[0], rr[1]), r2 = omax(rr[0], rr[1]); /* ascending */
    const double b1 = 0.5 * (cr[0].re + cr[1].re);
    const double a1 = 0.5 * (fabs(cr[0].im) + fabs(cr[1].im));
    if (!(a1 > 0.0) || !oisfinite(a1) || !oisfinite(b1)) return 0;
    const double A = sqrt(a1 * a1 + (b1 - r2) * (b1 - r2));
    const double B = sqrt(a1 * a1 + (b1 - r1) * (b1 - r1));
    if (!(A > 0.0 && B > 0.0 && B > A)) return 0;
    const double r21 = r2 - r1;
    const double k3 = (((A + B) * (A + B)) - r21 * r21) / ((4.0 * A) * B);
    if (!(k3 > 0.0 && k3 < 1.0)) return 0;
    const double K3 = ell_K(k3);
    if (!oisfinite(K3) || !(K3 > 0.0)) return 0;
    const double x3 = (A * (r0 - r1) - B * (r0 - r2)) / (A * (r0 - r1) + B * (r0 - r2));
    if (!oisfinite(x3)) return 0;
    const double phi0 = ktm_acos(oclamp(x3, -1.0, 1.0));
    const double F0 = ell_F(phi0, k3);
    if (!oisfinite(F0)) return 0;
    out->kind = RAD_REAL2;
    out->r1 = r2;
    out->r2 = r1;
    out->r_lo = r1;
    out->r_hi = r2;
    out->A = A;
    out->B = B;
    out->m = k3;
    out->Kc = K3;
    out->omega = sqrt(A * B);
    out->X0 = F0;
    out->phase_sign = (dr0 >= 0.0) ? 1 : -1;
    out->tau_sign = 1;
    rad_align(out, dr0, 1, 0);
    return 1;
  }
  if (nr == 0 && nc == 4) {
    Cx pos[4], neg[4];
    int np = 0, nn = 0;
    for (int i = 0; i < 4; ++i) {
      if (cr[i].im >= 0.0) {
        if (np < 4) pos[np] = cr[i];
        ++np;
      } else {
        if (nn < 4) neg[nn] = cr[i];
        ++nn;
      }
    }
    if (np != 2 || nn != 2) return 0;
    const double d00 = cx_abs(cx_sub(pos[0], cx(neg[0].re, -neg[0].im)));
    const double d01 = cx_abs(cx_sub(pos[0], cx(neg[1].re, -neg[1].im)));
    const int j0 = (d00 <= d01) ? 0 : 1;
    const double bA = 0.5 * (pos[0].re + neg[j0].re);
    const double aA = 0.5 * (fabs(pos[0].im) + fabs(neg[j0].im));
    const double bB = 0.5 * (pos[1].re + neg[1 - j0].re);
    const double aB = 0.5 * (fabs(pos[1].im) + fabs(neg[1 - j0].im));
    if (!(aA > 0.0 && aB > 0.0)) return 0;
    double b1 = bA, a1 = aA, b2 = bB, a2 = aB;
    if (bB > bA) {
      b1 = bB;
      a1 = aB;
      b2 = bA;
      a2 = aA;
    }
    if (!(b1 > b2)) return 0;
    const double C = sqrt((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2));
    const double D = sqrt((a1 + a2) * (a1 + a2) + (b1 - b2) * (b1 - b2));
    if (!(C > 0.0 && D > 0.0)) return 0;
    const double k4 = ((4.0 * C) * D) / ((C + D) * (C + D));
    if (!(k4 > 0.0 && k4 < 1.0)) return 0;
    const double K4 = ell_K(k4);
    if (!oisfinite(K4) || !(K4 > 0.0)) return 0;
    const double g_num = (4.0 * a2) * a2 - (C - D) * (C - D);
    const double g_den = (C + D) * (C + D) - (4.0 * a2) * a2;
    if (!(g_num > 0.0 && g_den > 0.0)) return 0;
    const double g0 = sqrt(g_num / g_den);
    if (!(g0 > 0.0) || !oisfinite(g0)) return 0;
    const double x4 = (r0 - b2) / omax(a2, 1e-15);
    const double phi0 = ktm_atan(x4) + ktm_atan(g0);
    const double F0 = ell_F(phi0, k4);
    if (!oisfinite(F0)) return 0;
    out->kind = RAD_COMPLEX4;
    out->m = k4;
    out->Kc = K4;
    out->omega = 0.5 * (C + D);
    out->X0 = F0;
    out->phase_sign = 1;
    out->tau_sign = (dr0 >= 0.0) ? 1 : -1;
    out->a2 = a2;
    out->b1 = b1;
    out->g0 = g0;
    rad_align(out, dr0, 0, 1);
    return 1;
  }
  return 0;
}

/* separable_radial_potential, main.cpp:1170-1176 */
static double sep_Rpot(const SepC* c, double r) {
  const double u = c->Lz - c->a * c->E;
  const double Kpot = c->Qc + u * u;
  const double A0 = c->E * (r * r + c->a * c->a) - c->a * c->Lz;
  const double Delta = (r * r - (2.0 * c->M) * r) + c->a * c->a;
  return A0 * A0 - Delta * Kpot;
}

/* first_equator_crossing_mino_time, main.cpp:1178-1219 */
static int eq_crossing(const SepC* c, double th0, double dth0, double* tau_first) {
  const double A = ((c->a * c->a) * c->E) * c->E;
  if (!(A > 1e-15)) return 0;
  const double B = (A - c->Lz * c->Lz) - c->Qc;
  const double disc = B * B + (4.0 * A) * c->Qc;
  if (!(disc >= 0.0)) return 0;
  const double sq = sqrt(disc);
  const double up = (B + sq) / (2.0 * A), um = (B - sq) / (2.0 * A);
  if (!(up > 0.0 && um < 0.0)) return 0;
  const double m = up / (up - um);
  if (!(m >= 0.0 && m < 1.0)) return 0;
  const double Kc = ell_K(m);
  if (!oisfinite(Kc) || !(Kc > 0.0)) return 0;
  const double omega = sqrt(A * (up - um));
  if (!(omega > 0.0) || !oisfinite(omega)) return 0;
  const double mu_plus = sqrt(up);
  const double mu0 = ktm_cos(th0);
  const double c0 = oclamp(fabs(mu0) / omax(mu_plus, 1e-15), 0.0, 1.0);
  const double phi0 = ktm_acos(c0);
  const double u_base = ell_F(phi0, m);
  if (!oisfinite(u_base)) return 0;
  const double tau_period = (4.0 * Kc) / omega;
  if (!(tau_period > 0.0) || !oisfinite(tau_period)) return 0;
  const int toward = (ktm_cos(th0) * dth0) > 0.0;
  const double u0 = toward ? u_base : -u_base;
  double tf = (Kc - u0) / omega;
  if (tf < 0.0) tf += tau_period;
  *tau_first = tf;
  return oisfinite(tf);
}

/* EllipticFallbackReason (main.cpp:178-186) */
enum { EF_NONE = 0, EF_INIT = 1, EF_THETA = 2, EF_RADIAL_INIT = 3, EF_RADIAL_INVALID = 4,
       EF_OUTSIDE_DISK = 5 };

/* The closed-form part of trace_single_elliptic_closed: 1 with (r, g) of a
 * disk crossing (to be used unless the standard tracer ends the ray at the
 * horizon), else 0 with the fallback reason. */
static int elliptic_closed_form(const Frame* f, const Geo* sbl, double* r_out, double* g_out, int* reason) {
  SepC c;
  if (!sep_init(sbl, &f->g, &c)) {
    *reason = EF_INIT;
    return 0;
  }
  double dr0, dth0, dpr0, dpth0;
  geo_rhs(&f->g, sbl->r, sbl->th, sbl->pr, sbl->pth, sbl->pt, sbl->pphi, &dr0, &dth0, &dpr0, &dpth0);
  double tau_first = 0.0;
  if (!eq_crossing(&c, sbl->th, dth0, &tau_first)) {
    *reason = EF_THETA;
    return 0;
  }
  RadMap mp;
  if (!rad_init(&c, sbl->r, dr0, &mp)) {
    *reason = EF_RADIAL_INIT;
    return 0;
  }
  const double rh_cut = f->rh * 1.03;
  const double X = (double)mp.phase_sign * mp.X0 + ((double)mp.tau_sign * mp.omega) * tau_first;
  const double r_now = rad_r(&mp, X);
  if (!oisfinite(r_now)) {
    *reason = EF_RADIAL_INVALID;
    return 0;
  }
  const double R = sep_Rpot(&c, r_now);
  const double R_scale = omax(1.0, fabs(((((c.E * c.E) * r_now) * r_now) * r_now) * r_now));
  if (R < -1e-8 * R_scale || (mp.kind != RAD_COMPLEX4 && r_now < mp.r1) || r_now < rh_cut) {
    *reason = EF_RADIAL_INVALID;
    return 0;
  }
  if (r_now > f->r_esc || !(r_now >= f->r_in && r_now <= f->r_out)) {
    *reason = EF_OUTSIDE_DISK;
    return 0;
  }
  *reason = EF_NONE;
  *r_out = r_now;
  *g_out = oclamp(disk_redshift(&f->g, r_now, sbl->pt, sbl->pphi), 0.0, 20.0);
  return 1;
}

static Ray trace_standard(const Frame* f, const Geo* sbl) {
  return (f->chart == KT_CHART_KS) ? trace_single_ks(f, sbl) : trace_single(f, *sbl);
}

/* trace_single_elliptic_closed, main.cpp:1227-1295 */
static Ray trace_elliptic(const Frame* f, const Geo* sbl, int* reason) {
  double r, g;
  const Ray std_ray = trace_standard(f, sbl);
  if (!elliptic_closed_form(f, sbl, &r, &g, reason)) return std_ray;
  if (std_ray.outcome == KT_OUT_HORIZON) return std_ray; /* horizon precedence */
  Ray o = ray_result(KT_OUT_DISK, r, g, 0.0, 0.0, 0.0);
  o.steps = std_ray.steps;
  o.attempts = std_ray.attempts;
  return o;
}

/* ------------------------------------------------------------- ray bundles
 * ray_bundle.hpp:56-436 */
static void hessian_H(const Metric* g, double r, double th, double pr, double pth, double pt,
                      double pphi, double Hs[4][4]) {
  const double e[4] = {1e-5 * (fabs(r) + 0.1), 1e-5, 1e-5 * (fabs(pr) + 1e-3),
                       1e-5 * (fabs(pth) + 1e-3)};
#define EVAL(d0, d1, d2, d3) m_ham(g, r + (d0), th + (d1), pr + (d2), pth + (d3), pt, pphi)
  const double H0 = EVAL(0.0, 0.0, 0.0, 0.0);
  double vp[4], vm[4];
  vp[0] = EVAL(e[0], 0.0, 0.0, 0.0);
  vm[0] = EVAL(-e[0], 0.0, 0.0, 0.0);
  vp[1] = EVAL(0.0, e[1], 0.0, 0.0);
  vm[1] = EVAL(0.0, -e[1], 0.0, 0.0);
  vp[2] = EVAL(0.0, 0.0, e[2], 0.0);
  vm[2] = EVAL(0.0, 0.0, -e[2], 0.0);
  vp[3] = EVAL(0.0, 0.0, 0.0, e[3]);
  vm[3] = EVAL(0.0, 0.0, 0.0, -e[3]);
  for (int a = 0; a < 4; ++a) Hs[a][a] = ((vp[a] - 2.0 * H0) + vm[a]) / (e[a] * e[a]);
  for (int a = 0; a < 4; ++a) {
    for (int b = a + 1; b < 4; ++b) {
      double da[4] = {0.0, 0.0, 0.0, 0.0}, db[4] = {0.0, 0.0, 0.0, 0.0};
      da[a] = e[a];
      db[b] = e[b];
      const double pp = EVAL(da[0] + db[0], da[1] + db[1], da[2] + db[2], da[3] + db[3]);
      const double pm = EVAL(da[0] - db[0], da[1] - db[1], da[2] - db[2], da[3] - db[3]);
      const double mp = EVAL(-da[0] + db[0], -da[1] + db[1], -da[2] + db[2], -da[3] + db[3]);
      const double mm = EVAL(-da[0] - db[0], -da[1] - db[1], -da[2] - db[2], -da[3] - db[3]);
      Hs[a][b] = Hs[b][a] = (((pp - pm) - mp) + mm) / ((4.0 * e[a]) * e[b]);
    }
  }
#undef EVAL
}

typedef struct {
  Geo geo;
  double W[4][2];
} Bundle;

static void bundle_rhs(const Metric* g, const Geo* s, const double W[4][2], double dz[4],
                       double dW[4][2]) {
  geo_rhs(g, s->r, s->th, s->pr, s->pth, s->pt, s->pphi, &dz[0], &dz[1], &dz[2], &dz[3]);
  double Hs[4][4], M[4][4];
  hessian_H(g, s->r, s->th, s->pr, s->pth, s->pt, s->pphi, Hs);
  for (int j = 0; j < 4; ++j) {
    M[0][j] = Hs[2][j];
    M[1][j] = Hs[3][j];
    M[2][j] = -Hs[0][j];
    M[3][j] = -Hs[1][j];
  }
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 2; ++k) {
      dW[i][k] = 0.0;
      for (int j = 0; j < 4; ++j) dW[i][k] += M[i][j] * W[j][k];
    }
}

static void bundle_make(const Geo* s, const double dz[4], double fct, const double W[4][2],
                        const double dW[4][2], Geo* ns, double nW[4][2]) {
  *ns = *s;
  ns->r += fct * dz[0];
  ns->th += fct * dz[1];
  ns->pr += fct * dz[2];
  ns->pth += fct * dz[3];
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 2; ++k) nW[i][k] = W[i][k] + fct * dW[i][k];
}

static void bundle_rk4(const Metric* g, Bundle* bs, double dlam) {
  const Geo s0 = bs->geo;
  double dz1[4], dz2[4], dz3[4], dz4[4], dW1[4][2], dW2[4][2], dW3[4][2], dW4[4][2];
  Geo s2, s3, s4;
  double W2[4][2], W3[4][2], W4[4][2];
  bundle_rhs(g, &s0, bs->W, dz1, dW1);
  bundle_make(&s0, dz1, 0.5 * dlam, bs->W, dW1, &s2, W2);
  bundle_rhs(g, &s2, W2, dz2, dW2);
  bundle_make(&s0, dz2, 0.5 * dlam, bs->W, dW2, &s3, W3);
  bundle_rhs(g, &s3, W3, dz3, dW3);
  bundle_make(&s0, dz3, dlam, bs->W, dW3, &s4, W4);
  bundle_rhs(g, &s4, W4, dz4, dW4);
  const double dp1 = dphi_vel(g, s0.r, s0.th, s0.pt, s0.pphi);
  const double dp2 = dphi_vel(g, s2.r, s2.th, s0.pt, s0.pphi);
  const double dp3 = dphi_vel(g, s3.r, s3.th, s0.pt, s0.pphi);
  const double dp4 = dphi_vel(g, s4.r, s4.th, s0.pt, s0.pphi);
  const double w = dlam / 6.0;
  bs->geo.r += w * (((dz1[0] + 2.0 * dz2[0]) + 2.0 * dz3[0]) + dz4[0]);
  bs->geo.th += w * (((dz1[1] + 2.0 * dz2[1]) + 2.0 * dz3[1]) + dz4[1]);
  bs->geo.pr += w * (((dz1[2] + 2.0 * dz2[2]) + 2.0 * dz3[2]) + dz4[2]);
  bs->geo.pth += w * (((dz1[3] + 2.0 * dz2[3]) + 2.0 * dz3[3]) + dz4[3]);
  bs->geo.ph += w * (((dp1 + 2.0 * dp2) + 2.0 * dp3) + dp4);
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 2; ++k)
      bs->W[i][k] += w * (((dW1[i][k] + 2.0 * dW2[i][k]) + 2.0 * dW3[i][k]) + dW4[i][k]);
}

static int bundle_adaptive(const Metric* g, Bundle* bs, double* dlam, double tol) {
  const Bundle s0 = *bs;
  Bundle sA = s0;
  bundle_rk4(g, &sA, *dlam);
  Bundle sB = s0;
  bundle_rk4(g, &sB, 0.5 * *dlam);
  bundle_rk4(g, &sB, 0.5 * *dlam);
  const double e0 = sA.geo.r - sB.geo.r, e1 = sA.geo.th - sB.geo.th;
  const double e2 = sA.geo.pr - sB.geo.pr, e3 = sA.geo.pth - sB.geo.pth;
  const double err = sqrt(((e0 * e0 + e1 * e1) + e2 * e2) + e3 * e3) / 15.0;
  const int acc = doubling_update(err, tol, dlam);
  *bs = (acc == 1) ? sB : s0;
  return acc == 1;
}

/* BundleResult (ray_bundle.hpp:267-275) -> the pixel record trace_geodesics
 * writes for it (main.cpp:2103-2110). */
static Ray bundle_result(int disk_hit, double r_hit, double red, double magnif, double th_esc,
                         double ph_esc, double phi_disk) {
  Ray o;
  o.outcome = disk_hit ? KT_OUT_DISK : KT_OUT_ESCAPED;
  o.r = disk_hit ? r_hit : 0.0;
  o.redshift = red;
  o.magnif = magnif;
  o.phi_disk = phi_disk;
  o.theta_esc = th_esc;
  o.phi_esc = ph_esc;
  o.steps = o.attempts = 0;
  return o;
}

static Ray trace_bundle(const Frame* f, int px, int py) {
  const Metric* g = &f->g;
  double alpha0, beta0;
  cam_pixel_angles(&f->cam, px, py, f->offx, f->offy, &alpha0, &beta0);
  Bundle bs;
  bs.geo = cam_angle_ray(&f->cam, alpha0, beta0, g);
  {
    const double eps = (f->cam.fov_h / (double)f->cam.W) * 0.5;
    const Geo ap = cam_angle_ray(&f->cam, alpha0 + eps, beta0, g);
    const Geo am = cam_angle_ray(&f->cam, alpha0 - eps, beta0, g);
    const Geo bp = cam_angle_ray(&f->cam, alpha0, beta0 + eps, g);
    const Geo bm = cam_angle_ray(&f->cam, alpha0, beta0 - eps, g);
    bs.W[0][0] = (ap.r - am.r) / (2.0 * eps);
    bs.W[1][0] = (ap.th - am.th) / (2.0 * eps);
    bs.W[2][0] = (ap.pr - am.pr) / (2.0 * eps);
    bs.W[3][0] = (ap.pth - am.pth) / (2.0 * eps);
    bs.W[0][1] = (bp.r - bm.r) / (2.0 * eps);
    bs.W[1][1] = (bp.th - bm.th) / (2.0 * eps);
    bs.W[2][1] = (bp.pr - bm.pr) / (2.0 * eps);
    bs.W[3][1] = (bp.pth - bm.pth) / (2.0 * eps);
  }
  const double rh_cut = f->rh * 1.03;
  double dlam = omax(f->step_init, 1e-10);
  const int max_iter = f->max_steps < 1 ? 1 : f->max_steps;
  uint32_t att = 0;
  for (int iter = 0; iter < max_iter; ++iter) {
    const Bundle bp = bs;
    double step_used = dlam;
    int rejects = 0;
    for (;;) {
      step_used = dlam;
      ++att;
      if (bundle_adaptive(g, &bs, &dlam, f->tol)) break;
      if (!oisfinite(dlam) || ++rejects > 64) {
        Ray o = bundle_result(0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
        o.steps = (uint32_t)iter;
        o.attempts = att;
        return o;
      }
    }
    const double r = bs.geo.r;
    double best_alpha = 2.0;
    int ev = EV_NONE;
    double disk_r = 0.0, disk_red = 1.0, disk_det = 1.0, disk_phi = 0.0;
    const double q0 = bp.geo.th - ORC_PI / 2.0;
    const double q1 = bs.geo.th - ORC_PI / 2.0;
    if (sign_change(q0, q1) || (omin(fabs(q0), fabs(q1)) < 0.35)) {
      double dr0, dth0, dpr0, dpth0, dr1, dth1, dpr1, dpth1;
      geo_rhs(g, bp.geo.r, bp.geo.th, bp.geo.pr, bp.geo.pth, bp.geo.pt, bp.geo.pphi, &dr0, &dth0,
              &dpr0, &dpth0);
      geo_rhs(g, bs.geo.r, bs.geo.th, bs.geo.pr, bs.geo.pth, bs.geo.pt, bs.geo.pphi, &dr1, &dth1,
              &dpr1, &dpth1);
      double alpha = 0.0;
      if (!first_event(bp.geo.th, bs.geo.th, dth0, dth1, step_used, ORC_PI / 2.0, &alpha))
        continue; /* ray_bundle.hpp:352-356: skips this step's horizon/escape tests */
      const double r_hit = hermite(bp.geo.r, bs.geo.r, dr0, dr1, step_used, alpha);
      if (r_hit >= f->r_in && r_hit <= f->r_out) {
        const double Om = m_kepler(g, r_hit);
        const double b = (-bs.geo.pphi) / (-bs.geo.pt);
        double G[4][4];
        m_cov_bl(g, r_hit, ORC_PI / 2.0, G);
        const double d2 = -((G[0][0] + (2.0 * G[0][3]) * Om) + (G[3][3] * Om) * Om);
        const double dv = 1.0 - Om * b;
        double red = (d2 > 0.0 && fabs(dv) > 1e-10) ? sqrt(d2) / dv : 1.0;
        red = red < 0.0 ? 0.0 : red > 20.0 ? 20.0 : red;
        const double J00 = bp.W[0][0] + alpha * (bs.W[0][0] - bp.W[0][0]);
        const double J01 = bp.W[0][1] + alpha * (bs.W[0][1] - bp.W[0][1]);
        const double J10 = bp.W[1][0] + alpha * (bs.W[1][0] - bp.W[1][0]);
        const double J11 = bp.W[1][1] + alpha * (bs.W[1][1] - bp.W[1][1]);
        double det = fabs(J00 * J11 - J01 * J10);
        det = det < 1e-12 ? 1e-12 : det;
        disk_r = r_hit;
        disk_red = red;
        disk_det = det;
        disk_phi = bp.geo.ph + alpha * (bs.geo.ph - bp.geo.ph);
        best_alpha = alpha;
        ev = EV_DISK;
      }
    }
    if (r <= rh_cut) {
      const double denom_h = bp.geo.r - r;
      double alpha_h = (fabs(denom_h) > 1e-12) ? ((bp.geo.r - rh_cut) / denom_h) : 0.0;
      alpha_h = alpha_h < 0.0 ? 0.0 : alpha_h > 1.0 ? 1.0 : alpha_h;
      if (alpha_h < best_alpha) {
        best_alpha = alpha_h;
        ev = EV_HORIZON;
      }
    }
    if (r >= f->r_esc) {
      const double denom_e = r - bp.geo.r;
      double alpha_e = (fabs(denom_e) > 1e-12) ? ((f->r_esc - bp.geo.r) / denom_e) : 1.0;
      alpha_e = alpha_e < 0.0 ? 0.0 : alpha_e > 1.0 ? 1.0 : alpha_e;
      if (alpha_e < best_alpha) {
        best_alpha = alpha_e;
        ev = EV_ESCAPE;
      }
    }
    if (ev == EV_NONE) continue;
    Ray o;
    if (ev == EV_DISK) {
      o = bundle_result(1, disk_r, disk_red, disk_det, 0.0, 0.0, disk_phi);
    } else if (ev == EV_HORIZON) {
      o = bundle_result(0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
    } else {
      const double th_esc = bp.geo.th + best_alpha * (bs.geo.th - bp.geo.th);
      const double ph_esc = bp.geo.ph + best_alpha * (bs.geo.ph - bp.geo.ph);
      o = bundle_result(0, f->r_esc, 1.0, 1.0, th_esc, ph_esc, 0.0);
    }
    o.steps = (uint32_t)iter + 1;
    o.attempts = att;
    return o;
  }
  Ray o = bundle_result(0, bs.geo.r, 1.0, 1.0, 0.0, 0.0, 0.0);
  o.steps = (uint32_t)max_iter;
  o.attempts = att;
  return o;
}

/* --------------------------------------------------------------- frames */

/* trace_geodesics' per-frame rules (main.cpp:2033-2082) and main's clamps
 * of the integrator controls (main.cpp:2683-2686). */
static void setup_frame(const kt_frame_desc* d, Frame* f) {
  f->g.M = d->M;
  f->g.a = d->a;
  f->g.Q = d->Q;
  f->g.L = d->Lambda;
  f->cam.r_obs = d->r_obs;
  f->cam.theta_obs = (d->theta_deg * ORC_PI) / 180.0;
  f->cam.phi_obs = (d->phi_deg * ORC_PI) / 180.0;
  f->cam.fov_h = (d->fov_deg * ORC_PI) / 180.0;
  f->cam.W = d->width;
  f->cam.H = d->height;
  int chart = d->chart;
  if (chart == KT_CHART_KS && fabs(d->Lambda) > 1e-15) chart = KT_CHART_BL;
  if (d->bundles && chart == KT_CHART_KS) chart = KT_CHART_BL;
  f->chart = chart;
  f->intg = d->integrator;
  f->bundles = d->bundles != 0;
  /* select_solver_mode (main.cpp:235-276) on the effective chart */
  f->solver = d->solver_mode;
  if (f->bundles && f->solver != KT_SOLVER_STANDARD) f->solver = KT_SOLVER_STANDARD;
  if (f->solver == KT_SOLVER_SEMI_ANALYTIC &&
      (chart != KT_CHART_BL || fabs(d->Q) > 1e-15 || fabs(d->Lambda) > 1e-15))
    f->solver = KT_SOLVER_STANDARD;
  if (f->solver == KT_SOLVER_ELLIPTIC_CLOSED && (fabs(d->Q) > 1e-15 || fabs(d->Lambda) > 1e-15))
    f->solver = KT_SOLVER_STANDARD;
  f->max_steps = d->max_steps < 1 ? 1 : d->max_steps;
  f->step_init = omax(1e-10, d->step_init);
  f->tol = omax(1e-10, d->tol);
  f->r_in = m_r_isco(&f->g);
  f->r_out = d->disk_out;
  f->r_esc = f->cam.r_obs * 1.05;
  f->rh = m_r_horizon(&f->g);
  f->offx = d->pixel_offset_x;
  f->offy = d->pixel_offset_y;
}

int orc_frame_derive(const kt_frame_desc* d, kt_frame_derived* out) {
  Frame f;
  setup_frame(d, &f);
  memset(out, 0, sizeof *out);
  out->chart = f.chart;
  out->integrator = (f.chart == KT_CHART_KS) ? KT_RK4_DOUBLING : f.intg;
  out->r_horizon = f.rh;
  out->rh_cut = f.rh * 1.03;
  out->r_isco = f.r_in;
  out->r_disk_in = f.r_in;
  out->r_disk_out = f.r_out;
  out->r_escape = f.r_esc;
  out->r_obs = f.cam.r_obs;
  out->theta_obs = f.cam.theta_obs;
  out->phi_obs = f.cam.phi_obs;
  out->fov_h = f.cam.fov_h;
  out->dlam0 = omax(f.step_init, 1e-10);
  out->max_steps = f.max_steps;
  out->solver = f.solver;
  out->tol = f.tol;
  out->bundle_eps = (f.cam.fov_h / (double)f.cam.W) * 0.5;
  out->r_fp32 = (d->precision == KT_PREC_MIXED && f.tol >= 1e-8)
                    ? omax(4.0 * d->M, 2.0 * f.rh) : ktm_inf(); /* renderer's mixed mode */
  return 0;
}

void orc_trace_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix, uint8_t* outcome,
                      double* r, double* redshift, double* magnif, double* phi_disk,
                      double* theta_esc, double* phi_esc, uint32_t* steps, uint32_t* attempts,
                      int nthreads) {
  Frame f;
  setup_frame(d, &f);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const int px = (int)(pix[i] % (uint32_t)d->width);
    const int py = (int)(pix[i] / (uint32_t)d->width);
    Ray o;
    if (f.bundles) {
      o = trace_bundle(&f, px, py);
    } else {
      double al, be;
      cam_pixel_angles(&f.cam, px, py, f.offx, f.offy, &al, &be);
      const Geo s = cam_angle_ray(&f.cam, al, be, &f.g);
      int reason = 0;
      o = (f.solver == KT_SOLVER_ELLIPTIC_CLOSED) ? trace_elliptic(&f, &s, &reason)
          : (f.chart == KT_CHART_KS) ? trace_single_ks(&f, &s)
          : (f.solver == KT_SOLVER_SEMI_ANALYTIC) ? trace_separable(&f, &s)
                                                  : trace_single(&f, s);
    }
    outcome[i] = o.outcome;
    r[i] = o.r;
    redshift[i] = o.redshift;
    magnif[i] = o.magnif;
    phi_disk[i] = o.phi_disk;
    theta_esc[i] = o.theta_esc;
    phi_esc[i] = o.phi_esc;
    if (steps) steps[i] = o.steps;
    if (attempts) attempts[i] = o.attempts;
  }
}

/* The elliptic-closed solver's fallback reason per pixel (0: the closed
 * form gave a disk crossing), for frames whose effective solver is it. */
void orc_elliptic_reasons(const kt_frame_desc* d, int64_t n, const uint32_t* pix, uint8_t* reason) {
  Frame f;
  setup_frame(d, &f);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const int px = (int)(pix[i] % (uint32_t)d->width);
    const int py = (int)(pix[i] / (uint32_t)d->width);
    double al, be, r, g;
    cam_pixel_angles(&f.cam, px, py, f.offx, f.offy, &al, &be);
    const Geo s = cam_angle_ray(&f.cam, al, be, &f.g);
    int why = 0;
    elliptic_closed_form(&f, &s, &r, &g, &why);
    reason[i] = (uint8_t)why;
  }
}

/* --------------------------------------------------------------- colour
 * main.cpp:153-170, 1663-1687, 1799-1866 */

/* (uint8_t)(double) as x86-64 code generated by g++ performs it: truncate
 * toward zero to a 32-bit integer, keep the low byte. */
static uint8_t to_u8(double v) { return (uint8_t)(int32_t)v; }

static void blackbody(double T, uint8_t c[3]) {
  T = oclamp(T, 800.0, 4e4);
  const double t = ktm_log10(T / 800.0) / ktm_log10(4e4 / 800.0);
  double R, G, B;
  if (t < 0.25) {
    R = 1;
    G = (t / 0.25) * 0.4;
    B = 0;
  } else if (t < 0.5) {
    const double f = (t - 0.25) / 0.25;
    R = 1;
    G = 0.4 + f * 0.4;
    B = f * 0.3;
  } else if (t < 0.75) {
    const double f = (t - 0.5) / 0.25;
    R = 1;
    G = 0.8 + f * 0.2;
    B = 0.3 + f * 0.5;
  } else {
    const double f = (t - 0.75) / 0.25;
    R = 1 - f * 0.2;
    G = 1;
    B = 0.8 + f * 0.2;
  }
  c[0] = to_u8(oclamp(R, 0.0, 1.0) * 255);
  c[1] = to_u8(oclamp(G, 0.0, 1.0) * 255);
  c[2] = to_u8(oclamp(B, 0.0, 1.0) * 255);
}

static double page_thorne(double r, double r_isco) {
  if (r <= r_isco) return 0.0;
  const double x = sqrt(r_isco / r);
  return (1.0 - x) / ((r * r) * r);
}

static double tonemap(double x, double exposure, double gamma) {
  x = x * exposure;
  x = x / (1.0 + x);
  return ktm_pow(oclamp(x, 0.0, 1.0), 1.0 / gamma);
}

static void disk_colour(double r, double red, double magnif, double M, double r_isco, double exposure,
                        double gamma, double temp_scale, uint8_t out[3]) {
  const double T = ((6500.0 * temp_scale) * sqrt((6.0 * M) / r)) * oclamp(red, 0.2, 5.0);
  const double pt_norm = page_thorne(r, r_isco);
  const double r_peak = 3.0 * r_isco;
  const double pt_peak = page_thorne(r_peak, r_isco);
  double I = (pt_peak > 0.0) ? pt_norm / pt_peak : 0.0;
  const double red_c = oclamp(red, 0.1, 10.0);
  const double lift = 1.0 + 0.85 * oclamp(1.0 - red_c, 0.0, 1.0);
  I *= ktm_pow(red_c, 4.0) * lift;
  I *= oclamp(1.0 / magnif, 0.05, 5.0);
  uint8_t c[3];
  blackbody(T, c);
  for (int k = 0; k < 3; ++k) out[k] = to_u8(tonemap((c[k] / 255.0) * I, exposure, gamma) * 255);
}

/* hsv_to_rgb (main.cpp:1689-1707); the uint8 channels as doubles. */
static void hsv_to_rgb(double h, double s, double v, double out[3]) {
  h = h - floor(h);
  const double hh = h * 6.0;
  const int hi = (int)hh;
  const double f = hh - (double)hi;
  const double p = v * (1.0 - s);
  const double q = v * (1.0 - s * f);
  const double t = v * (1.0 - s * (1.0 - f));
  double rr, gg, bb;
  switch (hi % 6) {
    case 0: rr = v; gg = t; bb = p; break;
    case 1: rr = q; gg = v; bb = p; break;
    case 2: rr = p; gg = v; bb = t; break;
    case 3: rr = p; gg = q; bb = v; break;
    case 4: rr = t; gg = p; bb = v; break;
    default: rr = v; gg = p; bb = q; break;
  }
  out[0] = (double)to_u8(rr * 255 + 0.5);
  out[1] = (double)to_u8(gg * 255 + 0.5);
  out[2] = (double)to_u8(bb * 255 + 0.5);
}

/* cell_hash (main.cpp:1710-1713) */
static double cell_hash(int cell_id, double a, double b) {
  const double v = ktm_sin((double)cell_id * a + b) * 43758.5453;
  return v - floor(v);
}

/* disk_colour_interstellar (main.cpp:1719-1797); fmod(x, 1.0) is exact and
 * equals x - trunc(x). */
static void disk_colour_interstellar(double r, double phi, double red, double magnif, double r_in,
                                     double r_out, double r_isco, const kt_color_params* cp,
                                     uint8_t out[3]) {
  const int NR = cp->disk_rings > 0 ? cp->disk_rings : 1;
  const int NS = cp->disk_sectors > 0 ? cp->disk_sectors : 1;
  const double sigma = cp->disk_sigma > 0 ? cp->disk_sigma : 0.5;
  const double r_norm = oclamp((r - r_in) / (r_out - r_in), 0.0, 1.0);
  const double phi_norm = (phi - floor(phi / (2.0 * ORC_PI)) * (2.0 * ORC_PI)) / (2.0 * ORC_PI);
  const double ring_pos = r_norm * NR;
  const double sec_pos = phi_norm * NS;
  double acc_r = 0.0, acc_g = 0.0, acc_b = 0.0, w_total = 0.0;
  const double inv2sig2 = 1.0 / (2.0 * sigma * sigma);
  const int SEARCH = (int)ceil(3.0 * sigma) + 1;
  for (int ri = -SEARCH; ri <= NR + SEARCH; ++ri) {
    const double dr = ring_pos - (double)ri;
    if (dr * dr * inv2sig2 > 16.0) continue;
    const int ri_clamped = ri < 0 ? 0 : ri >= NR ? NR - 1 : ri;
    for (int si_raw = -SEARCH; si_raw <= NS + SEARCH; ++si_raw) {
      double ds = sec_pos - (double)si_raw;
      ds = ds - floor((ds + NS * 0.5) / NS) * NS;
      const double dist2 = dr * dr + ds * ds;
      const double w = ktm_exp(-dist2 * inv2sig2);
      if (w < 1e-4) continue;
      const int si_clamped = ((si_raw % NS) + NS) % NS;
      const int cell_id = ri_clamped * NS + si_clamped;
      const double h1 = cell_hash(cell_id, 127.1, 311.7);
      const double h2 = cell_hash(cell_id, 269.5, 183.3);
      const double h3 = cell_hash(cell_id, 419.2, 371.9);
      if (h3 < 0.30) continue;
      const double hx = h1 * 0.14 + cp->disk_hue_offset;
      const double hue = hx - trunc(hx);
      const double sat = 0.70 + h2 * 0.30;
      const double val = 0.50 + h1 * 0.50;
      double c[3];
      hsv_to_rgb(hue, sat, val, c);
      acc_r += w * c[0];
      acc_g += w * c[1];
      acc_b += w * c[2];
      w_total += w;
    }
  }
  if (w_total < 1e-6) {
    out[0] = out[1] = out[2] = 0;
    return;
  }
  const double pt_norm = page_thorne(r, r_isco);
  const double r_peak = 3.0 * r_isco;
  const double pt_peak = page_thorne(r_peak, r_isco);
  double I = (pt_peak > 0.0) ? pt_norm / pt_peak : 0.0;
  const double red_c = oclamp(red, 0.1, 10.0);
  const double lift = 1.0 + 0.85 * oclamp(1.0 - red_c, 0.0, 1.0);
  I *= ktm_pow(red_c, 4.0) * lift;
  I *= oclamp(1.0 / magnif, 0.05, 5.0);
  const double norm = w_total * 255.0;
  out[0] = to_u8(tonemap(acc_r / norm * I, cp->exposure, cp->gamma) * 255);
  out[1] = to_u8(tonemap(acc_g / norm * I, cp->exposure, cp->gamma) * 255);
  out[2] = to_u8(tonemap(acc_b / norm * I, cp->exposure, cp->gamma) * 255);
}

static int iclamp(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

static void bg_sample(const uint8_t* px, int w, int h, double theta, double phi, uint8_t out[3]) {
  double pw = fmod(phi, 2.0 * ORC_PI);
  if (pw < 0) pw += 2.0 * ORC_PI;
  const double uf = (pw / (2.0 * ORC_PI)) * (double)(w - 1);
  const double vf = (theta / ORC_PI) * (double)(h - 1);
  const int u0 = (int)uf, u1 = (w > 1) ? ((u0 + 1) % w) : 0;
  const int v0 = (int)vf, v1 = (v0 + 1 < h - 1) ? v0 + 1 : h - 1;
  const double fu = uf - u0, fv = vf - v0;
  for (int k = 0; k < 3; ++k) {
    const double c00 = px[3 * (iclamp(v0, 0, h - 1) * w + iclamp(u0, 0, w - 1)) + k];
    const double c10 = px[3 * (iclamp(v0, 0, h - 1) * w + iclamp(u1, 0, w - 1)) + k];
    const double c01 = px[3 * (iclamp(v1, 0, h - 1) * w + iclamp(u0, 0, w - 1)) + k];
    const double c11 = px[3 * (iclamp(v1, 0, h - 1) * w + iclamp(u1, 0, w - 1)) + k];
    const double top = c00 + fu * (c10 - c00);
    const double bot = c01 + fu * (c11 - c01);
    out[k] = to_u8(top + fv * (bot - top));
  }
}

void orc_colorize(const kt_frame_desc* d, int64_t n, const uint8_t* outcome, const double* r,
                  const double* redshift, const double* magnif, const double* theta_esc,
                  const double* phi_esc, double exposure, double gamma, double temp_scale,
                  const uint8_t* bg, int bg_w, int bg_h, uint8_t* rgb) {
  Frame f;
  setup_frame(d, &f);
  for (int64_t i = 0; i < n; ++i) {
    uint8_t c[3] = {0, 0, 0};
    /* GeoPixel stores float32 (main.cpp:84-94); colorize reads them back. */
    if (outcome[i] == KT_OUT_DISK) {
      disk_colour((double)(float)r[i], (double)(float)redshift[i], (double)(float)magnif[i], d->M,
                  f.r_in, exposure, gamma, temp_scale, c);
    } else if (outcome[i] == KT_OUT_ESCAPED && bg && bg_w > 0 && bg_h > 0) {
      bg_sample(bg, bg_w, bg_h, (double)(float)theta_esc[i], (double)(float)phi_esc[i], c);
    }
    rgb[3 * i + 0] = c[0];
    rgb[3 * i + 1] = c[1];
    rgb[3 * i + 2] = c[2];
  }
}

void orc_colorize_cp(const kt_frame_desc* d, int64_t n, const uint8_t* outcome, const double* r,
                     const double* redshift, const double* magnif, const double* phi_disk,
                     const double* theta_esc, const double* phi_esc, const kt_color_params* cp,
                     const uint8_t* bg, int bg_w, int bg_h, uint8_t* rgb) {
  Frame f;
  setup_frame(d, &f);
  for (int64_t i = 0; i < n; ++i) {
    uint8_t c[3] = {0, 0, 0};
    if (outcome[i] == KT_OUT_DISK && cp->palette == 1) {
      disk_colour_interstellar((double)(float)r[i], (double)(float)phi_disk[i],
                               (double)(float)redshift[i], (double)(float)magnif[i], f.r_in,
                               d->disk_out, f.r_in, cp, c);
    } else if (outcome[i] == KT_OUT_DISK) {
      disk_colour((double)(float)r[i], (double)(float)redshift[i], (double)(float)magnif[i], d->M,
                  f.r_in, cp->exposure, cp->gamma, cp->temp_scale, c);
    } else if (outcome[i] == KT_OUT_ESCAPED && bg && bg_w > 0 && bg_h > 0) {
      bg_sample(bg, bg_w, bg_h, (double)(float)theta_esc[i], (double)(float)phi_esc[i], c);
    }
    rgb[3 * i + 0] = c[0];
    rgb[3 * i + 1] = c[1];
    rgb[3 * i + 2] = c[2];
  }
}

/* --camera-spp (main.cpp:2232-2322): the jitter offsets, and the average
 * of the passes' images in linear light. */
void orc_spp_offsets(int spp, double* xy) {
  int k = 0;
  if (spp <= 1) {
    xy[0] = xy[1] = 0.0;
    return;
  }
  if (spp == 2) {
    xy[0] = -0.35; xy[1] = 0.0; xy[2] = 0.35; xy[3] = 0.0;
    return;
  }
  if ((spp % 2) == 1) {
    xy[0] = xy[1] = 0.0;
    k = 1;
  }
  static const double seed[7][2] = {{0.35, 0.00}, {0.00, 0.35}, {0.25, 0.25}, {0.45, 0.20},
                                    {0.20, 0.45}, {0.40, 0.00}, {0.00, 0.40}};
  for (int j = 0; j < 7; ++j) {
    if (k + 2 > spp) break;
    xy[2 * k] = seed[j][0]; xy[2 * k + 1] = seed[j][1]; ++k;
    xy[2 * k] = -seed[j][0]; xy[2 * k + 1] = -seed[j][1]; ++k;
  }
  const double golden = 2.39996322972865332;
  for (int m = 0; k < spp; ++m) {
    const double rr = 0.49 * sqrt((double)(m + 1) / (double)(spp + 1));
    const double a = golden * (double)(m + 1);
    const double x = rr * ktm_cos(a), y = rr * ktm_sin(a);
    xy[2 * k] = x; xy[2 * k + 1] = y; ++k;
    if (k < spp) {
      xy[2 * k] = -x; xy[2 * k + 1] = -y; ++k;
    }
  }
}

static double spp_lround(double x) { /* std::lround for x >= 0 */
  const double t = trunc(x);
  return (x - t >= 0.5) ? t + 1.0 : t;
}

void orc_spp_combine(int64_t n, int spp, const uint8_t* passes, double gamma, uint8_t* rgb) {
  const double g = gamma < 1e-6 ? 1e-6 : gamma;
  const double inv_n = 1.0 / (double)spp;
  for (int64_t i = 0; i < 3 * n; ++i) {
    double acc = 0.0;
    for (int s = 0; s < spp; ++s) acc += ktm_pow(oclamp((double)passes[(int64_t)s * 3 * n + i] / 255.0, 0.0, 1.0), g);
    const double disp = ktm_pow(oclamp(acc * inv_n, 0.0, 1.0), 1.0 / g);
    rgb[i] = (uint8_t)(int64_t)spp_lround(255.0 * disp);
  }
}

/* ------------------------------------------------- known-answer helpers
 * Entry points for the checks of tests/core_tests.cpp:18-96 in the
 * reference (metric inverse, camera null condition, one adaptive step,
 * Omega_K sign, KS radius recovery). */
void orc_metric_bl(double M, double a, double Q, double L, double r, double th, double* cov16,
                   double* con16) {
  const Metric g = {M, a, Q, L};
  double A[4][4], B[4][4];
  m_cov_bl(&g, r, th, A);
  m_con_bl(&g, r, th, B);
  memcpy(cov16, A, sizeof A);
  memcpy(con16, B, sizeof B);
}

double orc_hamiltonian(double M, double a, double Q, double L, const double* s7) {
  const Metric g = {M, a, Q, L};
  return m_ham(&g, s7[0], s7[1], s7[3], s7[4], s7[5], s7[6]);
}

void orc_angle_ray(double M, double a, double Q, double L, double r_obs, double th_deg,
                   double ph_deg, double fov_deg, int W, int H, double alpha, double beta,
                   double* s7) {
  const Metric g = {M, a, Q, L};
  Cam c = {r_obs, (th_deg * ORC_PI) / 180.0, (ph_deg * ORC_PI) / 180.0, (fov_deg * ORC_PI) / 180.0,
           W, H};
  const Geo s = cam_angle_ray(&c, alpha, beta, &g);
  const double v[7] = {s.r, s.th, s.ph, s.pr, s.pth, s.pt, s.pphi};
  memcpy(s7, v, sizeof v);
}

int orc_adaptive_step(double M, double a, double Q, double L, double* s7, double* h, int dopri5,
                      double* fsal4, double tol) {
  const Metric g = {M, a, Q, L};
  Geo s = {s7[0], s7[1], s7[2], s7[3], s7[4], s7[5], s7[6]};
  int acc;
  if (dopri5) {
    Vec4 f = {{fsal4[0], fsal4[1], fsal4[2], fsal4[3]}};
    acc = dopri5_adaptive(&g, &s, h, &f, tol);
    memcpy(fsal4, f.v, sizeof f.v);
  } else {
    acc = rk4_adaptive(&g, &s, h, tol);
  }
  const double v[7] = {s.r, s.th, s.ph, s.pr, s.pth, s.pt, s.pphi};
  memcpy(s7, v, sizeof v);
  return acc;
}

double orc_keplerian_omega(double M, double a, double Q, double L, double r) {
  const Metric g = {M, a, Q, L};
  return m_kepler(&g, r);
}

void orc_bl_to_ks(double r, double th, double ph, double a, double* xyz) {
  m_bl_to_ks(r, th, ph, a, &xyz[0], &xyz[1], &xyz[2]);
}

double orc_r_ks(double X, double Y, double Z, double a) { return m_r_ks(X, Y, Z, a); }
