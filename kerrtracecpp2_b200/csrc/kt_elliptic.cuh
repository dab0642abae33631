// kt_elliptic.cuh -- the elliptic-closed solver's closed form
// (trace_single_elliptic_closed, main.cpp:705-1295), host and device.
//
// For a Kerr ray (Q = Lambda = 0): the Mino time of its first equator
// crossing from the polar motion (Jacobi cn, first_equator_crossing_mino_time,
// main.cpp:1178-1219), and its radius there from the four roots of the
// radial quartic (Durand-Kerner iteration) in one of three root
// configurations -- four real, two real and a complex pair, two complex
// pairs -- by Jacobi inversion (init_elliptic_radial_map,
// elliptic_radial_r_from_phase, main.cpp:893-1168), the elliptic integrals
// by Carlson's R_F.  The result is used only when the crossing lies in the
// disk; every other ray keeps the standard tracer's result, and so does a
// ray the standard tracer ends at the horizon (the reference's
// horizon-precedence check, main.cpp:1278-1288).  Complex products and
// quotients use the textbook formulas, |z| hypot.  Arithmetic in the
// reference's order, for bit equality; compiled with --fmad=false.
#pragma once

#include "kt_machines.cuh"

namespace kt {

struct Cx {
  double re, im;
};
KT_HD Cx cx(double re, double im) {
  Cx z;
  z.re = re;
  z.im = im;
  return z;
}
KT_HD Cx cx_add(Cx a, Cx b) { return cx(a.re + b.re, a.im + b.im); }
KT_HD Cx cx_sub(Cx a, Cx b) { return cx(a.re - b.re, a.im - b.im); }
KT_HD Cx cx_mul(Cx a, Cx b) { return cx(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
KT_HD Cx cx_div(Cx a, Cx b) {
  const double t = b.re * b.re + b.im * b.im;
  return cx((a.re * b.re + a.im * b.im) / t, (a.im * b.re - a.re * b.im) / t);
}
KT_HD double cx_abs(Cx a) { return ktm_hypot(a.re, a.im); }

// Carlson's R_F(x, y, z) by duplication to |1 - v/mu| < 1e-10 and the
// fifth-order series (carlson_rf, main.cpp:706-742).
KT_HD_CALL double ell_rf(double x, double y, double z) {
  if (!(x >= 0.0 && y >= 0.0 && z >= 0.0)) return ktm_nan();
  if (!finite(x) || !finite(y) || !finite(z)) return ktm_nan();
  double xn = x, yn = y, zn = z;
  for (int it = 0; it < 64; ++it) {
    const double mu = ((xn + yn) + zn) / 3.0;
    if (!(mu > 0.0) || !finite(mu)) return ktm_nan();
    const double X = 1.0 - xn / mu, Y = 1.0 - yn / mu, Z = 1.0 - zn / mu;
    const double eps = dmax(dmax(fabs(X), fabs(Y)), fabs(Z));
    if (eps < 1e-10) {
      const double E2 = X * Y - Z * Z;
      const double E3 = (X * Y) * Z;
      const double corr =
          (((1.0 - E2 / 10.0) + E3 / 14.0) + (E2 * E2) / 24.0) - ((3.0 * E2) * E3) / 44.0;
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

// F(phi | m) = sin(phi) R_F(cos^2, 1 - m sin^2, 1); K(m) = R_F(0, 1 - m, 1)
// (ellint_F_incomplete, ellint_K_complete, main.cpp:744-757).
KT_HD double ell_F(double phi, double m) {
  double s, c;
  ktm_sincos(phi, &s, &c);
  const double y = 1.0 - (m * s) * s;
  if (y <= 0.0) return ktm_nan();
  return s * ell_rf(c * c, y, 1.0);
}

KT_HD double ell_K(double m) {
  if (!(m >= 0.0 && m < 1.0)) return ktm_nan();
  return ell_rf(0.0, 1.0 - m, 1.0);
}

// sn^2(u | m) by bisection of F over [0, pi/2] (jacobi_sn2_from_u, main.cpp:759-777).
KT_HD double jac_sn2(double u, double m, double Kc) {
  if (!(m >= 0.0 && m < 1.0) || !(Kc > 0.0) || !finite(u)) return ktm_nan();
  double ur = fmod(u, 2.0 * Kc);
  if (ur < 0.0) ur += 2.0 * Kc;
  if (ur > Kc) ur = 2.0 * Kc - ur;
  double lo = 0.0, hi = 0.5 * kPi;
  KT_ROLLED
  for (int it = 0; it < 64; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double Fm = ell_F(mid, m);
    if (!finite(Fm)) return ktm_nan();
    if (Fm < ur)
      lo = mid;
    else
      hi = mid;
  }
  const double s = ktm_sin(0.5 * (lo + hi));
  return s * s;
}

// sn, cn (u | m) (jacobi_sn_cn_from_u, main.cpp:834-876).
KT_HD bool jac_sn_cn(double u, double m, double Kc, double* sn, double* cn) {
  *sn = *cn = ktm_nan();
  if (!(m >= 0.0 && m < 1.0) || !(Kc > 0.0) || !finite(u)) return false;
  const double twoK = 2.0 * Kc;
  long long n = (long long)floor(u / twoK);
  double ur = u - (double)n * twoK;
  if (ur < 0.0) {
    ur += twoK;
    --n;
  }
  const bool second = ur > Kc;
  const double target = second ? (twoK - ur) : ur;
  double lo = 0.0, hi = 0.5 * kPi;
  KT_ROLLED
  for (int it = 0; it < 72; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double Fm = ell_F(mid, m);
    if (!finite(Fm)) return false;
    if (Fm < target)
      lo = mid;
    else
      hi = mid;
  }
  double s, c;
  ktm_sincos(0.5 * (lo + hi), &s, &c);
  if (second) c = -c;
  if ((n & 1LL) != 0) {
    s = -s;
    c = -c;
  }
  *sn = s;
  *cn = c;
  return finite(s) && finite(c);
}

// The roots of z^4 + b0 z^3 + b1 z^2 + b2 z + b3 by Durand-Kerner from four
// points on the circle of radius 1 + max |b_i|, at most 160 sweeps
// (quartic_roots_monic_complex, main.cpp:779-812).
KT_HD_CALL void quartic_roots(const double b[4], Cx z[4]) {
  const double rad = 1.0 + dmax(dmax(dmax(fabs(b[0]), fabs(b[1])), fabs(b[2])), fabs(b[3]));
  const double pi = 3.141592653589793238462643383279502884;
  for (int i = 0; i < 4; ++i) {
    double s, c;
    ktm_sincos((0.5 * (double)i) * pi, &s, &c);
    z[i] = cx(rad * c, rad * s);
  }
  KT_ROLLED
  for (int it = 0; it < 160; ++it) {
    double max_delta = 0.0;
    Cx zn[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      Cx den = cx(1.0, 0.0);
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (i != j) den = cx_mul(den, cx_sub(z[i], z[j]));
      if (cx_abs(den) < 1e-20) den = cx(1e-20, 0.0);
      Cx p = cx_add(z[i], cx(b[0], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[1], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[2], 0.0));
      p = cx_add(cx_mul(p, z[i]), cx(b[3], 0.0));
      const Cx delta = cx_div(p, den);
      zn[i] = cx_sub(z[i], delta);
      max_delta = dmax(max_delta, cx_abs(delta));
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) z[i] = zn[i];
    if (max_delta < 1e-13) break;
  }
}

enum : int { kRadReal4 = 0, kRadReal2 = 1, kRadComplex4 = 2 };

// EllipticRadialMap (main.cpp:893-916): r(X) on the ray's radial branch,
// X = phase_sign X0 + tau_sign omega tau in Mino time tau.
struct RadMap {
  int kind, phase_sign, tau_sign;
  double r1, r2, r3, r4;
  double m, Kc, omega, X0;
  double A, B, r_lo, r_hi;
  double a2, b1, g0;
};

// elliptic_radial_r_from_phase (main.cpp:918-956).
KT_HD_CALL double rad_r(const RadMap& mp, double X) {
  if (mp.kind == kRadReal4) {
    const double sn2 = jac_sn2(X, mp.m, mp.Kc);
    if (!finite(sn2)) return ktm_nan();
    const double r24 = mp.r2 - mp.r4, r14 = mp.r1 - mp.r4;
    const double den = r24 - r14 * sn2;
    if (fabs(den) < 1e-14) return ktm_nan();
    return (mp.r1 * r24 - (mp.r2 * r14) * sn2) / den;
  }
  double sn, cn;
  if (!jac_sn_cn(X, mp.m, mp.Kc, &sn, &cn)) return ktm_nan();
  if (mp.kind == kRadReal2) {
    const double num = (mp.B * mp.r_hi - mp.A * mp.r_lo) + (mp.B * mp.r_hi + mp.A * mp.r_lo) * cn;
    const double den = (mp.B - mp.A) + (mp.B + mp.A) * cn;
    if (fabs(den) < 1e-14) return ktm_nan();
    return num / den;
  }
  // jacobi_sc_from_u (main.cpp:878-885)
  if (fabs(cn) < 1e-14) return ktm_nan();
  const double sc = sn / cn;
  if (!finite(sc)) return ktm_nan();
  const double den = 1.0 + mp.g0 * sc;
  if (fabs(den) < 1e-14) return ktm_nan();
  return -mp.a2 * ((mp.g0 - sc) / den) - mp.b1;
}

// align_initial_radial_sign (main.cpp:981-1000): the branch that moves r the
// way dr0 does.
KT_HD void rad_align(RadMap* mp, double dr0, bool flip_phase, bool flip_tau) {
  if (fabs(dr0) < 1e-14) return;
  const double probe = 1e-6;
  const double Xp = (double)mp->phase_sign * mp->X0 + ((double)mp->tau_sign * mp->omega) * probe;
  const double Xm = (double)mp->phase_sign * mp->X0 - ((double)mp->tau_sign * mp->omega) * probe;
  const double rp = rad_r(*mp, Xp), rm = rad_r(*mp, Xm);
  if (!finite(rp) || !finite(rm)) return;
  if ((dr0 >= 0.0) == (rp >= rm)) return;
  if (flip_phase) mp->phase_sign = -mp->phase_sign;
  if (flip_tau) mp->tau_sign = -mp->tau_sign;
}

// init_elliptic_radial_map (main.cpp:958-1168).
KT_HD_CALL bool rad_init(const SepConst& c, double r0, double dr0, RadMap* out) {
  const double u = c.Lz - c.a * c.E;
  const double Kpot = c.Qc + u * u;
  const double A0 = (c.E * c.a) * c.a - c.a * c.Lz;
  const double c4 = c.E * c.E;
  if (!(c4 > 1e-18)) return false;
  const double c2 = (2.0 * c.E) * A0 - Kpot;
  const double c1 = (2.0 * c.M) * Kpot;
  const double c0 = A0 * A0 - (c.a * c.a) * Kpot;
  const double b[4] = {0.0, c2 / c4, c1 / c4, c0 / c4};
  Cx z[4];
  quartic_roots(b, z);
  double rr[4];
  Cx cr[4];
  int nr = 0, nc = 0;
  for (int i = 0; i < 4; ++i) {
    if (!finite(z[i].re) || !finite(z[i].im)) return false;
    const double tol = 1e-7 * dmax(1.0, fabs(z[i].re));
    if (fabs(z[i].im) <= tol)
      rr[nr++] = z[i].re;
    else
      cr[nc++] = z[i];
  }
  RadMap mp;
  memset(&mp, 0, sizeof mp);
  mp.phase_sign = mp.tau_sign = 1;
  if (nr == 4) {
    for (int i = 1; i < 4; ++i)  // descending
      for (int j = i; j > 0 && rr[j] > rr[j - 1]; --j) {
        const double t = rr[j];
        rr[j] = rr[j - 1];
        rr[j - 1] = t;
      }
    mp.kind = kRadReal4;
    mp.r1 = rr[0];
    mp.r2 = rr[1];
    mp.r3 = rr[2];
    mp.r4 = rr[3];
    const double den_omega = (mp.r1 - mp.r3) * (mp.r2 - mp.r4);
    if (!(den_omega > 0.0)) return false;
    mp.omega = 0.5 * sqrt(den_omega);
    const double k_num = (mp.r2 - mp.r3) * (mp.r1 - mp.r4);
    const double k_den = (mp.r2 - mp.r4) * (mp.r1 - mp.r3);
    if (!(k_den > 0.0)) return false;
    mp.m = k_num / k_den;
    if (!(mp.m >= 0.0 && mp.m < 1.0)) return false;
    mp.Kc = ell_K(mp.m);
    if (!finite(mp.Kc) || !(mp.Kc > 0.0)) return false;
    const double den_obs = r0 - mp.r2, den_root = mp.r1 - mp.r4;
    if (fabs(den_obs) < 1e-14 || fabs(den_root) < 1e-14) return false;
    const double u0_raw = ((r0 - mp.r1) / den_obs) * ((mp.r2 - mp.r4) / den_root);
    if (!finite(u0_raw)) return false;
    if (u0_raw < -1e-6 || u0_raw > 1.0 + 1e-6) return false;
    const double u0 = dclamp(u0_raw, 0.0, 1.0);
    mp.X0 = ell_F(ktm_asin(sqrt(u0)), mp.m);
    if (!finite(mp.X0)) return false;
    const int alpha = (r0 >= mp.r3 && r0 <= mp.r2) ? -1 : 1;
    mp.phase_sign = alpha * ((dr0 >= 0.0) ? 1 : -1);
    mp.tau_sign = 1;
    rad_align(&mp, dr0, true, false);
  } else if (nr == 2 && nc == 2) {
    const double r1 = dmin(rr[0], rr[1]), r2 = dmax(rr[0], rr[1]);
    const double b1 = 0.5 * (cr[0].re + cr[1].re);
    const double a1 = 0.5 * (fabs(cr[0].im) + fabs(cr[1].im));
    if (!(a1 > 0.0) || !finite(a1) || !finite(b1)) return false;
    const double A = sqrt(a1 * a1 + (b1 - r2) * (b1 - r2));
    const double B = sqrt(a1 * a1 + (b1 - r1) * (b1 - r1));
    if (!(A > 0.0 && B > 0.0 && B > A)) return false;
    const double r21 = r2 - r1;
    const double k3 = (((A + B) * (A + B)) - r21 * r21) / ((4.0 * A) * B);
    if (!(k3 > 0.0 && k3 < 1.0)) return false;
    const double K3 = ell_K(k3);
    if (!finite(K3) || !(K3 > 0.0)) return false;
    const double x3 = (A * (r0 - r1) - B * (r0 - r2)) / (A * (r0 - r1) + B * (r0 - r2));
    if (!finite(x3)) return false;
    const double F0 = ell_F(ktm_acos(dclamp(x3, -1.0, 1.0)), k3);
    if (!finite(F0)) return false;
    mp.kind = kRadReal2;
    mp.r1 = r2;
    mp.r2 = r1;
    mp.r_lo = r1;
    mp.r_hi = r2;
    mp.A = A;
    mp.B = B;
    mp.m = k3;
    mp.Kc = K3;
    mp.omega = sqrt(A * B);
    mp.X0 = F0;
    mp.phase_sign = (dr0 >= 0.0) ? 1 : -1;
    mp.tau_sign = 1;
    rad_align(&mp, dr0, true, false);
  } else if (nr == 0 && nc == 4) {
    Cx pos[2], neg[2];
    int np = 0, nn = 0;
    for (int i = 0; i < 4; ++i) {
      if (cr[i].im >= 0.0) {
        if (np < 2) pos[np] = cr[i];
        ++np;
      } else {
        if (nn < 2) neg[nn] = cr[i];
        ++nn;
      }
    }
    if (np != 2 || nn != 2) return false;
    const double d00 = cx_abs(cx_sub(pos[0], cx(neg[0].re, -neg[0].im)));
    const double d01 = cx_abs(cx_sub(pos[0], cx(neg[1].re, -neg[1].im)));
    const int j0 = (d00 <= d01) ? 0 : 1;
    const Cx nA = j0 == 0 ? neg[0] : neg[1], nB = j0 == 0 ? neg[1] : neg[0];
    const double bA = 0.5 * (pos[0].re + nA.re), aA = 0.5 * (fabs(pos[0].im) + fabs(nA.im));
    const double bB = 0.5 * (pos[1].re + nB.re), aB = 0.5 * (fabs(pos[1].im) + fabs(nB.im));
    if (!(aA > 0.0 && aB > 0.0)) return false;
    double b1 = bA, a1 = aA, b2 = bB, a2 = aB;
    if (bB > bA) {
      b1 = bB;
      a1 = aB;
      b2 = bA;
      a2 = aA;
    }
    if (!(b1 > b2)) return false;
    const double C = sqrt((a1 - a2) * (a1 - a2) + (b1 - b2) * (b1 - b2));
    const double D = sqrt((a1 + a2) * (a1 + a2) + (b1 - b2) * (b1 - b2));
    if (!(C > 0.0 && D > 0.0)) return false;
    const double k4 = ((4.0 * C) * D) / ((C + D) * (C + D));
    if (!(k4 > 0.0 && k4 < 1.0)) return false;
    const double K4 = ell_K(k4);
    if (!finite(K4) || !(K4 > 0.0)) return false;
    const double g_num = (4.0 * a2) * a2 - (C - D) * (C - D);
    const double g_den = (C + D) * (C + D) - (4.0 * a2) * a2;
    if (!(g_num > 0.0 && g_den > 0.0)) return false;
    const double g0 = sqrt(g_num / g_den);
    if (!(g0 > 0.0) || !finite(g0)) return false;
    const double x4 = (r0 - b2) / dmax(a2, 1e-15);
    const double F0 = ell_F(ktm_atan(x4) + ktm_atan(g0), k4);
    if (!finite(F0)) return false;
    mp.kind = kRadComplex4;
    mp.m = k4;
    mp.Kc = K4;
    mp.omega = 0.5 * (C + D);
    mp.X0 = F0;
    mp.phase_sign = 1;
    mp.tau_sign = (dr0 >= 0.0) ? 1 : -1;
    mp.a2 = a2;
    mp.b1 = b1;
    mp.g0 = g0;
    rad_align(&mp, dr0, false, true);
  } else {
    return false;
  }
  *out = mp;
  return true;
}

// first_equator_crossing_mino_time (main.cpp:1178-1219).
KT_HD bool eq_crossing(const SepConst& c, double th0, double dth0, double* tau_first) {
  const double A = ((c.a * c.a) * c.E) * c.E;
  if (!(A > 1e-15)) return false;
  const double B = (A - c.Lz * c.Lz) - c.Qc;
  const double disc = B * B + (4.0 * A) * c.Qc;
  if (!(disc >= 0.0)) return false;
  const double sq = sqrt(disc);
  const double up = (B + sq) / (2.0 * A), um = (B - sq) / (2.0 * A);
  if (!(up > 0.0 && um < 0.0)) return false;
  const double m = up / (up - um);
  if (!(m >= 0.0 && m < 1.0)) return false;
  const double Kc = ell_K(m);
  if (!finite(Kc) || !(Kc > 0.0)) return false;
  const double omega = sqrt(A * (up - um));
  if (!(omega > 0.0) || !finite(omega)) return false;
  const double mu_plus = sqrt(up);
  const double mu0 = ktm_cos(th0);
  const double c0 = dclamp(fabs(mu0) / dmax(mu_plus, 1e-15), 0.0, 1.0);
  const double u_base = ell_F(ktm_acos(c0), m);
  if (!finite(u_base)) return false;
  const double tau_period = (4.0 * Kc) / omega;
  if (!(tau_period > 0.0) || !finite(tau_period)) return false;
  const double u0 = (mu0 * dth0) > 0.0 ? u_base : -u_base;
  double tf = (Kc - u0) / omega;
  if (tf < 0.0) tf += tau_period;
  *tau_first = tf;
  return finite(tf);
}

// EllipticFallbackReason (main.cpp:178-186).
enum : int { kEfNone = 0, kEfInit = 1, kEfTheta = 2, kEfRadialInit = 3, kEfRadialInvalid = 4,
             kEfOutsideDisk = 5 };

// The closed form for the camera ray s: true with the disk crossing's
// radius and redshift, else false with the reason the reference falls back
// to the standard tracer.
KT_HD_CALL bool elliptic_closed_form(const Frame& f, const Geo& s, double* r_out, double* g_out,
                                     int* reason) {
  SepConst c;
  if (!sep_init(f.g, s.th, s.pth, s.pt, s.pphi, &c)) {
    *reason = kEfInit;
    return false;
  }
  // geodesic_rhs's dr = g^rr p_r, dtheta = g^thth p_theta at the camera
  const Inv U = bl_inv(f.g, s.r, bl_ang(f.g, s.th));
  const double dr0 = U.rr * s.pr, dth0 = U.hh * s.pth;
  double tau_first = 0.0;
  if (!eq_crossing(c, s.th, dth0, &tau_first)) {
    *reason = kEfTheta;
    return false;
  }
  RadMap mp;
  if (!rad_init(c, s.r, dr0, &mp)) {
    *reason = kEfRadialInit;
    return false;
  }
  const double X = (double)mp.phase_sign * mp.X0 + ((double)mp.tau_sign * mp.omega) * tau_first;
  const double r_now = rad_r(mp, X);
  if (!finite(r_now)) {
    *reason = kEfRadialInvalid;
    return false;
  }
  const double u = c.Lz - c.a * c.E;
  const double A0 = c.E * (r_now * r_now + c.a * c.a) - c.a * c.Lz;
  const double Delta = (r_now * r_now - (2.0 * c.M) * r_now) + c.a * c.a;
  const double R = A0 * A0 - Delta * (c.Qc + u * u);  // separable_radial_potential
  const double R_scale = dmax(1.0, fabs(((((c.E * c.E) * r_now) * r_now) * r_now) * r_now));
  if (R < -1e-8 * R_scale || (mp.kind != kRadComplex4 && r_now < mp.r1) || r_now < f.rh_cut) {
    *reason = kEfRadialInvalid;
    return false;
  }
  if (r_now > f.r_esc || !(r_now >= f.r_in && r_now <= f.r_out)) {
    *reason = kEfOutsideDisk;
    return false;
  }
  *reason = kEfNone;
  *r_out = r_now;
  *g_out = dclamp(disk_redshift(f.g, f.eq, r_now, s.pt, s.pphi), 0.0, 20.0);
  return true;
}

}  // namespace kt
