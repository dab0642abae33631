// kt_physics.cuh -- FP64 physics of the geodesic path, host+device.
//
// The functions reproduce the reference renderer's floating-point operation
// order exactly (the parity bar is bit equality with the reference's CPU
// FP64 path); they are organised for the GPU:
//   * the angular part of the BL inverse metric (one sincos) is shared by
//     every evaluation at the same theta, so one RHS costs 3 sincos instead
//     of the reference's 15 trig calls, with identical values;
//   * frame constants (a^2, Xi^2, the observer's metric for the camera) are
//     computed once on the host with the same code;
//   * no function allocates or loops over unknown bounds.
// Compile device code with --fmad=false and host code with
// -ffp-contract=off: a fused multiply-add changes the rounding of the
// reference's separate multiply and add.
#pragma once

#include <math.h>
#include <stdint.h>

#include "ktmath.h"

#if defined(__CUDACC__)
#define KT_HD __host__ __device__ __forceinline__
#else
#define KT_HD inline
#endif

// A real call on the device (one copy of the body, its registers apart from
// the caller's); inline on the host.
#if defined(__CUDA_ARCH__)
#define KT_HD_CALL __host__ __device__ __noinline__
#elif defined(__CUDACC__)
#define KT_HD_CALL __host__ __device__ inline
#else
#define KT_HD_CALL inline
#endif

// Keep a loop rolled in device code: the loop body is the bulk of the
// kernel, and one copy of it fits the instruction cache.
#if defined(__CUDA_ARCH__)
#define KT_ROLLED _Pragma("unroll 1")
#else
#define KT_ROLLED
#endif

namespace kt {

constexpr double kPi = 3.14159265358979323846;  // M_PI
constexpr double kHalfPi = kPi / 2.0;           // M_PI/2.0 (exact halving)

// std::max / std::min / clamp semantics of the reference (NaN included).
KT_HD double dmax(double a, double b) { return (a < b) ? b : a; }
KT_HD double dmin(double a, double b) { return (b < a) ? b : a; }
KT_HD double dclamp(double v, double lo, double hi) { return v < lo ? lo : v > hi ? hi : v; }
KT_HD bool finite(double x) { return !ktm_isnan(x) && !ktm_isinf(x); }

// KNdSMetric parameters plus products the reference recomputes inline.
struct Metric {
  double M, a, Q, L;
  double a2;    // a*a
  double fa2;   // 4.0*a2        (r_KS, knds_metric.hpp:154)
  double Laa;   // (L*a)*a        (Delta_theta, Xi)
  double xi2;   // Xi()*Xi()
  double axi2;  // a*xi2
  double twoM;  // 2.0*M
  double Q2;    // Q*Q
};

KT_HD Metric make_metric(double M, double a, double Q, double L) {
  Metric g;
  g.M = M;
  g.a = a;
  g.Q = Q;
  g.L = L;
  g.a2 = a * a;
  g.fa2 = 4.0 * g.a2;
  g.Laa = (L * a) * a;
  const double xi = 1.0 + g.Laa / 3.0;
  g.xi2 = xi * xi;
  g.axi2 = a * g.xi2;
  g.twoM = 2.0 * M;
  g.Q2 = Q * Q;
  return g;
}

// ---------------------------------------------------------------- BL chart
// knds_metric.hpp:45-132

// theta-dependent factors: cos, sin^2, a^2 cos^2 (in Sigma), Delta_theta.
struct Ang {
  double ct, st2, Ath, dth;
};

// x / 3 as the IEEE quotient, either as ktm_div3's three operations (kD3,
// the single-ray kernels) or as the division (the bundle kernel, whose
// unrolled Hessian of nine metric inverses runs faster with it); both give
// the same bits.
template <bool kD3>
KT_HD double third_of(double x) {
  return kD3 ? ktm_div3(x) : x / 3.0;
}

template <bool kD3 = true>
KT_HD Ang bl_ang(const Metric& g, double th) {
  double st, ct;
  ktm_sincos(th, &st, &ct);
  Ang A;
  A.ct = ct;
  A.st2 = st * st;
  A.Ath = (g.a2 * ct) * ct;
  A.dth = 1.0 + third_of<kD3>((g.Laa * ct) * ct);
  return A;
}

// Delta_r, knds_metric.hpp:51
template <bool kD3 = true>
KT_HD double bl_delta_r(const Metric& g, double r, double r2a2) {
  return ((r2a2 * (1.0 - third_of<kD3>((g.L * r) * r))) - g.twoM * r) + g.Q2;
}

// Non-zero entries of g^{mu nu} (contravariant_BL, knds_metric.hpp:99-117).
struct Inv {
  double tt, tp, rr, hh, pp;  // g^tt, g^tphi, g^rr, g^thth, g^phiphi
};

template <bool kD3 = true>
KT_HD Inv bl_inv(const Metric& g, double r, const Ang& A) {
  const double r_sq = r * r;
  const double sig = r_sq + A.Ath;
  const double r2a2 = r_sq + g.a2;
  const double dr = bl_delta_r<kD3>(g, r, r2a2);
  const double dth = A.dth;
  const double pre = (sig * dr) * dth;
  Inv U;
  U.tt = ((-g.xi2) * ((dth * r2a2) * r2a2 - ((dr * g.a) * g.a) * A.st2)) / pre;
  U.tp = (g.axi2 * (dr - dth * r2a2)) / pre;
  U.rr = dr / sig;
  U.hh = dth / sig;
  U.pp = (A.st2 > 1e-14) ? (g.xi2 * (dr - ((dth * g.a) * g.a) * A.st2)) / (pre * A.st2) : 0.0;
  return U;
}

// hamiltonian, knds_metric.hpp:122-132
KT_HD double bl_ham(const Inv& U, double pr, double pth, double pt, double pphi) {
  return 0.5 * (((((U.tt * pt) * pt + ((2.0 * U.tp) * pt) * pphi) + (U.rr * pr) * pr) +
                 (U.hh * pth) * pth) +
                (U.pp * pphi) * pphi);
}

// Non-zero entries of g_{mu nu} (covariant_BL, knds_metric.hpp:71-88).
struct Cov {
  double tt, tp, rr, hh, pp;
};

KT_HD Cov bl_cov(const Metric& g, double r, const Ang& A) {
  const double r_sq = r * r;
  const double sig = r_sq + A.Ath;
  const double r2a2 = r_sq + g.a2;
  const double dr = bl_delta_r(g, r, r2a2);
  const double dth = A.dth;
  const double pre = sig * g.xi2;
  Cov G;
  G.tt = (-dr + ((dth * g.a) * g.a) * A.st2) / pre;
  G.tp = ((g.a * A.st2) * (dr - dth * r2a2)) / pre;
  G.rr = sig / dr;
  G.hh = sig / dth;
  G.pp = (A.st2 * ((dth * r2a2) * r2a2 - ((dr * g.a) * g.a) * A.st2)) / pre;
  return G;
}

// Geodesic right-hand side (geodesic_rhs, geodesic.hpp:143-166) together with
// dphi/dlambda (dphi_vel, geodesic.hpp:40-45): the reference evaluates
// dphi_vel at the same (r, theta) as the RHS, so it is the same g^{mu nu}.
// k = {dr, dtheta, dp_r, dp_theta, dphi}.
//
// Three code shapes with identical arithmetic (KT_RHS_VARIANT, the default of
// bl_rhs_centre's kVar):
//   0  the three angles (theta, theta +- 1e-6) and the five inverse metrics
//      (centre, r +- eps_r, theta +- eps_th) in rolled loops: one copy each;
//   1  angles rolled; the four finite-difference metrics as two pairs in a
//      rolled loop (two independent chains per iteration);
//   2  everything unrolled.
#ifndef KT_RHS_VARIANT
#define KT_RHS_VARIANT 1
#endif

KT_HD Ang ang_select(int i, const Ang& A0, const Ang& Ap, const Ang& Am) {
  Ang A;
  A.ct = 0.0;
  A.st2 = (i == 1) ? Ap.st2 : (i == 2) ? Am.st2 : A0.st2;
  A.Ath = (i == 1) ? Ap.Ath : (i == 2) ? Am.Ath : A0.Ath;
  A.dth = (i == 1) ? Ap.dth : (i == 2) ? Am.dth : A0.dth;
  return A;
}

// bl_rhs, also handing back the centre's angle factors and g^{mu nu} (the
// bundle RHS evaluates both again).
template <bool kD3 = true, int kVar = KT_RHS_VARIANT>
KT_HD void bl_rhs_centre(const Metric& g, double r, double th, double pr, double pth, double pt,
                         double pphi, double k[5], Ang* A_c, Inv* U_c) {
  const double eps_r = 1e-5 * dmax(fabs(r), 0.01);
  const double eps_th = 1e-6;
  Ang A0;
  double hp = 0.0, hm = 0.0, tp = 0.0, tm = 0.0;
  if constexpr (kVar == 2) {
    A0 = bl_ang<kD3>(g, th);
    const Inv U0 = bl_inv<kD3>(g, r, A0);
    k[0] = U0.rr * pr;
    k[1] = U0.hh * pth;
    k[4] = U0.tp * pt + U0.pp * pphi;
    *U_c = U0;
    hp = bl_ham(bl_inv<kD3>(g, r + eps_r, A0), pr, pth, pt, pphi);
    hm = bl_ham(bl_inv<kD3>(g, r - eps_r, A0), pr, pth, pt, pphi);
    tp = bl_ham(bl_inv<kD3>(g, r, bl_ang<kD3>(g, th + eps_th)), pr, pth, pt, pphi);
    tm = bl_ham(bl_inv<kD3>(g, r, bl_ang<kD3>(g, th - eps_th)), pr, pth, pt, pphi);
  } else {
    Ang Ap, Am;
    KT_ROLLED
    for (int j = 0; j < 3; ++j) {
      const double x = (j == 0) ? th : (j == 1) ? th + eps_th : th - eps_th;
      const Ang a = bl_ang<kD3>(g, x);
      if (j == 0) A0 = a;
      else if (j == 1) Ap = a;
      else Am = a;
    }
    if constexpr (kVar == 1) {
      {
        const Inv U0 = bl_inv<kD3>(g, r, A0);
        k[0] = U0.rr * pr;
        k[1] = U0.hh * pth;
        k[4] = U0.tp * pt + U0.pp * pphi;
        *U_c = U0;
      }
      KT_ROLLED
      for (int j = 0; j < 2; ++j) {
        // j = 0: (r + eps_r, theta), (r - eps_r, theta); j = 1: (r, theta +- eps_th)
        const double ra = (j == 0) ? r + eps_r : r;
        const double rb = (j == 0) ? r - eps_r : r;
        const Inv Ua = bl_inv<kD3>(g, ra, ang_select(j == 0 ? 0 : 1, A0, Ap, Am));
        const Inv Ub = bl_inv<kD3>(g, rb, ang_select(j == 0 ? 0 : 2, A0, Ap, Am));
        const double ha = bl_ham(Ua, pr, pth, pt, pphi);
        const double hb = bl_ham(Ub, pr, pth, pt, pphi);
        hp = (j == 0) ? ha : hp;
        hm = (j == 0) ? hb : hm;
        tp = (j == 1) ? ha : tp;
        tm = (j == 1) ? hb : tm;
      }
    } else {
      KT_ROLLED
      for (int i = 0; i < 5; ++i) {
        const double ri = (i == 1) ? r + eps_r : (i == 2) ? r - eps_r : r;
        const Inv U = bl_inv<kD3>(g, ri, ang_select(i == 3 ? 1 : i == 4 ? 2 : 0, A0, Ap, Am));
        if (i == 0) {
          k[0] = U.rr * pr;
          k[1] = U.hh * pth;
          k[4] = U.tp * pt + U.pp * pphi;
          *U_c = U;
        } else {
          const double h = bl_ham(U, pr, pth, pt, pphi);
          hp = (i == 1) ? h : hp;
          hm = (i == 2) ? h : hm;
          tp = (i == 3) ? h : tp;
          tm = (i == 4) ? h : tm;
        }
      }
    }
  }
  k[2] = -(hp - hm) / (2.0 * eps_r);
  k[3] = -(tp - tm) / (2.0 * eps_th);
  *A_c = A0;
}

KT_HD void bl_rhs(const Metric& g, double r, double th, double pr, double pth, double pt,
                  double pphi, double k[5]) {
  Ang A;
  Inv U;
  bl_rhs_centre(g, r, th, pr, pth, pt, pphi, k, &A, &U);
}

// Reciprocal and sincos of the mixed-precision right-hand sides, which are
// not compared bit for bit.  FP64 reciprocal on the device: the hardware seed
// (rcp.approx.ftz.f64) refined by two Newton-Raphson steps y <- y + y(1 - xy),
// each of which squares the relative error, to within an ulp of 1/x
// (arguments outside [1e-300, 1e300] in magnitude take the division); FP32:
// the correctly rounded __frcp_rn.  sincos on the device: CUDA's double
// sincos.  On the host both are the renderer's own.
template <class T>
KT_HD T mx_rcp(T x) {
#if defined(__CUDA_ARCH__)
  if (sizeof(T) == sizeof(float)) return (T)__frcp_rn((float)x);
  const double xd = (double)x;
  if (!(fabs(xd) >= 1e-300 && fabs(xd) <= 1e300)) return (T)(1.0 / xd);
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(xd));
  double e = fma(-xd, y, 1.0);
  y = fma(y, e, y);
  e = fma(-xd, y, 1.0);
  return (T)fma(y, e, y);
#else
  return (T)1 / x;
#endif
}

KT_HD void mx_sincos(double x, double* s, double* c) {
#if defined(__CUDA_ARCH__)
  sincos(x, s, c);
#else
  ktm_sincos(x, s, c);
#endif
}

// g^{mu nu} at (r, theta) in FP64 with the mixed path's operations (the
// mixed tracer's constraint reprojection): the closed forms of
// bl_rhs_analytic's comment below.
KT_HD Inv bl_inv_mx(const Metric& g, double r, double th) {
  double sn, c;
  mx_sincos(th, &sn, &c);
  const double third = 1.0 / 3.0;
  const double s2 = sn * sn, c2 = c * c;
  const double r2 = r * r, A = r2 + g.a2, S = r2 + g.a2 * c2;
  const double R = A * (1.0 - g.L * r2 * third) - 2.0 * g.M * r + g.Q2;
  const double Tt = 1.0 + g.L * g.a2 * c2 * third;
  const double iS = mx_rcp(S), iR = mx_rcp(R), iT = mx_rcp(Tt);
  const bool pole = !(s2 > 1e-14);
  Inv U;
  U.tt = -g.xi2 * iS * (A * A * iR - g.a2 * s2 * iT);
  U.tp = g.a * g.xi2 * iS * (iT - A * iR);
  U.rr = R * iS;
  U.hh = Tt * iS;
  U.pp = pole ? 0.0 : g.xi2 * iS * (iT * mx_rcp(s2) - g.a2 * iR);
  return U;
}

// Analytic Hamiltonian gradient for the mixed-precision tracer (no
// counterpart in the reference, which differentiates H by central
// differences).  With S = Sigma, R = Delta_r, T = Delta_theta, A = r^2+a^2,
// s2 = sin^2, c = cos, xi2 = Xi^2, the inverse metric is
//   g^tt = -xi2/S (A^2/R - a^2 s2/T)      g^tphi = a xi2/S (1/T - A/R)
//   g^rr = R/S     g^thth = T/S           g^phiphi = xi2/S (1/(T s2) - a^2/R)
// and dH/dr, dH/dtheta follow by the quotient rule from dS/dr = 2r,
// dR/dr = 2r(1 - L r^2/3) - (2L r/3) A - 2M, dS/dth = -2a^2 s c,
// dT/dth = -(2 L a^2/3) s c, d(s2)/dth = 2 s c.  One evaluation, four
// reciprocals; T is float (far field) or double.  k as bl_rhs.
template <class T>
KT_HD void bl_rhs_analytic(const Metric& g, double r_, double th_, double pr_, double pth_,
                           double pt_, double pphi_, double k[5]) {
  const T r = (T)r_, pr = (T)pr_, pth = (T)pth_, pt = (T)pt_, pphi = (T)pphi_;
  const T a = (T)g.a, a2 = (T)g.a2, L = (T)g.L, M = (T)g.M, Q2 = (T)g.Q2, xi2 = (T)g.xi2;
  T sn, c;
  if (sizeof(T) == sizeof(float)) {
    float sf, cf;
    sincosf((float)th_, &sf, &cf);
    sn = (T)sf;
    c = (T)cf;
  } else {
    double sd, cd;
    mx_sincos(th_, &sd, &cd);
    sn = (T)sd;
    c = (T)cd;
  }
  const T third = (T)(1.0 / 3.0);
  const T s2 = sn * sn, sc = sn * c;
  const T r2 = r * r;
  const T A = r2 + a2;
  const T S = r2 + a2 * c * c;
  const T Lr2_3 = L * r2 * third;
  const T R = A * ((T)1 - Lr2_3) - (T)2 * M * r + Q2;
  const T Tt = (T)1 + L * a2 * c * c * third;
  const T iS = mx_rcp(S), iR = mx_rcp(R), iT = mx_rcp(Tt);
  const bool pole = !(s2 > (T)1e-14);
  const T is2 = pole ? (T)0 : mx_rcp(s2);
  // g^{mu nu}
  const T X_tt = A * A * iR - a2 * s2 * iT;
  const T X_tp = iT - A * iR;
  const T X_pp = pole ? (T)0 : (iT * is2 - a2 * iR);
  const T U_tp = a * xi2 * iS * X_tp;
  const T U_rr = R * iS, U_hh = Tt * iS;
  const T U_pp = xi2 * iS * X_pp;
  // d/dr
  const T dS_r = (T)2 * r;
  const T dR_r = (T)2 * r * ((T)1 - Lr2_3) - ((T)2 * L * r * third) * A - (T)2 * M;
  const T diS_r = -dS_r * iS * iS, diR_r = -dR_r * iR * iR;
  const T dX_tt_r = (T)2 * A * dS_r * iR + A * A * diR_r;  // dA/dr = dS/dr = 2r
  const T dX_tp_r = -(dS_r * iR + A * diR_r);
  const T dX_pp_r = pole ? (T)0 : -a2 * diR_r;
  const T dU_tt_r = -xi2 * (diS_r * X_tt + iS * dX_tt_r);
  const T dU_tp_r = a * xi2 * (diS_r * X_tp + iS * dX_tp_r);
  const T dU_rr_r = dR_r * iS + R * diS_r;
  const T dU_hh_r = Tt * diS_r;
  const T dU_pp_r = xi2 * (diS_r * X_pp + iS * dX_pp_r);
  // d/dtheta
  const T dS_t = -(T)2 * a2 * sc;
  const T dT_t = -((T)2 * L * a2 * third) * sc;
  const T diS_t = -dS_t * iS * iS, diT_t = -dT_t * iT * iT;
  const T dis2_t = pole ? (T)0 : -(T)2 * sc * is2 * is2;
  const T dX_tt_t = -a2 * ((T)2 * sc * iT + s2 * diT_t);
  const T dX_pp_t = pole ? (T)0 : (diT_t * is2 + iT * dis2_t);
  const T dU_tt_t = -xi2 * (diS_t * X_tt + iS * dX_tt_t);
  const T dU_tp_t = a * xi2 * (diS_t * X_tp + iS * diT_t);
  const T dU_rr_t = R * diS_t;
  const T dU_hh_t = dT_t * iS + Tt * diS_t;
  const T dU_pp_t = xi2 * (diS_t * X_pp + iS * dX_pp_t);
  const T ptpt = pt * pt, ptpp = (T)2 * pt * pphi, prpr = pr * pr, phph = pth * pth,
          pppp = pphi * pphi;
  k[0] = (double)(U_rr * pr);
  k[1] = (double)(U_hh * pth);
  k[4] = (double)(U_tp * pt + U_pp * pphi);
  k[2] = (double)(-(T)0.5 * (dU_tt_r * ptpt + dU_tp_r * ptpp + dU_rr_r * prpr + dU_hh_r * phph +
                            dU_pp_r * pppp));
  k[3] = (double)(-(T)0.5 * (dU_tt_t * ptpt + dU_tp_t * ptpp + dU_rr_t * prpr + dU_hh_t * phph +
                            dU_pp_t * pppp));
}

// Analytic KS gradient for the mixed-precision tracer.  With
// g^ab = eta^ab - H l^a l^b (ingoing, knds_metric.hpp:202-218) the
// Hamiltonian is H_ham = (eta^ab p_a p_b)/2 - H ell^2/2 with
// ell = l^a p_a = -p_T + u/D + Z p_Z/r, u = (rX + aY) p_X + (rY - aX) p_Y,
// D = r^2 + a^2, H = (2Mr - Q^2)/rho2, rho2 = r^2 + a^2 Z^2/r^2, and r(X,Y,Z)
// the root of r^4 - (R^2 - a^2) r^2 - a^2 Z^2 = 0, whose gradient is
// dr/dX = X r/E, dr/dY = Y r/E, dr/dZ = Z (r^2+a^2)/(r E), E = 2r^2-(R^2-a^2).
// dx/dlam = p - H ell l, dp/dlam = -grad H_ham = (grad H) ell^2/2 + H ell grad ell.
template <class T>
KT_HD void ks_rhs_analytic(const Metric& g, double X_, double Y_, double Z_, double pX_,
                           double pY_, double pZ_, double pT_, double k[6]) {
  const T X = (T)X_, Y = (T)Y_, Z = (T)Z_, pX = (T)pX_, pY = (T)pY_, pZ = (T)pZ_, pT = (T)pT_;
  const T a = (T)g.a, a2 = (T)g.a2, M = (T)g.M, Q2 = (T)g.Q2;
  const T R2 = X * X + Y * Y + Z * Z;
  const T b = R2 - a2;
  const T r = sqrt((T)0.5 * (b + sqrt(b * b + (T)4 * a2 * Z * Z)));
  const T r2 = r * r;
  const T ir = mx_rcp(r);
  const T D = r2 + a2;
  const T iD = mx_rcp(D);
  const T iE = mx_rcp((T)2 * r2 - b);
  const T drX = X * r * iE, drY = Y * r * iE, drZ = Z * D * ir * iE;
  const T rho2 = r2 + a2 * Z * Z * ir * ir;
  const T irho2 = mx_rcp(rho2);
  const T N = (T)2 * M * r - Q2;
  const T H = N * irho2;
  const T l1 = (r * X + a * Y) * iD, l2 = (r * Y - a * X) * iD, l3 = Z * ir;
  const T u = (r * X + a * Y) * pX + (r * Y - a * X) * pY;
  const T ell = -pT + u * iD + Z * pZ * ir;
  const T w = X * pX + Y * pY;
  // d(rho2), dH, d(ell) for x_i = X, Y, Z
  const T dr[3] = {drX, drY, drZ};
  const T du[3] = {drX * w + r * pX - a * pY, drY * w + a * pX + r * pY, drZ * w};
  const T Hl = H * ell;
  k[0] = (double)(pX - Hl * l1);
  k[1] = (double)(pY - Hl * l2);
  k[2] = (double)(pZ - Hl * l3);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T drho2 = (T)2 * r * dr[i] + a2 * ((i == 2 ? (T)2 * Z : (T)0) * ir * ir -
                                              (T)2 * Z * Z * ir * ir * ir * dr[i]);
    const T dH = ((T)2 * M * dr[i] - H * drho2) * irho2;
    const T dD = (T)2 * r * dr[i];
    const T dell = (du[i] - u * iD * dD) * iD +
                   pZ * ((i == 2 ? r : (T)0) - Z * dr[i]) * ir * ir;
    k[3 + i] = (double)((T)0.5 * dH * ell * ell + Hl * dell);
  }
}

// keplerian_omega, knds_metric.hpp:354-363
KT_HD double kepler_omega(const Metric& g, double r) {
  const double s = (g.a < 0.0) ? 1.0 : -1.0;
  const double Meff = (g.M - g.Q2 / (2.0 * r)) + (((g.L * g.a) * r) * r) / 3.0;
  const double sq = sqrt(dmax(Meff, 0.0));
  const double den = r * sqrt(r) + (s * g.a) * sq;
  if (fabs(den) < 1e-14) return 0.0;
  return (s * sq) / den;
}

// disk_redshift, main.cpp:329-341 (equatorial metric: Ang at pi/2 given).
KT_HD double disk_redshift(const Metric& g, const Ang& eq, double r, double pt, double pphi) {
  const double Om = kepler_omega(g, r);
  const double b = (-pphi) / (-pt);
  const Cov G = bl_cov(g, r, eq);
  const double d2 = -((G.tt + (2.0 * G.tp) * Om) + (G.pp * Om) * Om);
  if (d2 <= 0.0) return 1.0;
  const double dv = fabs(1.0 - Om * b);
  if (dv < 1e-8) return 20.0;
  const double red = sqrt(d2) / dv;
  return finite(red) ? red : 1.0;
}

// Bundle-mode redshift (ray_bundle.hpp:367-378): signed Doppler factor.
KT_HD double bundle_redshift(const Metric& g, const Ang& eq, double r, double pt, double pphi) {
  const double Om = kepler_omega(g, r);
  const double b = (-pphi) / (-pt);
  const Cov G = bl_cov(g, r, eq);
  const double d2 = -((G.tt + (2.0 * G.tp) * Om) + (G.pp * Om) * Om);
  const double dv = 1.0 - Om * b;
  double red = (d2 > 0.0 && fabs(dv) > 1e-10) ? sqrt(d2) / dv : 1.0;
  red = red < 0.0 ? 0.0 : red > 20.0 ? 20.0 : red;
  return red;
}

// ---------------------------------------------- separable Kerr (Q = Lambda = 0)
// The semi-analytic solver's first integrals and potentials
// (main.cpp:440-504): E = -p_t, L_z = p_phi, Carter's Q_c; R(r) and
// Theta(theta); dr, dtheta carry the branch signs, dphi is sign-free.

struct SepConst {
  double M, a, E, Lz, Qc;
};

// Delta = r^2 - 2 M r + a^2 (main.cpp:470-472)
KT_HD double sep_delta(const SepConst& c, double r) { return (r * r - (2.0 * c.M) * r) + c.a * c.a; }

// R(r) = P^2 - Delta (Q_c + (L_z - a E)^2), P = E (r^2 + a^2) - a L_z (main.cpp:474-479)
KT_HD double sep_R(const SepConst& c, double r) {
  const double P = c.E * (r * r + c.a * c.a) - c.a * c.Lz;
  const double u = c.Lz - c.a * c.E;
  return P * P - sep_delta(c, r) * (c.Qc + u * u);
}

// Theta(theta) = Q_c - cos^2 (L_z^2 / max(sin^2, 1e-14) - a^2 E^2) (main.cpp:481-486)
KT_HD double sep_Theta_sc(const SepConst& c, double st, double ct) {
  const double st2 = dmax(st * st, 1e-14);
  return c.Qc - (ct * ct) * ((c.Lz * c.Lz) / st2 - ((c.a * c.a) * c.E) * c.E);
}
KT_HD double sep_Theta(const SepConst& c, double th) {
  double st, ct;
  ktm_sincos(th, &st, &ct);
  return sep_Theta_sc(c, st, ct);
}

// init_separable_consts (main.cpp:454-468) for a Kerr frame: false when
// E = -p_t is not a positive finite number or Q_c is not finite.
KT_HD bool sep_init(const Metric& g, double th, double pth, double pt, double pphi, SepConst* c) {
  c->M = g.M;
  c->a = g.a;
  c->E = -pt;
  c->Lz = pphi;
  if (!(finite(c->E) && finite(c->Lz) && c->E > 0.0)) return false;
  double st, ct;
  ktm_sincos(th, &st, &ct);
  const double st2 = dmax(st * st, 1e-14);
  c->Qc = pth * pth + (ct * ct) * ((c->Lz * c->Lz) / st2 - ((c->a * c->a) * c->E) * c->E);
  return finite(c->Qc);
}

// kerr_sep_rhs (main.cpp:488-504): k = {dr, dtheta, dphi}; false when any
// of them is not finite.  sr, sth: branch signs (>= 0 counts as +).
KT_HD bool sep_rhs(const SepConst& c, double r, double th, int sr, int sth, double k[3]) {
  double st, ct;
  ktm_sincos(th, &st, &ct);
  const double st2 = dmax(st * st, 1e-14);
  const double sig = dmax(r * r + ((c.a * c.a) * ct) * ct, 1e-14);
  const double del = sep_delta(c, r);
  const double P = c.E * (r * r + c.a * c.a) - c.a * c.Lz;
  const double R = sep_R(c, r);
  const double T = sep_Theta_sc(c, st, ct);
  k[0] = ((sr >= 0) ? 1.0 : -1.0) * sqrt(dmax(R, 0.0)) / sig;
  k[1] = ((sth >= 0) ? 1.0 : -1.0) * sqrt(dmax(T, 0.0)) / sig;
  k[2] = (c.Lz / st2 + c.a * (P / dmax(del, 1e-14) - c.E)) / sig;
  return finite(k[0]) && finite(k[1]) && finite(k[2]);
}

// ------------------------------------------------------------------ events
// geodesic.hpp:49-140

KT_HD double clamp01(double x) {
  if (x < 0.0) return 0.0;
  if (x > 1.0) return 1.0;
  return x;
}

KT_HD double hermite(double y0, double y1, double dy0, double dy1, double h, double alpha) {
  alpha = clamp01(alpha);
  const double a2 = alpha * alpha;
  const double a3 = a2 * alpha;
  const double h00 = (2.0 * a3 - 3.0 * a2) + 1.0;
  const double h10 = (a3 - 2.0 * a2) + alpha;
  const double h01 = -2.0 * a3 + 3.0 * a2;
  const double h11 = a3 - a2;
  return ((h00 * y0 + h10 * (h * dy0)) + h01 * y1) + h11 * (h * dy1);
}

KT_HD bool sign_change(double f0, double f1) {
  return ((f0 <= 0.0 && f1 >= 0.0) || (f0 >= 0.0 && f1 <= 0.0));
}

// first_event_alpha_hermite with 8 bins x 8 bisections (geodesic.hpp:98-140).
KT_HD bool first_event(double y0, double y1, double dy0, double dy1, double h, double target,
                       double* alpha_out) {
  const double f_eps = 1e-12;
  double a0 = 0.0;
  double f0 = y0 - target;
  if (fabs(f0) <= f_eps) {
    *alpha_out = 0.0;
    return true;
  }
  for (int i = 1; i <= 8; ++i) {
    const double a1 = (double)i / 8.0;
    const double f1 = (i == 8) ? (y1 - target) : (hermite(y0, y1, dy0, dy1, h, a1) - target);
    if (fabs(f1) <= f_eps) {
      *alpha_out = a1;
      return true;
    }
    if (sign_change(f0, f1)) {
      double lo = a0, hi = a1;
      for (int k = 0; k < 8; ++k) {
        const double mid = 0.5 * (lo + hi);
        const double fm = hermite(y0, y1, dy0, dy1, h, mid) - target;
        if (sign_change(f0, fm))
          hi = mid;
        else
          lo = mid;
      }
      *alpha_out = 0.5 * (lo + hi);
      return true;
    }
    a0 = a1;
    f0 = f1;
  }
  return false;
}

// ------------------------------------------------------------------ camera
// camera.hpp:38-145.  The observer's metric is a frame constant.
struct CamConst {
  double r_obs, theta_obs, phi_obs, fov_h;
  int W, H;
  double half_wm1, half_hm1, span;  // 0.5*(W-1), 0.5*(H-1), (double)span
  double offx, offy;
  double gtt, gtphi, grr, gthth, gphph;  // g_{mu nu} at the observer
  double Utt, Utp, Urr, Uhh, Upp;        // g^{mu nu} at the observer
  double sqrt_grr, sqrt_gthth, inv_guard_grr, inv_guard_gthth, sqrt_gphph_guard;
  double ut, ephi_p, ephi_t;
  int tetrad_ok;
  int pad0;
};

KT_HD CamConst make_camera(const Metric& g, double r_obs, double theta_obs, double phi_obs,
                           double fov_h, int W, int H, double offx, double offy) {
  CamConst c;
  c.r_obs = r_obs;
  c.theta_obs = theta_obs;
  c.phi_obs = phi_obs;
  c.fov_h = fov_h;
  c.W = W;
  c.H = H;
  c.half_wm1 = 0.5 * (double)(W - 1);
  c.half_hm1 = 0.5 * (double)(H - 1);
  c.span = (double)((W > 1) ? (W - 1) : 1);
  c.offx = offx;
  c.offy = offy;
  const Ang A = bl_ang(g, theta_obs);
  const Cov G = bl_cov(g, r_obs, A);
  const Inv U = bl_inv(g, r_obs, A);
  c.gtt = G.tt;
  c.gtphi = G.tp;
  c.grr = G.rr;
  c.gthth = G.hh;
  c.gphph = G.pp;
  c.Utt = U.tt;
  c.Utp = U.tp;
  c.Urr = U.rr;
  c.Uhh = U.hh;
  c.Upp = U.pp;
  c.sqrt_grr = sqrt(fabs(G.rr));
  c.sqrt_gthth = sqrt(fabs(G.hh));
  c.inv_guard_grr = dmax(c.sqrt_grr, 1e-14);
  c.inv_guard_gthth = dmax(c.sqrt_gthth, 1e-14);
  c.sqrt_gphph_guard = sqrt(dmax(fabs(G.pp), 1e-14));
  const double denom_phi = G.pp - (G.tp * G.tp) / G.tt;
  c.tetrad_ok = (G.tt < -1e-14) && finite(denom_phi) && (denom_phi > 1e-14) &&
                finite(c.sqrt_grr) && (c.sqrt_grr > 1e-14) && finite(c.sqrt_gthth) &&
                (c.sqrt_gthth > 1e-14);
  c.ut = 1.0 / sqrt(-G.tt);
  c.ephi_p = 1.0 / sqrt(denom_phi);
  c.ephi_t = ((-G.tp) / G.tt) * c.ephi_p;
  c.pad0 = 0;
  return c;
}

// pixel_ray's angles (camera.hpp:38-47).
KT_HD void pixel_angles(const CamConst& c, int px, int py, double* alpha, double* beta) {
  const double x = (double)px + c.offx;
  const double y = (double)py + c.offy;
  *alpha = (c.fov_h * (x - c.half_wm1)) / c.span;
  *beta = (c.fov_h * (c.half_hm1 - y)) / c.span;
}

// GeodesicState (geodesic.hpp:33-37)
struct Geo {
  double r, th, ph, pr, pth, pt, pphi;
};

// angle_ray (camera.hpp:50-145)
KT_HD Geo angle_ray(const CamConst& c, double alpha, double beta) {
  double sa, ca, sb, cb;
  ktm_sincos(alpha, &sa, &ca);
  ktm_sincos(beta, &sb, &cb);
  double pUt = 1.0;
  double pUr = ((-ca) * cb) / c.inv_guard_grr;
  double pUth = (-sb) / c.inv_guard_gthth;
  double pUphi = ((-sa) * cb) / c.sqrt_gphph_guard;
  if (c.tetrad_ok) {
    const double n_r = (-ca) * cb;
    const double n_th = -sb;
    const double n_ph = (-sa) * cb;
    pUt = c.ut + n_ph * c.ephi_t;
    pUr = n_r / c.sqrt_grr;
    pUth = n_th / c.sqrt_gthth;
    pUphi = n_ph * c.ephi_p;
  }
  double pt = c.gtt * pUt + c.gtphi * pUphi;
  const double pr = c.grr * pUr;
  const double pth = c.gthth * pUth;
  const double pphi = c.gtphi * pUt + c.gphph * pUphi;
  const double A = c.Utt;
  const double B = (2.0 * c.Utp) * pphi;
  const double C = ((c.Urr * pr) * pr + (c.Uhh * pth) * pth) + (c.Upp * pphi) * pphi;
  const double disc = B * B - (4.0 * A) * C;
  if (disc >= 0.0 && fabs(A) > 1e-15) {
    const double sq = sqrt(disc);
    const double pt1 = (-B - sq) / (2.0 * A);
    const double pt2 = (-B + sq) / (2.0 * A);
    pt = (pt1 < 0.0) ? pt1 : pt2;
    if (pt > 0.0) pt = dmin(pt1, pt2);
  }
  Geo s;
  s.r = c.r_obs;
  s.th = c.theta_obs;
  s.ph = c.phi_obs;
  s.pr = pr;
  s.pth = pth;
  s.pt = pt;
  s.pphi = pphi;
  return s;
}

// ---------------------------------------------------------------- KS chart
// knds_metric.hpp:150-230 (ingoing, Lambda = 0), main.cpp:1306-1454

KT_HD double r_ks(const Metric& g, double X, double Y, double Z) {
  const double R2 = (X * X + Y * Y) + Z * Z;
  const double b = R2 - g.a2;
  return sqrt(0.5 * (b + sqrt(b * b + (g.fa2 * Z) * Z)));
}

// g^{ab} = eta^{ab} - H l^a l^b, all 16 entries in the reference's
// evaluation order (the product (H l^a) l^b is not symmetric in rounding).
KT_HD void ks_inv(const Metric& g, double X, double Y, double Z, double G[16]) {
  const double r = r_ks(g, X, Y, Z);
  const double r_sq = r * r;
  const double rho2 = r_sq + ((g.a2 * Z) * Z) / r_sq;
  const double H = (g.twoM * r - g.Q2) / rho2;
  const double r2a2 = r_sq + g.a2;
  const double lU[4] = {-1.0, (r * X + g.a * Y) / r2a2, (r * Y - g.a * X) / r2a2, Z / r};
#pragma unroll
  for (int mu = 0; mu < 4; ++mu) {
    const double hl = H * lU[mu];
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
      const double eta = (mu != nu) ? 0.0 : (mu == 0 ? -1.0 : 1.0);
      G[4 * mu + nu] = eta - hl * lU[nu];
    }
  }
}

KT_HD double ks_ham(const double G[16], const double p[4]) {
  double H = 0.0;
#pragma unroll
  for (int mu = 0; mu < 4; ++mu)
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) H += (G[4 * mu + nu] * p[mu]) * p[nu];
  return 0.5 * H;
}

struct KSState {
  double X, Y, Z, pX, pY, pZ, pT;
};

// geodesic_rhs_ks, main.cpp:1432-1454.  k = {dX, dY, dZ, dpX, dpY, dpZ}.
// The centre and the six finite-difference points share one rolled loop.
KT_HD void ks_rhs(const Metric& g, double X, double Y, double Z, double pX, double pY, double pZ,
                  double pT, double k[6]) {
  const double p[4] = {pT, pX, pY, pZ};
  const double eX = 1e-5 * (fabs(X) + 0.1);
  const double eY = 1e-5 * (fabs(Y) + 0.1);
  const double eZ = 1e-5 * (fabs(Z) + 0.1);
  double h1 = 0.0, h2 = 0.0, h3 = 0.0, h4 = 0.0, h5 = 0.0, h6 = 0.0;
  KT_ROLLED
  for (int i = 0; i < 7; ++i) {
    const double x = (i == 1) ? X + eX : (i == 2) ? X - eX : X;
    const double y = (i == 3) ? Y + eY : (i == 4) ? Y - eY : Y;
    const double z = (i == 5) ? Z + eZ : (i == 6) ? Z - eZ : Z;
    double G[16];
    ks_inv(g, x, y, z, G);
    if (i == 0) {
      k[0] = ((G[4] * pT + G[5] * pX) + G[6] * pY) + G[7] * pZ;
      k[1] = ((G[8] * pT + G[9] * pX) + G[10] * pY) + G[11] * pZ;
      k[2] = ((G[12] * pT + G[13] * pX) + G[14] * pY) + G[15] * pZ;
    } else {
      const double h = ks_ham(G, p);
      h1 = (i == 1) ? h : h1;
      h2 = (i == 2) ? h : h2;
      h3 = (i == 3) ? h : h3;
      h4 = (i == 4) ? h : h4;
      h5 = (i == 5) ? h : h5;
      h6 = (i == 6) ? h : h6;
    }
  }
  k[3] = -(h1 - h2) / (2.0 * eX);
  k[4] = -(h3 - h4) / (2.0 * eY);
  k[5] = -(h5 - h6) / (2.0 * eZ);
}

// BL_to_KS_spatial (knds_metric.hpp:368-387) from precomputed sin/cos.
KT_HD void bl_to_ks_sc(double r, double st, double ct, double sf, double cf, double a, double* X,
                       double* Y, double* Z) {
  *X = st * (r * cf - a * sf);
  *Y = st * (r * sf + a * cf);
  *Z = r * ct;
}

// KS_to_BL_spatial (knds_metric.hpp:390-411); the reference's first atan2
// results are overwritten before use.
KT_HD void ks_to_bl(const Metric& g, double X, double Y, double Z, double* r, double* th,
                    double* ph) {
  const double rr = r_ks(g, X, Y, Z);
  *r = rr;
  const double Zr = Z / rr;
  *th = ktm_acos(Zr < -1.0 ? -1.0 : Zr > 1.0 ? 1.0 : Zr);
  const double st_val = sqrt(dmax(1.0 - (Z * Z) / (rr * rr), 0.0));
  const double r2a2 = rr * rr + g.a2;
  if (st_val > 1e-10) {
    const double cf = (X * rr + Y * g.a) / (st_val * r2a2);
    const double sf = (Y * rr - X * g.a) / (st_val * r2a2);
    *ph = ktm_atan2(sf, cf);
  } else {
    *ph = 0.0;
  }
}

// jacobian_bl_to_ks, main.cpp:1348-1371: J[i][j] = d(X,Y,Z)_i / d(r,th,ph)_j.
KT_HD void jacobian_bl_to_ks(double r, double th, double ph, double a, double J[3][3]) {
  const double er = 1e-6 * (fabs(r) + 1.0);
  const double eth = 1e-6;
  const double eph = 1e-6;
  double st, ct, sf, cf, st_p, ct_p, st_m, ct_m, sf_p, cf_p, sf_m, cf_m;
  ktm_sincos(th, &st, &ct);
  ktm_sincos(ph, &sf, &cf);
  ktm_sincos(th + eth, &st_p, &ct_p);
  ktm_sincos(th - eth, &st_m, &ct_m);
  ktm_sincos(ph + eph, &sf_p, &cf_p);
  ktm_sincos(ph - eph, &sf_m, &cf_m);
  double p[6][3];
  bl_to_ks_sc(r + er, st, ct, sf, cf, a, &p[0][0], &p[0][1], &p[0][2]);
  bl_to_ks_sc(r - er, st, ct, sf, cf, a, &p[1][0], &p[1][1], &p[1][2]);
  bl_to_ks_sc(r, st_p, ct_p, sf, cf, a, &p[2][0], &p[2][1], &p[2][2]);
  bl_to_ks_sc(r, st_m, ct_m, sf, cf, a, &p[3][0], &p[3][1], &p[3][2]);
  bl_to_ks_sc(r, st, ct, sf_p, cf_p, a, &p[4][0], &p[4][1], &p[4][2]);
  bl_to_ks_sc(r, st, ct, sf_m, cf_m, a, &p[5][0], &p[5][1], &p[5][2]);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    J[i][0] = (p[0][i] - p[1][i]) / (2.0 * er);
    J[i][1] = (p[2][i] - p[3][i]) / (2.0 * eth);
    J[i][2] = (p[4][i] - p[5][i]) / (2.0 * eph);
  }
}

// solve_3x3 with partial pivoting, main.cpp:1314-1346.
KT_HD bool solve_3x3(const double Ain[3][3], const double bin[3], double x[3]) {
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
    if (best < 1e-14) return false;
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
  return true;
}

// init_ks_state, main.cpp:1404-1430.  Lambda = 0 is checked by the caller.
KT_HD bool init_ks_state(const Metric& g, const Geo& sb, KSState* k) {
  double st, ct, sf, cf;
  ktm_sincos(sb.th, &st, &ct);
  ktm_sincos(sb.ph, &sf, &cf);
  bl_to_ks_sc(sb.r, st, ct, sf, cf, g.a, &k->X, &k->Y, &k->Z);
  double J[3][3], A3[3][3];
  jacobian_bl_to_ks(sb.r, sb.th, sb.ph, g.a, J);
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) A3[j][i] = J[i][j];
  const double b3[3] = {sb.pr, sb.pth, sb.pphi};
  double x3[3];
  if (!solve_3x3(A3, b3, x3)) return false;
  k->pX = x3[0];
  k->pY = x3[1];
  k->pZ = x3[2];
  double G[16];
  ks_inv(g, k->X, k->Y, k->Z, G);
  const double A = G[0];
  const double B = 2.0 * ((G[1] * k->pX + G[2] * k->pY) + G[3] * k->pZ);
  const double C = (((((G[5] * k->pX) * k->pX + (G[10] * k->pY) * k->pY) + (G[15] * k->pZ) * k->pZ) +
                     ((2.0 * G[6]) * k->pX) * k->pY) +
                    ((2.0 * G[7]) * k->pX) * k->pZ) +
                   ((2.0 * G[11]) * k->pY) * k->pZ;
  const double disc = B * B - (4.0 * A) * C;
  if (disc < 0.0 || fabs(A) < 1e-15) return false;
  const double sq = sqrt(disc);
  const double pT1 = (-B - sq) / (2.0 * A);
  const double pT2 = (-B + sq) / (2.0 * A);
  k->pT = (pT1 < 0.0) ? pT1 : pT2;
  if (k->pT > 0.0) k->pT = dmin(pT1, pT2);
  return finite(k->pT);
}

// ks_covector_to_bl's p_phi component (main.cpp:1391-1402).
KT_HD double ks_pphi_bl(double r, double th, double ph, double a, double pX, double pY,
                        double pZ) {
  double J[3][3];
  jacobian_bl_to_ks(r, th, ph, a, J);
  double s = 0.0;
  s += J[0][2] * pX;
  s += J[1][2] * pY;
  s += J[2][2] * pZ;
  return s;
}

// --------------------------------------------------------------- bundles
// ray_bundle.hpp:56-214.  Hessian of H by central differences: the 33
// evaluations fall on 9 distinct (r, theta) points, so 9 g^{mu nu}; the
// centre's (U00) and its angle factors come from bl_rhs_centre.
KT_HD void bundle_hessian(const Metric& g, double r, double th, double pr, double pth, double pt,
                          double pphi, const Ang& A0, const Inv& U00, double Hs[4][4]) {
  const double e0 = 1e-5 * (fabs(r) + 0.1);
  const double e1 = 1e-5;
  const double e2 = 1e-5 * (fabs(pr) + 1e-3);
  const double e3 = 1e-5 * (fabs(pth) + 1e-3);
  const Ang Ap = bl_ang<false>(g, th + e1);
  const Ang Am = bl_ang<false>(g, th + (-e1));
  const double rp = r + e0, rm = r + (-e0);
  const double prp = pr + e2, prm = pr + (-e2);
  const double pthp = pth + e3, pthm = pth + (-e3);
  // g^{mu nu} at (r + {0,+,-}e0, theta + {0,+,-}e1)
  const Inv Up0 = bl_inv<false>(g, rp, A0), Um0 = bl_inv<false>(g, rm, A0);
  const Inv U0p = bl_inv<false>(g, r, Ap), U0m = bl_inv<false>(g, r, Am);
  const Inv Upp = bl_inv<false>(g, rp, Ap), Upm = bl_inv<false>(g, rp, Am);
  const Inv Ump = bl_inv<false>(g, rm, Ap), Umm = bl_inv<false>(g, rm, Am);
  const double H0 = bl_ham(U00, pr, pth, pt, pphi);
  const double e[4] = {e0, e1, e2, e3};
  double vp[4], vm[4];
  vp[0] = bl_ham(Up0, pr, pth, pt, pphi);
  vm[0] = bl_ham(Um0, pr, pth, pt, pphi);
  vp[1] = bl_ham(U0p, pr, pth, pt, pphi);
  vm[1] = bl_ham(U0m, pr, pth, pt, pphi);
  vp[2] = bl_ham(U00, prp, pth, pt, pphi);
  vm[2] = bl_ham(U00, prm, pth, pt, pphi);
  vp[3] = bl_ham(U00, pr, pthp, pt, pphi);
  vm[3] = bl_ham(U00, pr, pthm, pt, pphi);
#pragma unroll
  for (int a = 0; a < 4; ++a) Hs[a][a] = ((vp[a] - 2.0 * H0) + vm[a]) / (e[a] * e[a]);
  // cross(a,b) = (pp - pm - mp + mm) / (4 e_a e_b)
#define KT_CROSS(a, b, pp, pm, mp, mm) \
  Hs[a][b] = Hs[b][a] = ((((pp) - (pm)) - (mp)) + (mm)) / ((4.0 * e[a]) * e[b])
  KT_CROSS(0, 1, bl_ham(Upp, pr, pth, pt, pphi), bl_ham(Upm, pr, pth, pt, pphi),
           bl_ham(Ump, pr, pth, pt, pphi), bl_ham(Umm, pr, pth, pt, pphi));
  KT_CROSS(0, 2, bl_ham(Up0, prp, pth, pt, pphi), bl_ham(Up0, prm, pth, pt, pphi),
           bl_ham(Um0, prp, pth, pt, pphi), bl_ham(Um0, prm, pth, pt, pphi));
  KT_CROSS(0, 3, bl_ham(Up0, pr, pthp, pt, pphi), bl_ham(Up0, pr, pthm, pt, pphi),
           bl_ham(Um0, pr, pthp, pt, pphi), bl_ham(Um0, pr, pthm, pt, pphi));
  KT_CROSS(1, 2, bl_ham(U0p, prp, pth, pt, pphi), bl_ham(U0p, prm, pth, pt, pphi),
           bl_ham(U0m, prp, pth, pt, pphi), bl_ham(U0m, prm, pth, pt, pphi));
  KT_CROSS(1, 3, bl_ham(U0p, pr, pthp, pt, pphi), bl_ham(U0p, pr, pthm, pt, pphi),
           bl_ham(U0m, pr, pthp, pt, pphi), bl_ham(U0m, pr, pthm, pt, pphi));
  KT_CROSS(2, 3, bl_ham(U00, prp, pthp, pt, pphi), bl_ham(U00, prp, pthm, pt, pphi),
           bl_ham(U00, prm, pthp, pt, pphi), bl_ham(U00, prm, pthm, pt, pphi));
#undef KT_CROSS
}

// bundle_rhs (ray_bundle.hpp:130-156): geodesic RHS (k[0..4] as bl_rhs) and
// dW = J_s Hess W (dW[i][k], 4x2).
KT_HD void bundle_rhs(const Metric& g, double r, double th, double pr, double pth, double pt,
                      double pphi, const double W[8], double k[5], double dW[8]) {
  Ang A0;
  Inv U00;
  bl_rhs_centre<false>(g, r, th, pr, pth, pt, pphi, k, &A0, &U00);
  double Hs[4][4];
  bundle_hessian(g, r, th, pr, pth, pt, pphi, A0, U00, Hs);
  double M[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    M[0][j] = Hs[2][j];
    M[1][j] = Hs[3][j];
    M[2][j] = -Hs[0][j];
    M[3][j] = -Hs[1][j];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) s += M[i][j] * W[2 * j + c];
      dW[2 * i + c] = s;
    }
}

// The bundle RHS split over the two lanes of a ray (the paired bundle kernel,
// two threads per ray).  Both lanes run the same instructions on
// lane-dependent inputs, so the warp never diverges: each evaluates 3 of the
// 5 angle factors (theta itself on both), 7 of the 13 inverse metrics (the
// centre's on both) and 19 of the 37 Hamiltonians of bundle_rhs, and
// bundle_rhs_combine assembles the RHS from the two halves in bundle_rhs's
// own operation order, so the result is bit-identical to it.
//
// Inverse metrics, lane 0 | lane 1 (rp = r + e0, rm = r + (-e0)):
//   t0 (r, theta) both        t1 (rp | rm, theta)      t2 (r, theta +e1 | +(-e1))
//   t3 (r + eps_r | r - eps_r, theta)                  t4 (r, theta + eps_th | - eps_th)
//   t5 (rp, theta +e1 | +(-e1))                        t6 (rm, theta +e1 | +(-e1))
// Momenta of the Hamiltonians of t0..t2: (pr, pth), (prp, pth), (prm, pth),
// (pr, pthp), (pr, pthm); at t0 lane 1 takes the four corners (prp, pthp),
// (prp, pthm), (prm, pthp), (prm, pthm) of the (2,3) cross term instead.
// t3..t6 take (pr, pth).
struct BundleHalf {
  double h5[3][5];  // t0..t2
  double h1[4];     // t3..t6
  double k0, k1, k4;  // dr, dtheta, dphi from the centre's g^{mu nu}
};

#ifndef KT_BUNDLE_HALF_ROLLED
#define KT_BUNDLE_HALF_ROLLED 1
#endif

// Code shape of the split (kRolled): the angle factors, the three
// five-Hamiltonian inverse metrics and the four one-Hamiltonian ones in
// rolled loops (one copy of bl_ang, two of bl_inv, six of bl_ham: the paired
// kernel's instruction fetch), or everything unrolled.  Same arithmetic.
template <bool kRolled = (KT_BUNDLE_HALF_ROLLED != 0)>
KT_HD void bundle_rhs_half(const Metric& g, double r, double th, double pr, double pth, double pt,
                           double pphi, bool odd, BundleHalf* o);

template <>
KT_HD void bundle_rhs_half<true>(const Metric& g, double r, double th, double pr, double pth,
                                 double pt, double pphi, bool odd, BundleHalf* o) {
  const double sgn = odd ? -1.0 : 1.0;
  const double eps_r = 1e-5 * dmax(fabs(r), 0.01);
  const double eps_th = 1e-6;
  const double e0 = 1e-5 * (fabs(r) + 0.1);
  const double e1 = 1e-5;
  const double e2 = 1e-5 * (fabs(pr) + 1e-3);
  const double e3 = 1e-5 * (fabs(pth) + 1e-3);
  Ang A[3];  // theta; theta + e1 | + (-e1); theta + eps_th | - eps_th
  KT_ROLLED
  for (int j = 0; j < 3; ++j) {
    const double x = (j == 0) ? th : th + sgn * ((j == 1) ? e1 : eps_th);
    A[j] = bl_ang<false>(g, x);
  }
  const double rp = r + e0, rm = r + (-e0);
  const double prp = pr + e2, prm = pr + (-e2);
  const double pthp = pth + e3, pthm = pth + (-e3);
  // t0..t2: five Hamiltonians each (lane 1 at t0: the (2,3) corners)
  KT_ROLLED
  for (int t = 0; t < 3; ++t) {
    const double rad = (t == 1) ? (odd ? rm : rp) : r;
    const Inv U = bl_inv<false>(g, rad, A[t == 2 ? 1 : 0]);
    if (t == 0) {
      o->k0 = U.rr * pr;
      o->k1 = U.hh * pth;
      o->k4 = U.tp * pt + U.pp * pphi;
    }
    const bool c23 = (t == 0) && odd;
    o->h5[t][0] = bl_ham(U, c23 ? prp : pr, c23 ? pthp : pth, pt, pphi);
    o->h5[t][1] = bl_ham(U, prp, c23 ? pthm : pth, pt, pphi);
    o->h5[t][2] = bl_ham(U, prm, c23 ? pthp : pth, pt, pphi);
    o->h5[t][3] = bl_ham(U, c23 ? prm : pr, c23 ? pthm : pthp, pt, pphi);
    o->h5[t][4] = bl_ham(U, c23 ? prm : pr, pthm, pt, pphi);
  }
  // t3..t6: one Hamiltonian each
  KT_ROLLED
  for (int t = 0; t < 4; ++t) {
    const double rad = (t == 0) ? (odd ? r - eps_r : r + eps_r) : (t == 1) ? r : (t == 2) ? rp : rm;
    o->h1[t] = bl_ham(bl_inv<false>(g, rad, A[t == 1 ? 2 : (t == 0 ? 0 : 1)]), pr, pth, pt, pphi);
  }
}

template <>
KT_HD void bundle_rhs_half<false>(const Metric& g, double r, double th, double pr, double pth,
                                  double pt, double pphi, bool odd, BundleHalf* o) {
  const double sgn = odd ? -1.0 : 1.0;
  const double eps_r = 1e-5 * dmax(fabs(r), 0.01);
  const double eps_th = 1e-6;
  const double e0 = 1e-5 * (fabs(r) + 0.1);
  const double e1 = 1e-5;
  const double e2 = 1e-5 * (fabs(pr) + 1e-3);
  const double e3 = 1e-5 * (fabs(pth) + 1e-3);
  const Ang A0 = bl_ang<false>(g, th);
  const Ang A1 = bl_ang<false>(g, th + sgn * e1);       // theta + e1 | theta + (-e1)
  const Ang A2 = bl_ang<false>(g, th + sgn * eps_th);   // theta + eps_th | theta - eps_th
  const double rp = r + e0, rm = r + (-e0);
  const double prp = pr + e2, prm = pr + (-e2);
  const double pthp = pth + e3, pthm = pth + (-e3);
  // t0: the centre; its Hamiltonians: lane 0 H0, the e2 and e3 pairs; lane 1
  // the (2,3) corners (its fifth value repeats the fourth)
  {
    const Inv U = bl_inv<false>(g, r, A0);
    o->k0 = U.rr * pr;
    o->k1 = U.hh * pth;
    o->k4 = U.tp * pt + U.pp * pphi;
    o->h5[0][0] = bl_ham(U, odd ? prp : pr, odd ? pthp : pth, pt, pphi);
    o->h5[0][1] = bl_ham(U, prp, odd ? pthm : pth, pt, pphi);
    o->h5[0][2] = bl_ham(U, prm, odd ? pthp : pth, pt, pphi);
    o->h5[0][3] = bl_ham(U, odd ? prm : pr, odd ? pthm : pthp, pt, pphi);
    o->h5[0][4] = bl_ham(U, odd ? prm : pr, pthm, pt, pphi);
  }
  // t1, t2: (rp | rm, theta) and (r, theta + e1 | + (-e1)), five momenta each
  {
    const Inv U = bl_inv<false>(g, odd ? rm : rp, A0);
    o->h5[1][0] = bl_ham(U, pr, pth, pt, pphi);
    o->h5[1][1] = bl_ham(U, prp, pth, pt, pphi);
    o->h5[1][2] = bl_ham(U, prm, pth, pt, pphi);
    o->h5[1][3] = bl_ham(U, pr, pthp, pt, pphi);
    o->h5[1][4] = bl_ham(U, pr, pthm, pt, pphi);
  }
  {
    const Inv U = bl_inv<false>(g, r, A1);
    o->h5[2][0] = bl_ham(U, pr, pth, pt, pphi);
    o->h5[2][1] = bl_ham(U, prp, pth, pt, pphi);
    o->h5[2][2] = bl_ham(U, prm, pth, pt, pphi);
    o->h5[2][3] = bl_ham(U, pr, pthp, pt, pphi);
    o->h5[2][4] = bl_ham(U, pr, pthm, pt, pphi);
  }
  // t3..t6: one Hamiltonian each
  o->h1[0] = bl_ham(bl_inv<false>(g, odd ? r - eps_r : r + eps_r, A0), pr, pth, pt, pphi);
  o->h1[1] = bl_ham(bl_inv<false>(g, r, A2), pr, pth, pt, pphi);
  o->h1[2] = bl_ham(bl_inv<false>(g, rp, A1), pr, pth, pt, pphi);
  o->h1[3] = bl_ham(bl_inv<false>(g, rm, A1), pr, pth, pt, pphi);
}

// The RHS from the two halves (E: lane 0, O: lane 1), bundle_rhs's
// expressions: k as bl_rhs_centre, Hess(H) as bundle_hessian, dW = J_s Hess W.
KT_HD void bundle_rhs_combine(const BundleHalf& E, const BundleHalf& O, double r, double pr,
                              double pth, const double W[8], double k[5], double dW[8]) {
  const double eps_r = 1e-5 * dmax(fabs(r), 0.01);
  const double eps_th = 1e-6;
  k[0] = E.k0;
  k[1] = E.k1;
  k[4] = E.k4;
  k[2] = -(E.h1[0] - O.h1[0]) / (2.0 * eps_r);
  k[3] = -(E.h1[1] - O.h1[1]) / (2.0 * eps_th);
  const double e[4] = {1e-5 * (fabs(r) + 0.1), 1e-5, 1e-5 * (fabs(pr) + 1e-3),
                       1e-5 * (fabs(pth) + 1e-3)};
  const double H0 = E.h5[0][0];
  const double vp[4] = {E.h5[1][0], E.h5[2][0], E.h5[0][1], E.h5[0][3]};
  const double vm[4] = {O.h5[1][0], O.h5[2][0], E.h5[0][2], E.h5[0][4]};
  double Hs[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a) Hs[a][a] = ((vp[a] - 2.0 * H0) + vm[a]) / (e[a] * e[a]);
#define KT_CROSS(a, b, pp, pm, mp, mm) \
  Hs[a][b] = Hs[b][a] = ((((pp) - (pm)) - (mp)) + (mm)) / ((4.0 * e[a]) * e[b])
  KT_CROSS(0, 1, E.h1[2], O.h1[2], E.h1[3], O.h1[3]);
  KT_CROSS(0, 2, E.h5[1][1], E.h5[1][2], O.h5[1][1], O.h5[1][2]);
  KT_CROSS(0, 3, E.h5[1][3], E.h5[1][4], O.h5[1][3], O.h5[1][4]);
  KT_CROSS(1, 2, E.h5[2][1], E.h5[2][2], O.h5[2][1], O.h5[2][2]);
  KT_CROSS(1, 3, E.h5[2][3], E.h5[2][4], O.h5[2][3], O.h5[2][4]);
  KT_CROSS(2, 3, O.h5[0][0], O.h5[0][1], O.h5[0][2], O.h5[0][3]);
#undef KT_CROSS
  double M[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    M[0][j] = Hs[2][j];
    M[1][j] = Hs[3][j];
    M[2][j] = -Hs[0][j];
    M[3][j] = -Hs[1][j];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) s += M[i][j] * W[2 * j + c];
      dW[2 * i + c] = s;
    }
}

// ------------------------------------------------------------------ colour
// main.cpp:153-170, 1663-1687, 1799-1814

// (uint8_t)(double) as g++ on x86-64 performs it: truncate toward zero to a
// 32-bit integer and keep the low byte (values outside [0,256) occur when
// the background interpolation extrapolates).
KT_HD uint8_t to_u8(double v) { return (uint8_t)(int32_t)v; }

KT_HD void blackbody(double T, double log10_50, uint8_t c[3]) {
  T = dclamp(T, 800.0, 4e4);
  const double t = ktm_log10(T / 800.0) / log10_50;
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
  c[0] = to_u8(dclamp(R, 0.0, 1.0) * 255);
  c[1] = to_u8(dclamp(G, 0.0, 1.0) * 255);
  c[2] = to_u8(dclamp(B, 0.0, 1.0) * 255);
}

KT_HD double page_thorne(double r, double r_isco) {
  if (r <= r_isco) return 0.0;
  const double x = sqrt(r_isco / r);
  return (1.0 - x) / ((r * r) * r);
}

KT_HD double tonemap(double x, double exposure, double gamma) {
  x = x * exposure;
  x = x / (1.0 + x);
  return ktm_pow(dclamp(x, 0.0, 1.0), 1.0 / gamma);
}

struct ColourConst {
  double M, r_isco, exposure, gamma, temp_scale;
  double log10_50;  // log10(4e4/800.0), a per-frame constant
  double pt_peak;   // page_thorne(3 r_isco, r_isco)
  // interstellar palette (ColorParams, main.cpp:72-81) and the disk edges
  int palette, rings, sectors, pad0;
  double sigma, hue_offset, r_in, r_out;
};

KT_HD void disk_colour(const ColourConst& cc, double r, double red, double magnif, uint8_t out[3]) {
  const double T = ((6500.0 * cc.temp_scale) * sqrt((6.0 * cc.M) / r)) * dclamp(red, 0.2, 5.0);
  const double pt_norm = page_thorne(r, cc.r_isco);
  double I = (cc.pt_peak > 0.0) ? pt_norm / cc.pt_peak : 0.0;
  const double red_c = dclamp(red, 0.1, 10.0);
  const double lift = 1.0 + 0.85 * dclamp(1.0 - red_c, 0.0, 1.0);
  I *= ktm_pow(red_c, 4.0) * lift;
  I *= dclamp(1.0 / magnif, 0.05, 5.0);
  uint8_t c[3];
  blackbody(T, cc.log10_50, c);
#pragma unroll
  for (int k = 0; k < 3; ++k) out[k] = to_u8(tonemap((c[k] / 255.0) * I, cc.exposure, cc.gamma) * 255);
}

// hsv_to_rgb (main.cpp:1689-1707).
KT_HD void hsv_to_rgb(double h, double s, double v, double out[3]) {
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
  // the reference returns uint8 (x*255 + 0.5 truncated) and blends those
  out[0] = (double)to_u8(rr * 255.0 + 0.5);
  out[1] = (double)to_u8(gg * 255.0 + 0.5);
  out[2] = (double)to_u8(bb * 255.0 + 0.5);
}

// cell_hash (main.cpp:1710-1713): fractional part of a scrambled sine.
KT_HD double cell_hash(int cell_id, double salt_a, double salt_b) {
  const double v = ktm_sin((double)cell_id * salt_a + salt_b) * 43758.5453;
  return v - floor(v);
}

// disk_colour_interstellar (main.cpp:1719-1797): rings x sectors of hashed
// warm colours, Gaussian-blended across cell edges (about 30% of the cells
// are gaps), then the blackbody path's physical intensity.  fmod(x, 1.0) of
// the hue is x - trunc(x), which is exact.
KT_HD void disk_colour_interstellar(const ColourConst& cc, double r, double phi, double red,
                                    double magnif, uint8_t out[3]) {
  const int NR = cc.rings > 0 ? cc.rings : 1;
  const int NS = cc.sectors > 0 ? cc.sectors : 1;
  const double sigma = cc.sigma > 0 ? cc.sigma : 0.5;
  const double two_pi = 2.0 * 3.14159265358979323846;
  const double r_norm = dclamp((r - cc.r_in) / (cc.r_out - cc.r_in), 0.0, 1.0);
  const double phi_norm = (phi - floor(phi / two_pi) * two_pi) / two_pi;
  const double ring_pos = r_norm * (double)NR;
  const double sec_pos = phi_norm * (double)NS;
  double acc_r = 0.0, acc_g = 0.0, acc_b = 0.0, w_total = 0.0;
  const double inv2sig2 = 1.0 / ((2.0 * sigma) * sigma);
  const int SEARCH = (int)ceil(3.0 * sigma) + 1;
  KT_ROLLED
  for (int ri = -SEARCH; ri <= NR + SEARCH; ++ri) {
    const double dr = ring_pos - (double)ri;
    if ((dr * dr) * inv2sig2 > 16.0) continue;
    const int ri_clamped = ri < 0 ? 0 : ri >= NR ? NR - 1 : ri;
    KT_ROLLED
    for (int si_raw = -SEARCH; si_raw <= NS + SEARCH; ++si_raw) {
      double ds = sec_pos - (double)si_raw;
      ds = ds - floor((ds + (double)NS * 0.5) / (double)NS) * (double)NS;
      const double dist2 = dr * dr + ds * ds;
      const double w = ktm_exp(-dist2 * inv2sig2);
      if (w < 1e-4) continue;
      const int si_clamped = ((si_raw % NS) + NS) % NS;
      const int cell_id = ri_clamped * NS + si_clamped;
      const double h1 = cell_hash(cell_id, 127.1, 311.7);
      const double h2 = cell_hash(cell_id, 269.5, 183.3);
      const double h3 = cell_hash(cell_id, 419.2, 371.9);
      if (h3 < 0.30) continue;
      const double hx = h1 * 0.14 + cc.hue_offset;
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
  const double pt_norm = page_thorne(r, cc.r_isco);
  double I = (cc.pt_peak > 0.0) ? pt_norm / cc.pt_peak : 0.0;
  const double red_c = dclamp(red, 0.1, 10.0);
  const double lift = 1.0 + 0.85 * dclamp(1.0 - red_c, 0.0, 1.0);
  I *= ktm_pow(red_c, 4.0) * lift;
  I *= dclamp(1.0 / magnif, 0.05, 5.0);
  const double norm = w_total * 255.0;
  out[0] = to_u8(tonemap(acc_r / norm * I, cc.exposure, cc.gamma) * 255);
  out[1] = to_u8(tonemap(acc_g / norm * I, cc.exposure, cc.gamma) * 255);
  out[2] = to_u8(tonemap(acc_b / norm * I, cc.exposure, cc.gamma) * 255);
}

KT_HD int iclamp(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

// BackgroundImage::sample (main.cpp:153-170) on an RGB8 image.
KT_HD void bg_sample(const uint8_t* px, int w, int h, double theta, double phi, uint8_t out[3]) {
  double pw = fmod(phi, 2.0 * kPi);
  if (pw < 0) pw += 2.0 * kPi;
  const double uf = (pw / (2.0 * kPi)) * (double)(w - 1);
  const double vf = (theta / kPi) * (double)(h - 1);
  const int u0 = (int)uf, u1 = (w > 1) ? ((u0 + 1) % w) : 0;
  const int v0 = (int)vf, v1 = (v0 + 1 < h - 1) ? v0 + 1 : h - 1;
  const double fu = uf - u0, fv = vf - v0;
  const int r0 = iclamp(v0, 0, h - 1) * w, r1 = iclamp(v1, 0, h - 1) * w;
  const int c0 = iclamp(u0, 0, w - 1), c1 = iclamp(u1, 0, w - 1);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double c00 = px[3 * (r0 + c0) + k];
    const double c10 = px[3 * (r0 + c1) + k];
    const double c01 = px[3 * (r1 + c0) + k];
    const double c11 = px[3 * (r1 + c1) + k];
    const double top = c00 + fu * (c10 - c00);
    const double bot = c01 + fu * (c11 - c01);
    out[k] = to_u8(top + fv * (bot - top));
  }
}

}  // namespace kt
