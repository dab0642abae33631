// kt_smooth.cuh -- physics of the differentiable ("smooth") tracer.
//
// The smooth tracer runs the reference's algorithm -- camera ray
// (camera.hpp:50-145), the KS chart with its BL fallback (main.cpp:1404-1430,
// 1533-1665) or the BL chart (main.cpp:343-434), RK4 step doubling with the
// reference's controller (geodesic.hpp:204-257, main.cpp:1488-1528), Hermite
// disk crossing, horizon and escape events -- with three changes that make
// its outputs smooth functions of the frame parameters:
//   * the Hamiltonian gradient is analytic (the reference differences H with
//     steps of 1e-5, whose rounding noise moves g by ~1e-6 per ulp of input);
//   * the disk crossing is the root of the Hermite interpolant solved to
//     convergence (the reference stops after 8 bisections, a staircase in
//     the parameters with steps of 2^-11 of a step);
//   * the BL <-> KS Jacobian is analytic (the reference differences it).
// Everything here is templated on the scalar type T: double for the tracer,
// Dual<N> for derivatives.
//
// Parameters of differentiation: the metric's (a, Q, Lambda) enter the
// Hamiltonian; (theta_obs, r_obs) enter through the camera ray.  M and the
// disk's radii are constants (the hit radius and redshift do not depend on
// the disk edges; the edges only decide which rays hit).
#pragma once

#include "kt_dual.cuh"
#include "kt_machines.cuh"

// Functions called from many places in the smooth kernels are real calls on
// the device (KT_HD_CALL, kt_physics.cuh): the kernels are otherwise too big
// for the instruction cache.

namespace kt {

constexpr int kSmPrm = 3;  // (a, Q, Lambda)

template <class T>
struct SmPrm {
  T a, Q, L;
};

template <class T>
KT_HD SmPrm<T> sm_prm(const Metric& g) {
  SmPrm<T> p;
  p.a = T(g.a);
  p.Q = T(g.Q);
  p.L = T(g.L);
  return p;
}

// ------------------------------------------------------------- BL metric
// knds_metric.hpp:45-117 in the form
//   A = r^2 + a^2, S = r^2 + a^2 cos^2, R = A (1 - L r^2/3) - 2 M r + Q^2,
//   Tt = 1 + L a^2 cos^2/3, xi = 1 + L a^2/3,
//   g^tt = -xi^2/S (A^2/R - a^2 s2/Tt)   g^tphi = a xi^2/S (1/Tt - A/R)
//   g^rr = R/S   g^thth = Tt/S   g^phiphi = xi^2/S (1/(Tt s2) - a^2/R)
//   g_tt = (-R + Tt a^2 s2)/(S xi^2)     g_tphi = a s2 (R - Tt A)/(S xi^2)
//   g_rr = S/R   g_thth = S/Tt   g_phiphi = s2 (Tt A^2 - R a^2 s2)/(S xi^2)
template <class T>
struct SmBL {
  T tt, tp, rr, hh, pp;
};

template <class T>
KT_HD void sm_bl_metric(double M, const SmPrm<T>& P, const T& r, const T& s, const T& c,
                        SmBL<T>* cov, SmBL<T>* inv) {
  const T a2 = P.a * P.a;
  const T r2 = r * r;
  const T s2 = s * s, c2 = c * c;
  const T A = r2 + a2;
  const T S = r2 + a2 * c2;
  const T R = A * (1.0 - P.L * r2 / 3.0) - 2.0 * M * r + P.Q * P.Q;
  const T Tt = 1.0 + P.L * a2 * c2 / 3.0;
  const T xi = 1.0 + P.L * a2 / 3.0;
  const T xi2 = xi * xi;
  if (cov) {
    const T pre = S * xi2;
    cov->tt = (Tt * a2 * s2 - R) / pre;
    cov->tp = P.a * s2 * (R - Tt * A) / pre;
    cov->rr = S / R;
    cov->hh = S / Tt;
    cov->pp = s2 * (Tt * A * A - R * a2 * s2) / pre;
  }
  if (inv) {
    const T iS = 1.0 / S, iR = 1.0 / R, iT = 1.0 / Tt;
    inv->tt = -xi2 * iS * (A * A * iR - a2 * s2 * iT);
    inv->tp = P.a * xi2 * iS * (iT - A * iR);
    inv->rr = R * iS;
    inv->hh = Tt * iS;
    inv->pp = (s2 > 1e-14) ? xi2 * iS * (iT / s2 - a2 * iR) : T(0.0);
  }
}

// ------------------------------------------------------------- KS chart
// state y = (X, Y, Z, p_X, p_Y, p_Z), constant p_T.  g^ab = eta^ab - F l^a l^b
// (ingoing, Lambda = 0, knds_metric.hpp:150-230) with l = (-1, (rX+aY)/D,
// (rY-aX)/D, Z/r), D = r^2 + a^2, F = (2Mr - Q^2)/rho2, rho2 = r^2 + a^2 Z^2/r^2,
// r(X, Y, Z; a) the root of r^4 - (R^2 - a^2) r^2 - a^2 Z^2 = 0.  Then
//   H = (-p_T^2 + |p|^2 - F ell^2)/2,  ell = -p_T + u/D + Z p_Z/r,
//   u = (rX + aY) p_X + (rY - aX) p_Y,
// and the implicit-function derivatives of r are
//   r_X = X r/E, r_Y = Y r/E, r_Z = Z D/(r E), r_a = a (Z^2 - r^2)/(r E),
//   E = 2 r^2 - (R^2 - a^2).
struct ChartKS {
  static constexpr int kX = 3;  // coordinates (and momenta)
  static constexpr int kN = 6;  // state size
  static constexpr int kC = 1;  // constants of motion: p_T
  static constexpr int kEq = 2;  // state index of the equator coordinate (Z)
  static constexpr double kEqTarget = 0.0;
  static constexpr int kG = 6;            // geodesic components (error norm, events)
  static constexpr bool kBundle = false;  // no Jacobi matrix in the state

  // gy = dH/dy (X, Y, Z, pX, pY, pZ), gc = dH/dp_T, gp = dH/d(a, Q, Lambda)
  // (only with kPrm: the right-hand side needs gy and gc alone).
  template <class T, bool kPrm = true>
  KT_HD static void grad(double M, const SmPrm<T>& P, const T* y, const T* c, T* gy, T* gc, T* gp) {
    const T &X = y[0], &Y = y[1], &Z = y[2], &pX = y[3], &pY = y[4], &pZ = y[5], &pT = c[0];
    const T a = P.a, a2 = P.a * P.a;
    const T R2 = X * X + Y * Y + Z * Z;
    const T b = R2 - a2;
    const T r = sm_sqrt(0.5 * (b + sm_sqrt(b * b + 4.0 * a2 * Z * Z)));
    const T r2 = r * r;
    const T ir = 1.0 / r;
    const T D = r2 + a2;
    const T iD = 1.0 / D;
    const T iE = 1.0 / (2.0 * r2 - b);
    const T Z2 = Z * Z;
    const T rho2 = r2 + a2 * Z2 * ir * ir;
    const T irho2 = 1.0 / rho2;
    const T N = 2.0 * M * r - P.Q * P.Q;
    const T F = N * irho2;
    const T qX = r * X + a * Y, qY = r * Y - a * X;
    const T u = qX * pX + qY * pY;
    const T ell = -pT + u * iD + Z * pZ * ir;
    const T w = X * pX + Y * pY;
    const T Fl = F * ell;
    gy[3] = pX - Fl * qX * iD;
    gy[4] = pY - Fl * qY * iD;
    gy[5] = pZ - Fl * Z * ir;
    gc[0] = -pT + Fl;
    // d/dX, d/dY, d/dZ, d/da
    const T rv[4] = {X * r * iE, Y * r * iE, Z * D * ir * iE, a * (Z2 - r2) * ir * iE};
    const T ir3 = ir * ir * ir;
#pragma unroll
    for (int v = 0; v < (kPrm ? 4 : 3); ++v) {
      const T rr = rv[v];
      T drho2 = 2.0 * r * rr - 2.0 * a2 * Z2 * ir3 * rr;
      if (v == 2) drho2 = drho2 + 2.0 * a2 * Z * ir * ir;
      if (v == 3) drho2 = drho2 + 2.0 * a * Z2 * ir * ir;
      const T dF = (2.0 * M * rr - F * drho2) * irho2;
      T dD = 2.0 * r * rr;
      if (v == 3) dD = dD + 2.0 * a;
      T du = rr * w;
      if (v == 0) du = du + r * pX - a * pY;
      if (v == 1) du = du + a * pX + r * pY;
      if (v == 3) du = du + Y * pX - X * pY;
      T dzr = -Z * rr * ir * ir;  // d(Z/r)
      if (v == 2) dzr = dzr + ir;
      const T dell = (du - u * iD * dD) * iD + pZ * dzr;
      const T dH = -(0.5 * dF * ell * ell + Fl * dell);
      if (v < 3)
        gy[v] = dH;
      else
        gp[0] = dH;
    }
    if (kPrm) {
      gp[1] = P.Q * ell * ell * irho2;  // dF/dQ = -2Q/rho2
      gp[2] = T(0.0);                   // the KS chart carries no Lambda
    }
  }

  template <class T>
  KT_HD static T ham(double M, const SmPrm<T>& P, const T* y, const T* c) {
    const T &X = y[0], &Y = y[1], &Z = y[2], &pX = y[3], &pY = y[4], &pZ = y[5], &pT = c[0];
    const T a = P.a;
    const T r = radius(a, y);
    const T D = r * r + a * a;
    const T F = (2.0 * M * r - P.Q * P.Q) / (r * r + a * a * Z * Z / (r * r));
    const T ell = -pT + ((r * X + a * Y) * pX + (r * Y - a * X) * pY) / D + Z * pZ / r;
    return 0.5 * (-pT * pT + pX * pX + pY * pY + pZ * pZ - F * ell * ell);
  }

  template <class T, class A>
  KT_HD static T radius(const A& a, const T* y) {
    const T b = y[0] * y[0] + y[1] * y[1] + y[2] * y[2] - a * a;
    return sm_sqrt(0.5 * (b + sm_sqrt(b * b + 4.0 * a * a * y[2] * y[2])));
  }
};

// ------------------------------------------------------------- BL chart
// state y = (r, theta, p_r, p_theta), constants (p_t, p_phi), passenger phi
// (dphi/dlam = dH/dp_phi).  With the metric of sm_bl_metric, the Hamiltonian
// (knds_metric.hpp:122-132) is, collected over the metric's denominators,
//   H = K / (2 S),  K = R p_r^2 + Tt p_theta^2 + xi^2 (W iT - P^2 iR),
//   P = A p_t + a p_phi,  W = a^2 s2 p_t^2 + 2 a p_t p_phi + p_phi^2 / s2
// (1/s2 -> 0 within 1e-14 of the axis, the reference's guard on g^phiphi),
// iR = 1/R, iT = 1/Tt.  Its derivatives in (r, theta, a, Q, Lambda) follow
// from those of A, S, R, Tt, s2, xi^2 and a.
struct ChartBL {
  static constexpr int kX = 2;
  static constexpr int kN = 4;
  static constexpr int kC = 2;
  static constexpr int kEq = 1;  // theta
  static constexpr double kEqTarget = 1.57079632679489661923;  // M_PI/2 as the reference
  static constexpr int kG = 4;
  static constexpr bool kBundle = false;

  // x/3 is taken as x * (1/3) (on a Dual, one product per component instead
  // of a division).  kFast (the mixed-precision bundle): reciprocals and
  // sincos from mx_rcp / mx_sincos; otherwise the smooth tracer's
  // arithmetic, identical on host and device.
  template <class T, bool kPrm = true, bool kFast = false>
  KT_HD static void grad(double M, const SmPrm<T>& P, const T* y, const T* c, T* gy, T* gc, T* gp) {
    const T &r = y[0], &th = y[1], &pr = y[2], &pth = y[3], &pt = c[0], &pph = c[1];
    const T a = P.a, L = P.L;
    const T a2 = a * a;
    auto third = [](const T& x) -> T { return x * (1.0 / 3.0); };
    auto rcp = [](const T& x) -> T {
      if constexpr (kFast) return sm_rcp_fast(x);
      else return 1.0 / x;
    };
    T sn, co;
    if constexpr (kFast) sm_sincos_fast(th, &sn, &co);
    else sm_sincos(th, &sn, &co);
    const T s2 = sn * sn, c2 = co * co, sc = sn * co;
    const T r2 = r * r;
    const T A = r2 + a2;
    const T S = r2 + a2 * c2;
    const T Lr2_3 = third(L * r2);
    const T R = A * (1.0 - Lr2_3) - 2.0 * M * r + P.Q * P.Q;
    const T Tt = 1.0 + third(L * a2 * c2);
    const T xi = 1.0 + third(L * a2);
    const T xi2 = xi * xi;
    const T iS = rcp(S), iR = rcp(R), iT = rcp(Tt);
    const bool pole = !(s2 > 1e-14);
    const T is2 = pole ? T(0.0) : rcp(s2);
    const T Pp = A * pt + a * pph;
    const T W = a2 * s2 * pt * pt + 2.0 * a * pt * pph + pph * pph * is2;
    const T K = R * pr * pr + Tt * pth * pth + xi2 * (W * iT - Pp * Pp * iR);
    const T H = 0.5 * K * iS;
    gy[2] = R * pr * iS;
    gy[3] = Tt * pth * iS;
    gc[0] = xi2 * ((a2 * s2 * pt + a * pph) * iT - Pp * A * iR) * iS;
    gc[1] = xi2 * ((a * pt + pph * is2) * iT - Pp * a * iR) * iS;
    const T prpr = pr * pr, hh = pth * pth, ptpt = pt * pt;
    const T WiT_P2iR = W * iT - Pp * Pp * iR;
    // dH/dv = (dK/dv - 2 H dS/dv) / (2 S) for v = r, theta, a, Q, Lambda
    const T zero(0.0);
#pragma unroll
    for (int v = 0; v < (kPrm ? 5 : 2); ++v) {
      const T dA = v == 0 ? 2.0 * r : v == 2 ? 2.0 * a : zero;
      const T dS = v == 0 ? 2.0 * r : v == 1 ? -2.0 * a2 * sc : v == 2 ? 2.0 * a * c2 : zero;
      const T dR = v == 0 ? 2.0 * r * (1.0 - Lr2_3) - third(2.0 * L * r) * A - 2.0 * M
                   : v == 2 ? 2.0 * a * (1.0 - Lr2_3)
                   : v == 3 ? 2.0 * P.Q
                   : v == 4 ? third(-A * r2)
                            : zero;
      const T dT = v == 1 ? -third(2.0 * L * a2) * sc
                   : v == 2 ? third(2.0 * L * a * c2)
                   : v == 4 ? third(a2 * c2)
                            : zero;
      const T ds2 = v == 1 ? 2.0 * sc : zero;
      const T dxi2 = v == 2 ? 2.0 * xi * third(2.0 * L * a) : v == 4 ? 2.0 * xi * third(a2) : zero;
      const double da = v == 2 ? 1.0 : 0.0;
      const T dP = dA * pt + da * pph;
      const T dW = (v == 2 ? 2.0 * a * s2 * ptpt + 2.0 * pt * pph : zero) + a2 * ds2 * ptpt -
                   (pole ? zero : pph * pph * ds2 * is2 * is2);
      const T dK = dR * prpr + dT * hh + dxi2 * WiT_P2iR +
                   xi2 * (dW * iT - W * dT * iT * iT - 2.0 * Pp * dP * iR + Pp * Pp * dR * iR * iR);
      const T dH = (0.5 * dK - H * dS) * iS;
      if (v < 2)
        gy[v] = dH;
      else
        gp[v - 2] = dH;
    }
  }

  template <class T>
  KT_HD static T ham(double M, const SmPrm<T>& P, const T* y, const T* c) {
    T sn, co;
    sm_sincos(y[1], &sn, &co);
    const T a = P.a, a2 = a * a, r2 = y[0] * y[0];
    const T s2 = sn * sn, c2 = co * co;
    const T A = r2 + a2, S = r2 + a2 * c2;
    const T R = A * (1.0 - P.L * r2 / 3.0) - 2.0 * M * y[0] + P.Q * P.Q;
    const T Tt = 1.0 + P.L * a2 * c2 / 3.0;
    const T xi = 1.0 + P.L * a2 / 3.0;
    const T is2 = (s2 > 1e-14) ? 1.0 / s2 : T(0.0);
    const T Pp = A * c[0] + a * c[1];
    const T W = a2 * s2 * c[0] * c[0] + 2.0 * a * c[0] * c[1] + c[1] * c[1] * is2;
    const T K = R * y[2] * y[2] + Tt * y[3] * y[3] + xi * xi * (W / Tt - Pp * Pp / R);
    return 0.5 * K / S;
  }

  template <class T, class A>
  KT_HD static T radius(const A&, const T* y) { return y[0]; }
};

// ------------------------------------------------------- BL ray bundle
// The Jacobi bundle of ray_bundle.hpp:117-263 for the smooth tracer: state
// y = (r, theta, p_r, p_theta, W) with the 4x2 Jacobi matrix W row-major
// (y[4 + 2 i + k] = W[i][k]), constants (p_t, p_phi), passenger phi.  The
// geodesic is the BL chart's; dW = J_s Hess(H) W with the analytic Hessian
// (the reference differences H with steps of 1e-5, whose rounding noise
// moves the magnification by ~1e-5).  The error norm and the events look at
// the geodesic (kG = 4 components) only, as bundle_adaptive does.
struct ChartBLB {
  static constexpr int kX = 2;
  static constexpr int kN = 12;
  static constexpr int kC = 2;
  static constexpr int kEq = 1;
  static constexpr double kEqTarget = ChartBL::kEqTarget;
  static constexpr int kG = 4;
  static constexpr bool kBundle = true;

  template <class T, class A>
  KT_HD static T radius(const A&, const T* y) { return y[0]; }
};

// f = (dH/dp, -dH/dx) and the passenger rate (BL: dphi = dH/dp_phi).  For a
// bundle, one evaluation of the BL gradient in Dual<2> along W's columns
// gives the geodesic RHS (the values, bit for bit the BL chart's) and
// Hess(H) W (the tangents), so dW = J_s Hess(H) W (ray_bundle.hpp:117-156).
template <class C, class T>
KT_HD_CALL void sm_rhs(double M, const SmPrm<T>& P, const T* y, const T* c, T* f, T* fpas) {
  if constexpr (C::kBundle) {
    typedef Dual<2> D;
    SmPrm<D> Pd;
    Pd.a = D(P.a);
    Pd.Q = D(P.Q);
    Pd.L = D(P.L);
    D yd[4], cd[2], gy[4], gc[2], gp[kSmPrm];
    for (int i = 0; i < 4; ++i) {
      yd[i] = D(y[i]);
      yd[i].d[0] = y[4 + 2 * i];
      yd[i].d[1] = y[5 + 2 * i];
    }
    cd[0] = D(c[0]);
    cd[1] = D(c[1]);
    ChartBL::grad<D, false>(M, Pd, yd, cd, gy, gc, gp);
    f[0] = gy[2].v;
    f[1] = gy[3].v;
    f[2] = -gy[0].v;
    f[3] = -gy[1].v;
    for (int k = 0; k < 2; ++k) {
      f[4 + k] = gy[2].d[k];
      f[6 + k] = gy[3].d[k];
      f[8 + k] = -gy[0].d[k];
      f[10 + k] = -gy[1].d[k];
    }
    if (fpas) *fpas = gc[1].v;
  } else {
    T gy[C::kN], gc[C::kC], gp[kSmPrm];
    C::template grad<T, false>(M, P, y, c, gy, gc, gp);
    for (int i = 0; i < C::kX; ++i) {
      f[i] = gy[C::kX + i];
      f[C::kX + i] = -gy[i];
    }
    if (fpas) *fpas = (C::kC > 1) ? gc[C::kC - 1] : T(0.0);
  }
}

// Bundle RHS (bundle_rhs, ray_bundle.hpp:130-156) from one evaluation of
// the analytic BL gradient of H in Dual<2>, the tangents being W's two
// columns: the values are the geodesic RHS (dr = dH/dp_r, dtheta = dH/dp_theta,
// dp = -dH/dx, dphi = dH/dp_phi), the tangents the Hessian-vector products
// Hess(H) W, so dW = J_s Hess(H) W needs no finite-difference Hessian (the
// reference evaluates 33 Hamiltonians at 9 metric points for it).  FP64;
// the mixed-precision bundle tracer's RHS.
KT_HD void bundle_rhs_analytic(const Metric& g, const double y[4], double pt, double pphi,
                               const double W[8], double k[5], double dW[8]) {
  typedef Dual<2> D;
  SmPrm<D> P;
  P.a = D(g.a);
  P.Q = D(g.Q);
  P.L = D(g.L);
  D yd[4], cd[2], gy[4], gc[2], gp[3];
  for (int i = 0; i < 4; ++i) {
    yd[i] = D(y[i]);
    yd[i].d[0] = W[2 * i];
    yd[i].d[1] = W[2 * i + 1];
  }
  cd[0] = D(pt);
  cd[1] = D(pphi);
  ChartBL::grad<D, false, true>(g.M, P, yd, cd, gy, gc, gp);
  k[0] = gy[2].v;
  k[1] = gy[3].v;
  k[2] = -gy[0].v;
  k[3] = -gy[1].v;
  k[4] = gc[1].v;
  for (int c = 0; c < 2; ++c) {
    dW[c] = gy[2].d[c];
    dW[2 + c] = gy[3].d[c];
    dW[4 + c] = -gy[0].d[c];
    dW[6 + c] = -gy[1].d[c];
  }
}

// --------------------------------------------------------------- camera
// camera.hpp:50-145: the BL photon of pixel angles (alpha, beta) for an
// observer at (r_obs, theta_obs, phi_obs), in T.  y = (r, theta, pr, ptheta),
// c = (p_t, p_phi).
template <class T>
KT_HD void sm_camera(double M, const SmPrm<T>& P, const T& r_obs, const T& th_obs, double alpha,
                     double beta, T y[4], T c[2]) {
  T s, co;
  sm_sincos(th_obs, &s, &co);
  SmBL<T> G, U;
  sm_bl_metric(M, P, r_obs, s, co, &G, &U);
  const T sgrr = sm_sqrt(sm_abs(G.rr)), sghh = sm_sqrt(sm_abs(G.hh));
  const T denom_phi = G.pp - G.tp * G.tp / G.tt;
  const bool tetrad = (G.tt < -1e-14) && (denom_phi > 1e-14) && (sgrr > 1e-14) && (sghh > 1e-14);
  double sa, ca, sb, cb;
  ktm_sincos(alpha, &sa, &ca);
  ktm_sincos(beta, &sb, &cb);
  const double n_r = (-ca) * cb, n_th = -sb, n_ph = (-sa) * cb;
  T pUt, pUr, pUth, pUph;
  if (tetrad) {
    const T ephi_p = 1.0 / sm_sqrt(denom_phi);
    pUt = 1.0 / sm_sqrt(-G.tt) + n_ph * ((-G.tp / G.tt) * ephi_p);
    pUr = n_r / sgrr;
    pUth = n_th / sghh;
    pUph = n_ph * ephi_p;
  } else {
    pUt = T(1.0);
    pUr = n_r / (sgrr > 1e-14 ? sgrr : T(1e-14));
    pUth = n_th / (sghh > 1e-14 ? sghh : T(1e-14));
    const T gpp = sm_abs(G.pp);
    pUph = n_ph / sm_sqrt(gpp > 1e-14 ? gpp : T(1e-14));
  }
  T pt = G.tt * pUt + G.tp * pUph;
  const T pr = G.rr * pUr, pth = G.hh * pUth, pph = G.tp * pUt + G.pp * pUph;
  const T qa = U.tt, qb = 2.0 * U.tp * pph;
  const T qc = U.rr * pr * pr + U.hh * pth * pth + U.pp * pph * pph;
  const T disc = qb * qb - 4.0 * qa * qc;
  if (disc >= 0.0 && sm_abs(qa) > 1e-15) {
    const T sq = sm_sqrt(disc);
    const T pt1 = (-qb - sq) / (2.0 * qa), pt2 = (-qb + sq) / (2.0 * qa);
    pt = (pt1 < 0.0) ? pt1 : pt2;
    if (pt > 0.0) pt = (val(pt2) < val(pt1)) ? pt2 : pt1;
  }
  y[0] = r_obs;
  y[1] = th_obs;
  y[2] = pr;
  y[3] = pth;
  c[0] = pt;
  c[1] = pph;
}

// init_ks_state (main.cpp:1404-1430) with the analytic Jacobian of
// BL_to_KS_spatial (knds_metric.hpp:368-387):
//   X = s (r cf - a sf), Y = s (r sf + a cf), Z = r c,
// and p_XYZ from J^T p_XYZ = (p_r, p_theta, p_phi) by Cramer's rule.
// Returns false where the reference's init fails (singular J, no real p_T).
template <class T>
KT_HD bool sm_bl_to_ks(double M, const SmPrm<T>& P, const T ybl[4], const T cbl[2], double phi,
                       T y[6], T c[1]) {
  T s, co;
  sm_sincos(ybl[1], &s, &co);
  double sf, cf;
  ktm_sincos(phi, &sf, &cf);
  const T& r = ybl[0];
  const T a = P.a;
  const T xr = r * cf - a * sf, yr = r * sf + a * cf;
  y[0] = s * xr;
  y[1] = s * yr;
  y[2] = r * co;
  // J[i][j] = d(X, Y, Z)_i / d(r, theta, phi)_j
  const T J00 = s * cf, J01 = co * xr, J02 = -s * yr;
  const T J10 = s * sf, J11 = co * yr, J12 = s * xr;
  const T J20 = co, J21 = -r * s, J22(0.0);
  // A = J^T: rows (J00 J10 J20), (J01 J11 J21), (J02 J12 J22)
  const T det = J00 * (J11 * J22 - J21 * J12) - J10 * (J01 * J22 - J21 * J02) +
                J20 * (J01 * J12 - J11 * J02);
  const double scale = fabs(val(J00)) + fabs(val(J11)) + fabs(val(J21)) + fabs(val(J12)) + 1.0;
  if (!(fabs(val(det)) > 1e-14 * scale * scale * scale)) return false;
  const T &b0 = ybl[2], &b1 = ybl[3], &b2 = cbl[1];
  const T idet = 1.0 / det;
  y[3] = (b0 * (J11 * J22 - J21 * J12) - J10 * (b1 * J22 - J21 * b2) + J20 * (b1 * J12 - J11 * b2)) * idet;
  y[4] = (J00 * (b1 * J22 - J21 * b2) - b0 * (J01 * J22 - J21 * J02) + J20 * (J01 * b2 - b1 * J02)) * idet;
  y[5] = (J00 * (J11 * b2 - b1 * J12) - J10 * (J01 * b2 - b1 * J02) + b0 * (J01 * J12 - J11 * J02)) * idet;
  // p_T from g^ab p_a p_b = 0 with g^ab = eta^ab - F l^a l^b
  const T &X = y[0], &Y = y[1], &Z = y[2], &pX = y[3], &pY = y[4], &pZ = y[5];
  const T rk = ChartKS::radius(a, y);
  const T D = rk * rk + a * a;
  const T F = (2.0 * M * rk - P.Q * P.Q) / (rk * rk + a * a * Z * Z / (rk * rk));
  const T l1 = (rk * X + a * Y) / D, l2 = (rk * Y - a * X) / D, l3 = Z / rk;
  const T lp = l1 * pX + l2 * pY + l3 * pZ;
  const T qa = -1.0 - F;
  const T qb = 2.0 * F * lp;
  const T qc = pX * pX + pY * pY + pZ * pZ - F * lp * lp;
  const T disc = qb * qb - 4.0 * qa * qc;
  if (disc < 0.0 || sm_abs(qa) < 1e-15) return false;
  const T sq = sm_sqrt(disc);
  const T pT1 = (-qb - sq) / (2.0 * qa), pT2 = (-qb + sq) / (2.0 * qa);
  c[0] = (pT1 < 0.0) ? pT1 : pT2;
  if (c[0] > 0.0) c[0] = (val(pT2) < val(pT1)) ? pT2 : pT1;
  return finite(val(c[0]));
}

// ------------------------------------------------------- disk redshift
// disk_redshift (main.cpp:329-341) with keplerian_omega
// (knds_metric.hpp:354-363) and the equatorial covariant metric.  Returns
// false where the reference returns a constant (1 or 20): no derivative.
template <class T>
KT_HD bool sm_redshift(double M, const SmPrm<T>& P, const T& r, const T& pt, const T& pph, T* red) {
  const double s = (val(P.a) < 0.0) ? 1.0 : -1.0;
  const T Meff = M - P.Q * P.Q / (2.0 * r) + P.L * P.a * r * r / 3.0;
  const T sq = Meff > 0.0 ? sm_sqrt(Meff) : T(0.0);
  const T den = r * sm_sqrt(r) + s * P.a * sq;
  const T Om = (sm_abs(den) < 1e-14) ? T(0.0) : s * sq / den;
  const T b = (-pph) / (-pt);
  SmBL<T> G;
  const T one(1.0), zero(0.0);
  sm_bl_metric<T>(M, P, r, one, zero, &G, (SmBL<T>*)nullptr);
  const T d2 = -(G.tt + 2.0 * G.tp * Om + G.pp * Om * Om);
  if (d2 <= 0.0) {
    *red = T(1.0);
    return false;
  }
  const T dv = sm_abs(1.0 - Om * b);
  if (dv < 1e-8) {
    *red = T(20.0);
    return false;
  }
  *red = sm_sqrt(d2) / dv;
  if (!finite(val(*red))) {
    *red = T(1.0);
    return false;
  }
  return true;
}

// The bundle's own redshift (ray_bundle.hpp:360-371): sqrt(d2) / (1 - Omega b)
// where d2 > 0 and |1 - Omega b| > 1e-10, else 1, clamped to [0, 20].
// Returns false where that is a constant (no derivative).
template <class T>
KT_HD bool sm_redshift_bundle(double M, const SmPrm<T>& P, const T& r, const T& pt, const T& pph,
                              T* red) {
  const double s = (val(P.a) < 0.0) ? 1.0 : -1.0;
  const T Meff = M - P.Q * P.Q / (2.0 * r) + P.L * P.a * r * r / 3.0;
  const T sq = Meff > 0.0 ? sm_sqrt(Meff) : T(0.0);
  const T den = r * sm_sqrt(r) + s * P.a * sq;
  const T Om = (sm_abs(den) < 1e-14) ? T(0.0) : s * sq / den;
  const T b = (-pph) / (-pt);
  SmBL<T> G;
  const T one(1.0), zero(0.0);
  sm_bl_metric<T>(M, P, r, one, zero, &G, (SmBL<T>*)nullptr);
  const T d2 = -(G.tt + 2.0 * G.tp * Om + G.pp * Om * Om);
  const T dv = 1.0 - Om * b;
  if (!(d2 > 0.0 && fabs(val(dv)) > 1e-10)) {
    *red = T(1.0);
    return false;
  }
  *red = sm_sqrt(d2) / dv;
  if (!finite(val(*red))) {
    *red = T(1.0);
    return false;
  }
  if (*red < 0.0) {
    *red = T(0.0);
    return false;
  }
  if (*red > 20.0) {
    *red = T(20.0);
    return false;
  }
  return true;
}

// ------------------------------------------------------ Hermite crossing
// hermite_interp_scalar (geodesic.hpp:57-69) without the clamp (alpha is a
// root inside [0, 1]) and its alpha-derivative.
template <class T, class U>
KT_HD T sm_hermite(const T& y0, const T& y1, const T& d0, const T& d1, double h, const U& al) {
  const U a2 = al * al;
  const U a3 = a2 * al;
  return (2.0 * a3 - 3.0 * a2 + 1.0) * y0 + (a3 - 2.0 * a2 + al) * (h * d0) +
         (3.0 * a2 - 2.0 * a3) * y1 + (a3 - a2) * (h * d1);
}

// The same with the step size as a T (its derivative carried).
template <class T, class U>
KT_HD T sm_hermite_h(const T& y0, const T& y1, const T& d0, const T& d1, const T& h, const U& al) {
  const U a2 = al * al;
  const U a3 = a2 * al;
  return (2.0 * a3 - 3.0 * a2 + 1.0) * y0 + (a3 - 2.0 * a2 + al) * (h * d0) +
         (3.0 * a2 - 2.0 * a3) * y1 + (a3 - a2) * (h * d1);
}

KT_HD double sm_hermite_da(double y0, double y1, double d0, double d1, double h, double al) {
  const double a2 = al * al;
  return (6.0 * a2 - 6.0 * al) * y0 + (3.0 * a2 - 4.0 * al + 1.0) * (h * d0) +
         (6.0 * al - 6.0 * a2) * y1 + (3.0 * a2 - 2.0 * al) * (h * d1);
}

// First crossing of `target` in [0, 1] (first_event_alpha_hermite,
// geodesic.hpp:104-140: 8 bins scanned in order) refined to convergence:
// bisection while the bracket is wide, then safeguarded Newton steps.
KT_HD bool sm_first_crossing(double y0, double y1, double d0, double d1, double h, double target,
                             double* alpha) {
  const double f_eps = 1e-12;
  double a0 = 0.0, f0 = y0 - target;
  if (fabs(f0) <= f_eps) {
    *alpha = 0.0;
    return true;
  }
  for (int i = 1; i <= 8; ++i) {
    const double a1 = (double)i / 8.0;
    const double f1 = (i == 8) ? (y1 - target) : sm_hermite(y0, y1, d0, d1, h, a1) - target;
    if (fabs(f1) <= f_eps) {
      *alpha = a1;
      return true;
    }
    if (sign_change(f0, f1)) {
      double lo = a0, hi = a1, flo = f0;
      for (int k = 0; k < 20; ++k) {
        const double mid = 0.5 * (lo + hi);
        const double fm = sm_hermite(y0, y1, d0, d1, h, mid) - target;
        if (sign_change(flo, fm)) {
          hi = mid;
        } else {
          lo = mid;
          flo = fm;
        }
      }
      double al = 0.5 * (lo + hi);
      for (int k = 0; k < 6; ++k) {
        const double fa = sm_hermite(y0, y1, d0, d1, h, al) - target;
        const double da = sm_hermite_da(y0, y1, d0, d1, h, al);
        if (!(fabs(da) > 0.0)) break;
        const double nx = al - fa / da;
        if (!(nx >= lo && nx <= hi)) break;
        if (nx == al) break;
        al = nx;
      }
      *alpha = al;
      return true;
    }
    a0 = a1;
    f0 = f1;
  }
  return false;
}

}  // namespace kt
