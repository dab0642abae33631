// kt_smray.cuh -- one ray of the smooth tracer and its discrete adjoint.
//
// Forward: RK4 step doubling (geodesic.hpp:204-257, main.cpp:1456-1528) with
// the reference's controller (doubling_update), events after every accepted
// step as main.cpp:1570-1657 (KS) / main.cpp:364-433 (BL), outputs in the
// reference's TraceResult slots.  With recording on, the state and step size
// at the start of every k-th accepted step are kept (k = 32; when the 64
// slots fill, every other one is dropped and k doubles).
//
// Adjoint of a disk hit (outputs g, r_hit with cotangents gbar, rbar):
//   * the event: the crossing parameter alpha* solves
//     q(alpha) = Hermite(y_{N-1}, y_N, f_{N-1}, f_N; h, alpha)[eq] - target = 0,
//     so d alpha* = -dq / q'(alpha*) (implicit function theorem).  The hit
//     outputs are differentiated in Dual over the hit state, the constants
//     and (a, Q, Lambda); alpha*'s share goes back through q, and f_{N-1},
//     f_N pass theirs on through VJPs of the RHS;
//   * the accepted steps, last to first.  Step n starts from (y_n, H_n),
//     H_n the controller's dlam; its attempts j = 0..R have sizes h_0 = H_n,
//     h_{j+1} = rho(h_j, e_j) after a rejection, and the accepted one gives
//     y_{n+1} = B(y_n, h_R), H_{n+1} = sigma(h_R, e_R), with
//     e = |A - B|/15, A one RK4 step h, B two RK4 steps h/2.  The
//     accept/reject pattern is replayed as recorded; everything continuous
//     in it is differentiated: the RK4 stages (in y, h and the parameters),
//     the error estimates and the controller formulas of doubling_update
//     (zero where a clamp is active).  Without the controller terms the
//     gradient misses the motion of the step sizes with the parameters,
//     which at tol 1e-7 is up to ~1% of a pixel's derivative;
//   * states come back from the checkpoints: a segment of k steps is replayed
//     from its checkpoint (same controller, same rejections, so the same
//     accepted steps); segments longer than 32 steps are replayed once into
//     inner checkpoints every 32 steps.  The last sm_ring_steps (256; 128
//     for bundles) step starts are kept by the forward itself, so a ray of
//     at most that many steps needs no replay at all.
// VJP of the RHS f = J grad_y H (J = [[0, I], [-I, 0]]): v^T df/dy =
// H_yy (J^T v) and v^T df/dc = d/dc (grad_y H) . (J^T v) = the derivative of
// dH/dc along J^T v, so one Dual<1> evaluation of the full gradient of H along
// d = J^T v = (-v_p, v_x) gives the state, constant and parameter cotangents.
#pragma once

#include "kt_smooth.cuh"

namespace kt {

constexpr int kSmCkSteps = 32;  // accepted steps between checkpoints
// Step starts the forward keeps (the last kSmRing of them): a ray of at most
// that many accepted steps needs no replay in its reverse sweep.  A multiple
// of kSmCkSteps; smaller for the bundle's 12-double state.
#ifndef KT_SM_RING
#define KT_SM_RING 256
#endif
#ifndef KT_SM_RING_BUNDLE
#define KT_SM_RING_BUNDLE 128
#endif
template <int N>
constexpr int sm_ring_steps() { return N >= 12 ? KT_SM_RING_BUNDLE : KT_SM_RING; }
constexpr int kSmCkCap = 64;    // checkpoints per level
constexpr int kSmMaxDoublings = 6;  // k up to 32 * 2^6: 131072 accepted steps

// The per-ray records below are sized by the chart's state size N (4 for
// BL, 6 for KS, 12 for a BL ray bundle).
template <int N>
struct SmCk {  // state at the start of an accepted step and dlam before its attempts
  double y[N];
  double h;
};

template <int N>
struct SmSt {  // state at the start of an accepted step, dlam before its attempts, attempts
  double y[N];
  double H;
  int na;
};

// Data of the final (event) step kept for the adjoint.
template <int N>
struct SmEvent {
  double yp[N];  // y_{N-1}
  double y[N];   // y_N
  double H;      // dlam before the attempts of step N-1
  double h;      // accepted step size of step N-1
  double alpha;
  int deriv;     // 1: redshift has a derivative (not a constant or clamped)
  int mderiv;    // 1: the bundle's magnification has a derivative (not clamped)
};

// Stages of one adaptive attempt from y with step h, t = 0..9: path A =
// RK4 stages 2-4 of one step h (t = 0-2), path B1 = stages 2-4 of a step h/2
// (t = 3-5), path B2 = stages 1-4 of a step h/2 from B1's result (t = 6-9);
// stage 1 of A and B1 is k1 = f(y), given.  Stage inputs base + h/2 k1,
// base + h/2 k2, base + h k3; result base + h/6 (k1 + 2 k2 + 2 k3 + k4)
// (rk4_step_ks, main.cpp:1456-1486).  One rolled loop, one RHS call site: the
// kernel's code stays small enough for the instruction cache.
template <int N>
struct SmStages {
  double u[10][N];  // stage inputs
  double k[10][N];  // f(u)
};

KT_HD void sm_stage_of(int t, int* sub, int* s) {
  *sub = t < 3 ? 0 : (t < 6 ? 1 : 2);
  *s = *sub == 0 ? t + 1 : (*sub == 1 ? t - 2 : t - 6);
}

// Paths A and B of an attempt (results yA, yB and B's passenger) and their
// difference dAB = yA - yB formed from the paths' increments,
// (h/6 sum_A) - ((h/12 sum_B1) + (h/12 sum_B2)): the same quantity as the
// difference of the two end states, without the rounding of the states
// themselves, which near-cancel in it -- the error estimate it feeds moves
// the step sizes, so that rounding would move the trace by ~1e-12 whatever
// the parameters.  With `rec`, the stage inputs and slopes are kept.
template <class C>
KT_HD_CALL void sm_paths(double M, const SmPrm<double>& P, const double* c, const double* y, double pas,
                         const double* k1, double k1p, double hh, double* yA, double* yB, double* pB,
                         double* dAB, SmStages<C::kN>* rec) {
  constexpr int n = C::kN;
  double base[n], kp[n], sum[n], yB1[n], u[n], k[n], incA[n], incB1[n];
  double pbase = pas, sump = k1p, pB1 = pas, kk;
  KT_ROLLED
  for (int t = 0; t < 10; ++t) {
    int sub, s;
    sm_stage_of(t, &sub, &s);
    const double hs = sub == 0 ? hh : 0.5 * hh;
    if (s == 1 && sub < 2) {
      for (int i = 0; i < n; ++i) {
        base[i] = y[i];
        kp[i] = k1[i];
        sum[i] = k1[i];
      }
      pbase = pas;
      sump = k1p;
    }
    if (s == 0) {
      for (int i = 0; i < n; ++i) {
        base[i] = yB1[i];
        u[i] = yB1[i];
      }
      pbase = pB1;
    } else {
      const double cs = (s == 3) ? hs : 0.5 * hs;
      for (int i = 0; i < n; ++i) u[i] = base[i] + cs * kp[i];
    }
    sm_rhs<C>(M, P, u, c, k, &kk);
    if (rec)
      for (int i = 0; i < n; ++i) {
        rec->u[t][i] = u[i];
        rec->k[t][i] = k[i];
      }
    if (s == 0) {
      for (int i = 0; i < n; ++i) {
        kp[i] = k[i];
        sum[i] = k[i];
      }
      sump = kk;
      continue;
    }
    const double w = (s == 3) ? 1.0 : 2.0;
    for (int i = 0; i < n; ++i) {
      sum[i] = sum[i] + w * k[i];
      kp[i] = k[i];
    }
    sump = sump + w * kk;
    if (s == 3) {
      for (int i = 0; i < n; ++i) {
        const double inc = hs / 6.0 * sum[i];
        const double r = base[i] + inc;
        yA[i] = sub == 0 ? r : yA[i];
        yB1[i] = sub == 1 ? r : yB1[i];
        yB[i] = sub == 2 ? r : yB[i];
        incA[i] = sub == 0 ? inc : incA[i];
        incB1[i] = sub == 1 ? inc : incB1[i];
        dAB[i] = sub == 2 ? incA[i] - (incB1[i] + inc) : dAB[i];
      }
      const double pr = pbase + hs / 6.0 * sump;
      pB1 = sub == 1 ? pr : pB1;
      *pB = sub == 2 ? pr : *pB;
    }
  }
}

// One adaptive attempt from (y, pas) with k1 = f(y) and step *h:
// err = |A - B| / 15, doubling_update; on acceptance (yo, paso) = B.
template <class C>
KT_HD int sm_attempt(double M, const SmPrm<double>& P, double tol, const double* c, const double* y,
                     double pas, const double* k1, double k1p, double* h, double* yo, double* paso) {
  double yA[C::kN], yB[C::kN], dAB[C::kN], pB = 0.0;
  sm_paths<C>(M, P, c, y, pas, k1, k1p, *h, yA, yB, &pB, dAB, nullptr);
  double e2 = 0.0;
  for (int i = 0; i < C::kG; ++i) {
    const double d = dAB[i];
    e2 = e2 + d * d;
  }
  const int res = doubling_update(sqrt(e2) / 15.0, tol, h);
  if (res == 1) {
    for (int i = 0; i < C::kN; ++i) yo[i] = yB[i];
    *paso = pB;
  }
  return res;
}

// ---- DOPRI5 (BL chart) ------------------------------------------------------
// dopri5_adaptive (geodesic.hpp:312-414) for the smooth tracer: stages
// k2..k6 from the Dormand-Prince tableau, the fifth-order result y5, k7 =
// f(y5), the error norm sqrt(sum_i (dy_i / (tol (1 + |y_i|)))^2 / 4) with
// dy = y5 - y4 formed from the stages as h sum_j (b5_j - b4_j) k_j (the same
// quantity without the rounding of the two states), and the reference's
// controller.  Phi is not advanced (the reference's `advance` updates r,
// theta, p_r, p_theta only).  The stage records are u[s] (s = 1..6, u[6] =
// y5) and k[s] (s = 0..6).

// The tableau: a_{s j} for stage s = 1..5 (the inputs of k2..k6) and s = 6
// (b5, the result y5), row-major 6 x 6, then b5_j - b4_j for j = 0..6 (the
// exact rationals, each rounded once).  In constant memory on the device (the
// stage loops are rolled, and all lanes read the same entry).
#define KT_DP5_TABLEAU                                                                      \
  {1.0 / 5.0, 0.0, 0.0, 0.0, 0.0, 0.0,                                                       \
   3.0 / 40.0, 9.0 / 40.0, 0.0, 0.0, 0.0, 0.0,                                               \
   44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0.0, 0.0, 0.0,                                     \
   19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0.0, 0.0,          \
   9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0.0,   \
   35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0,          \
   71.0 / 57600.0, 0.0, -71.0 / 16695.0, 71.0 / 1920.0, -17253.0 / 339200.0, 22.0 / 525.0,   \
   -1.0 / 40.0}
#if defined(__CUDACC__)
static __constant__ double kDp5TabDev[43] = KT_DP5_TABLEAU;
#endif
static const double kDp5TabHost[43] = KT_DP5_TABLEAU;
#undef KT_DP5_TABLEAU

KT_HD double dp5_tab(int i) {
#if defined(__CUDA_ARCH__)
  return kDp5TabDev[i];
#else
  return kDp5TabHost[i];
#endif
}
KT_HD double dp5_a(int s, int j) { return dp5_tab((s - 1) * 6 + j); }
KT_HD double dp5_e(int j) { return dp5_tab(36 + j); }

template <class C>
KT_HD_CALL void sm_dp_paths(double M, const SmPrm<double>& P, const double* c, const double* y,
                            const double* k1, double hh, double* y5, double* dy, SmStages<C::kN>* rec) {
  constexpr int n = C::kN;
  double kk[7][n], u[n], fp;
  for (int i = 0; i < n; ++i) kk[0][i] = k1[i];
  KT_ROLLED
  for (int s = 1; s <= 6; ++s) {
    for (int i = 0; i < n; ++i) u[i] = y[i];
    for (int j = 0; j < s; ++j) {
      const double hw = hh * dp5_a(s, j);
      for (int i = 0; i < n; ++i) u[i] = u[i] + hw * kk[j][i];
    }
    sm_rhs<C>(M, P, u, c, kk[s], &fp);
    if (rec)
      for (int i = 0; i < n; ++i) rec->u[s][i] = u[i];
    if (s == 6)
      for (int i = 0; i < n; ++i) y5[i] = u[i];
  }
  for (int i = 0; i < n; ++i) {
    double d = 0.0;
    for (int j = 0; j < 7; ++j) d = d + (hh * dp5_e(j)) * kk[j][i];
    dy[i] = d;
  }
  if (rec)
    for (int j = 0; j < 7; ++j)
      for (int i = 0; i < n; ++i) rec->k[j][i] = kk[j][i];
}

KT_HD double sm_dp_err(const double* dy, const double* y, double tol, int n) {
  double e2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double ratio = dy[i] / (tol * (1.0 + fabs(y[i])));
    e2 = e2 + ratio * ratio;
  }
  return sqrt(e2 / (double)n);
}

// The controller of dopri5_adaptive (geodesic.hpp:392-413): 1 accepted,
// 0 rejected, -1 a non-finite error norm (h halved, FSAL dropped).
KT_HD int dp5_update(double err, double* h) {
  if (!finite(err)) {
    *h = (finite(*h) && *h > 1e-10) ? *h * 0.5 : 1e-6;
    if (*h < 1e-10) *h = 1e-10;
    return -1;
  }
  if (err <= 1.0 || *h < 1e-10) {
    const double fac = (err > 1e-12) ? 0.9 * ktm_pow(1.0 / err, 0.2) : 4.0;
    double hnew = *h * fac;
    if (!finite(hnew)) hnew = *h;
    if (hnew > 100.0) hnew = 100.0;
    if (hnew < 1e-10) hnew = 1e-10;
    *h = hnew;
    return 1;
  }
  double hnew = (*h * 0.9) * ktm_pow(1.0 / err, 0.25);
  if (!finite(hnew)) hnew = *h * 0.5;
  *h = dmax(hnew, 1e-10);
  return 0;
}

// One DOPRI5 attempt from (y, pas) with k1 = f(y): on acceptance (yo, paso)
// = (y5, pas).
template <class C>
KT_HD int sm_attempt_dp(double M, const SmPrm<double>& P, double tol, const double* c, const double* y,
                        double pas, const double* k1, double, double* h, double* yo, double* paso) {
  double y5[C::kN], dy[C::kN];
  sm_dp_paths<C>(M, P, c, y, k1, *h, y5, dy, nullptr);
  const int res = dp5_update(sm_dp_err(dy, y, tol, C::kN), h);
  if (res == 1) {
    for (int i = 0; i < C::kN; ++i) yo[i] = y5[i];
    *paso = pas;
  }
  return res;
}

struct SmRk4;
struct SmDp5;

// Outputs of a stop without event: {ESCAPED, r, 1, theta, phi} of the state.
template <class C>
KT_HD void sm_stop(const Frame& f, const double* y, double pas, int status, uint32_t steps,
                   uint32_t attempts, RayResult* o) {
  double rr, tt, pp;
  if (C::kN == 6) {
    ks_to_bl(f.g, y[0], y[1], y[2], &rr, &tt, &pp);
  } else {
    rr = y[0];
    tt = y[1];
    pp = pas;
  }
  o->steps = steps;
  o->attempts = attempts;
  if (C::kBundle)  // BundleResult{} / {false, r, 1, 1} (ray_bundle.hpp:320, 435)
    set_result(o, kOutEscaped, status, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
  else
    set_result(o, kOutEscaped, status, rr, 1.0, 1.0, tt, pp, 0.0);
}

// Trace one ray from (y, c, pas).  With ck != NULL, checkpoints are recorded
// (*ck_k = final interval, *ck_n = count); with ring != NULL, step m's start
// (y, dlam, attempts) is kept in ring[m % R], R = sm_ring_steps (the last R
// steps).  On a disk hit `ev` receives the
// final step; returns the number of accepted steps N (0 if the ray ended
// otherwise or more than 131072 steps were taken with recording on).
template <class C, class I = SmRk4>
KT_HD int sm_trace(const Frame& f, const SmPrm<double>& P, const double* y_in, const double* c,
                   double pas_in, RayResult* o, SmEvent<C::kN>* ev, SmCk<C::kN>* ck, int* ck_k, int* ck_n,
                   SmSt<C::kN>* ring) {
  const double M = f.g.M;
  double y[C::kN], yp[C::kN], k1[C::kN], kprev[C::kN];
  double pas = pas_in, pasp, k1p, kprevp;
  for (int i = 0; i < C::kN; ++i) y[i] = y_in[i];
  double h = f.dlam0;
  uint32_t attempts = 0;
  int k = kSmCkSteps, nck = 0, doublings = 0;
  bool rec_ok = ck != nullptr;
  sm_rhs<C>(M, P, y, c, k1, &k1p);
  double prev_r = C::radius(f.g.a, y);
  KT_ROLLED
  for (int it = 0;; ++it) {
    if (rec_ok && it % k == 0) {
      if (nck == kSmCkCap) {
        if (doublings == kSmMaxDoublings) {
          rec_ok = false;
        } else {
          for (int j = 0; j < kSmCkCap / 2; ++j) ck[j] = ck[2 * j];
          nck = kSmCkCap / 2;
          k *= 2;
          ++doublings;
        }
      }
      if (rec_ok && it % k == 0) {
        for (int i = 0; i < C::kN; ++i) ck[nck].y[i] = y[i];
        ck[nck].h = h;
        ++nck;
      }
    }
    for (int i = 0; i < C::kN; ++i) {
      yp[i] = y[i];
      kprev[i] = k1[i];
    }
    pasp = pas;
    kprevp = k1p;
    const double H_start = h;
    const uint32_t att0 = attempts;
    constexpr int R = sm_ring_steps<C::kN>();
    if (ring) {
      for (int i = 0; i < C::kN; ++i) ring[it % R].y[i] = y[i];
      ring[it % R].H = h;
    }
    double step_used = h;
    int rejects = 0;
    KT_ROLLED
    for (;;) {
      step_used = h;
      ++attempts;
      if (I::template attempt<C>(M, P, f.tol, c, yp, pasp, kprev, kprevp, &h, y, &pas) == 1) break;
      int status;
      if (reject_cap(h, &rejects, &status)) {
        sm_stop<C>(f, yp, pasp, status, (uint32_t)it, attempts, o);
        return 0;
      }
    }
    if (ring) ring[it % R].na = (int)(attempts - att0);
    sm_rhs<C>(M, P, y, c, k1, &k1p);
    // events (main.cpp:1570-1657, 364-433)
    const double r_now = C::radius(f.g.a, y);
    double best_alpha = 2.0;
    int evt = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0, disk_m = 1.0;
    int deriv = 0, mderiv = 0;
    bool skip = false;
    const double q0 = yp[C::kEq] - C::kEqTarget, q1 = y[C::kEq] - C::kEqTarget;
    if (sign_change(q0, q1) || dmin(fabs(q0), fabs(q1)) < 0.35) {
      double alpha = 0.0;
      if (sm_first_crossing(yp[C::kEq], y[C::kEq], kprev[C::kEq], k1[C::kEq], step_used,
                            C::kEqTarget, &alpha)) {
        double yh[C::kG];
        for (int i = 0; i < C::kG; ++i) yh[i] = sm_hermite(yp[i], y[i], kprev[i], k1[i], step_used, alpha);
        const double r_hit = C::radius(f.g.a, yh);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          double red, pph;
          if constexpr (C::kN == 6) {
            pph = yh[0] * yh[4] - yh[1] * yh[3];
          } else {
            pph = c[C::kC - 1];
          }
          if constexpr (C::kBundle) {
            // ray_bundle.hpp:360-392: the bundle's redshift, and |det| of
            // W's (r, theta) rows interpolated linearly to the crossing
            deriv = sm_redshift_bundle<double>(M, P, r_hit, c[0], pph, &red) ? 1 : 0;
            disk_red = red;
            double J[4];
            for (int m = 0; m < 4; ++m) J[m] = yp[4 + m] + alpha * (y[4 + m] - yp[4 + m]);
            const double det = fabs(J[0] * J[3] - J[1] * J[2]);
            mderiv = det < 1e-12 ? 0 : 1;
            disk_m = det < 1e-12 ? 1e-12 : det;
          } else {
            deriv = sm_redshift<double>(M, P, r_hit, c[0], pph, &red) ? 1 : 0;
            if (!(red > 0.0 && red < 20.0)) deriv = 0;
            disk_red = dclamp(red, 0.0, 20.0);
          }
          disk_r = r_hit;
          if (C::kN == 6) {
            double rr, tt;
            ks_to_bl(f.g, yh[0], yh[1], yh[2], &rr, &tt, &disk_phi);
          } else {
            disk_phi = pasp + alpha * (pas - pasp);
          }
          best_alpha = alpha;
          evt = kEvDisk;
        }
      } else if (C::kBundle) {
        skip = true;  // ray_bundle.hpp:352-356 `continue`: no horizon/escape test this step
      }
    }
    if (C::kBundle && skip &&
        ((r_now <= f.r_doom && k1[0] < 0.0) || (r_now >= f.r_cdoom && k1[0] > 0.0))) {
      // a ray creeping onto a horizon in BL coordinates (theta frozen near
      // the equator, the horizon test skipped) ends with the record the
      // controller's eventual failure would give it
      o->steps = (uint32_t)it + 1;
      o->attempts = attempts;
      set_result(o, kOutEscaped, kStCreep, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
      return 0;
    }
    if (!skip) horizon_escape(prev_r, r_now, f.rh_cut, f.r_esc, &best_alpha, &evt);
    if (evt != kEvNone) {
      o->steps = (uint32_t)it + 1;
      o->attempts = attempts;
      if (evt == kEvDisk) {
        set_result(o, kOutDisk, kStEvent, disk_r, disk_red, disk_m, disk_phi, 0.0, 0.0);
        if (ev) {
          for (int i = 0; i < C::kN; ++i) {
            ev->yp[i] = yp[i];
            ev->y[i] = y[i];
          }
          ev->H = H_start;
          ev->h = step_used;
          ev->alpha = best_alpha;
          ev->deriv = deriv;
          ev->mderiv = mderiv;
        }
        if (ck_k) *ck_k = k;
        if (ck_n) *ck_n = nck;
        return (ck == nullptr || rec_ok) ? it + 1 : 0;
      }
      if (C::kBundle) {
        // trace_bundle's records (ray_bundle.hpp:418-433): a horizon hit is
        // BundleResult{} (escaped toward (0, 0)); an escape carries theta, phi
        const double te = evt == kEvHorizon ? 0.0 : yp[1] + best_alpha * (y[1] - yp[1]);
        const double pe = evt == kEvHorizon ? 0.0 : pasp + best_alpha * (pas - pasp);
        set_result(o, kOutEscaped, kStEvent, 0.0, 1.0, 1.0, 0.0, te, pe);
      } else if (evt == kEvHorizon) {
        set_result(o, kOutHorizon, kStEvent, prev_r + best_alpha * (r_now - prev_r), 0.0, 1.0, 0.0,
                   0.0, 0.0);
      } else if (C::kN == 6) {
        double xe[3];
        for (int i = 0; i < 3; ++i) xe[i] = yp[i] + best_alpha * (y[i] - yp[i]);
        double re, te, pe;
        ks_to_bl(f.g, xe[0], xe[1], xe[2], &re, &te, &pe);
        set_result(o, kOutEscaped, kStEvent, re, 1.0, 1.0, te, pe, 0.0);
      } else {
        const double te = yp[1] + best_alpha * (y[1] - yp[1]);
        const double pe = pasp + best_alpha * (pas - pasp);
        set_result(o, kOutEscaped, kStEvent, f.r_esc, 1.0, 1.0, te, pe, 0.0);
      }
      return 0;
    }
    prev_r = r_now;
    if (it + 1 >= f.max_steps) {
      sm_stop<C>(f, y, pas, kStStepCap, (uint32_t)(it + 1), attempts, o);
      return 0;
    }
  }
}

// Replay `n` accepted steps from checkpoint `ck0` (the controller from its
// dlam, rejections included).  Stores each step's start (y_n, H_n) and its
// number of attempts into st[0..n) and/or a checkpoint every k2 steps into ck2.
template <class C, class I = SmRk4>
KT_HD void sm_replay(const Frame& f, const SmPrm<double>& P, const double* c, const SmCk<C::kN>& ck0, int n,
                     SmSt<C::kN>* st, SmCk<C::kN>* ck2, int k2) {
  const double M = f.g.M;
  double y[C::kN], y1[C::kN], k1[C::kN], k1p, pas = 0.0, pas1;
  for (int i = 0; i < C::kN; ++i) y[i] = ck0.y[i];
  double h = ck0.h;
  KT_ROLLED
  for (int m = 0; m < n; ++m) {
    if (ck2 && m % k2 == 0) {
      for (int i = 0; i < C::kN; ++i) ck2[m / k2].y[i] = y[i];
      ck2[m / k2].h = h;
    }
    if (st) {
      for (int i = 0; i < C::kN; ++i) st[m].y[i] = y[i];
      st[m].H = h;
    }
    sm_rhs<C>(M, P, y, c, k1, &k1p);
    int rejects = 0, na = 0;
    KT_ROLLED
    for (;;) {
      ++na;
      if (I::template attempt<C>(M, P, f.tol, c, y, pas, k1, k1p, &h, y1, &pas1) == 1) break;
      int status;
      if (reject_cap(h, &rejects, &status)) break;  // not reached: the forward accepted
    }
    if (st) st[m].na = na;
    for (int i = 0; i < C::kN; ++i) y[i] = y1[i];
    pas = pas1;
  }
}

// Partial derivatives of doubling_update's new dlam in (dlam, err) on the
// branch it takes (zero where a clamp or a constant is chosen).
KT_HD void sm_ctl_partials(double err, double tol, double h, double* dh, double* de) {
  *dh = 0.0;
  *de = 0.0;
  if (!finite(err)) {
    double hn = (finite(h) && h > 1e-10) ? h * 0.5 : 1e-6;
    if (!(hn < 1e-10) && finite(h) && h > 1e-10) *dh = 0.5;
    return;
  }
  const bool accepted = (err < tol || h < 1e-10);
  if (accepted) {
    const double scale = (err > 1e-14) ? 0.9 * ktm_pow(tol / err, 0.2) : 4.0;
    double hn = h * scale;
    if (!finite(hn)) {
      if (h > 100.0 || h < 1e-10) return;
      *dh = 1.0;
      return;
    }
    if (hn > 100.0 || hn < 1e-10) return;
    *dh = scale;
    if (err > 1e-14) *de = -0.2 * hn / err;
  } else {
    const double half = h * 0.5;
    double hn = (h * 0.9) * ktm_pow(tol / err, 0.25);
    bool use_half = !finite(hn) || hn > half;
    if (use_half) hn = half;
    if (hn < 1e-10) return;
    if (use_half) {
      *dh = 0.5;
    } else {
      *dh = hn / h;
      *de = -0.25 * hn / err;
    }
  }
}

// v^T df/d(y, c, prm) at u: ybar = .., cbar += .., pbar += ..
//
// Bundle (u = (z, W), f = (J_s grad H(z), J_s Hess(H)(z) W)): with d = J^T v_z
// and d_k = J^T v_{W,k} (v_{W,k} the cotangent of W's column k),
//   v^T f = d . grad H + sum_k d_k^T Hess(H) W_k,
// so z gets Hess(H) d + sum_k D^3 H[., W_k, d_k], W_k gets Hess(H) d_k, and
// the constants and (a, Q, Lambda) the matching mixed derivatives: one
// Dual<1> evaluation of grad H along d, and per column one hyper-dual
// evaluation at z + e1 W_k + e2 d_k (its e2 part is Hess(H) d_k, its e1 e2
// part D^3 H[., W_k, d_k]).  A zero column cotangent skips its evaluation.
template <class C>
KT_HD_CALL void sm_vjp_f(double M, const SmPrm<double>& P, const double* u, const double* c,
                         const double* v, double* ubar, double* cbar, double* pbar) {
  if constexpr (C::kBundle) {
    sm_vjp_f<ChartBL>(M, P, u, c, v, ubar, cbar, pbar);
    SmPrm<HDual> Ph;
    Ph.a = HDual(P.a);
    Ph.Q = HDual(P.Q);
    Ph.L = HDual(P.L);
    KT_ROLLED
    for (int k = 0; k < 2; ++k) {
      const double w0 = v[4 + k], w1 = v[6 + k], w2 = v[8 + k], w3 = v[10 + k];
      if (w0 == 0.0 && w1 == 0.0 && w2 == 0.0 && w3 == 0.0) {
        for (int i = 0; i < 4; ++i) ubar[4 + 2 * i + k] = 0.0;
        continue;
      }
      const double dk[4] = {-w2, -w3, w0, w1};
      HDual yh[4], ch[2], gy[4], gc[2], gp[kSmPrm];
      for (int i = 0; i < 4; ++i) yh[i] = HDual(u[i], u[4 + 2 * i + k], dk[i], 0.0);
      ch[0] = HDual(c[0]);
      ch[1] = HDual(c[1]);
      ChartBL::grad<HDual, true>(M, Ph, yh, ch, gy, gc, gp);
      for (int i = 0; i < 4; ++i) {
        ubar[i] = ubar[i] + gy[i].c;
        ubar[4 + 2 * i + k] = gy[i].b;
      }
      for (int j = 0; j < 2; ++j) cbar[j] = cbar[j] + gc[j].c;
      for (int q = 0; q < kSmPrm; ++q) pbar[q] = pbar[q] + gp[q].c;
    }
  } else {
    Dual<1> yd[C::kN], cd[C::kC], gy[C::kN], gc[C::kC], gp[kSmPrm];
    for (int i = 0; i < C::kX; ++i) {
      yd[i] = Dual<1>(u[i]);
      yd[i].d[0] = -v[C::kX + i];
      yd[C::kX + i] = Dual<1>(u[C::kX + i]);
      yd[C::kX + i].d[0] = v[i];
    }
    for (int j = 0; j < C::kC; ++j) cd[j] = Dual<1>(c[j]);
    SmPrm<Dual<1>> Pd;
    Pd.a = Dual<1>(P.a);
    Pd.Q = Dual<1>(P.Q);
    Pd.L = Dual<1>(P.L);
    C::grad(M, Pd, yd, cd, gy, gc, gp);
    for (int i = 0; i < C::kN; ++i) ubar[i] = gy[i].d[0];
    for (int j = 0; j < C::kC; ++j) cbar[j] = cbar[j] + gc[j].d[0];
    for (int q = 0; q < kSmPrm; ++q) pbar[q] = pbar[q] + gp[q].d[0];
  }
}

// Reverse of one attempt from y with size hh.  gout: cotangent of the dlam
// the controller sets after it (H_{n+1} after the accepted attempt, the next
// attempt's size after a rejection); yb_out: cotangent of path B's result
// (y_{n+1}; NULL for a rejected attempt); hbar_extra: a further cotangent of
// hh (the event's, on the last step).  ybar/cbar/pbar += ..; returns the
// cotangent of hh.
//
// The forward pass records the 10 stages; the reverse walks them back
// (q = 0-3: B2 stages 4..1, q = 4-6: B1 stages 4..2, q = 7-9: A stages 4..2,
// q = 10: the shared k1 = f(y)) with one VJP call site.  For a stage s of a
// sub-step with size hs and result cotangent Y: kbar_s = hs/6 w_s Y +
// beta_{s+1} hs ubar_{s+1}, ubar_s = VJP_f(u_s, kbar_s), the sub-step's base
// gets Y + sum ubar_s, and its size gets sum w_s/6 Y.k_s + beta_s ubar_s.k_{s-1}.
template <class C>
KT_HD double sm_attempt_bwd(const Frame& f, const SmPrm<double>& P, const double* c, const double* y,
                            double hh, double gout, const double* yb_out, double hbar_extra,
                            double* ybar, double* cbar, double* pbar, SmStages<C::kN>* st) {
  constexpr int n = C::kN;
  const double M = f.g.M;
  double k1[n], k1p, yA[n], yB[n], pB = 0.0;
  sm_rhs<C>(M, P, y, c, k1, &k1p);
  double d[n], e2 = 0.0;
  sm_paths<C>(M, P, c, y, 0.0, k1, k1p, hh, yA, yB, &pB, d, st);
  for (int i = 0; i < C::kG; ++i) e2 = e2 + d[i] * d[i];
  for (int i = C::kG; i < n; ++i) d[i] = 0.0;  // outside the error norm
  const double e = sqrt(e2) / 15.0;
  double dh, de;
  sm_ctl_partials(e, f.tol, hh, &dh, &de);
  const double eb = gout * de;
  const double kap = (e > 0.0 && finite(e)) ? eb / (225.0 * e) : 0.0;
  double hb = gout * dh + hbar_extra;
  const double wst[4] = {1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0};
  double Y[n], bacc[n], kbn[n], k0s[n], uc[n], vc[n], ub[n];
  double hs = 0.5 * hh, hsub = 0.0;
  for (int i = 0; i < n; ++i) {
    Y[i] = (yb_out ? yb_out[i] : 0.0) - kap * d[i];
    bacc[i] = Y[i];
    kbn[i] = hs * wst[3] * Y[i];
    k0s[i] = 0.0;
  }
  KT_ROLLED
  for (int q = 0; q <= 10; ++q) {
    if (q == 4 || q == 7) {
      // finish B2 (-> cotangent of B1's result) or B1; start B1 or A
      hb = hb + 0.5 * hsub;
      hsub = 0.0;
      hs = (q == 4) ? 0.5 * hh : hh;
      for (int i = 0; i < n; ++i) {
        if (q == 7) ybar[i] = ybar[i] + bacc[i];
        Y[i] = (q == 4) ? bacc[i] : kap * d[i];
        bacc[i] = Y[i];
        kbn[i] = hs * wst[3] * Y[i];
      }
    }
    if (q == 10) {
      hb = hb + hsub;
      for (int i = 0; i < n; ++i) ybar[i] = ybar[i] + bacc[i];
    }
    const int t = q < 10 ? 9 - q : 0;
    int sub, s;
    sm_stage_of(t, &sub, &s);
    for (int i = 0; i < n; ++i) {
      uc[i] = (q == 10) ? y[i] : st->u[t][i];
      vc[i] = (q == 10) ? k0s[i] : kbn[i];
    }
    sm_vjp_f<C>(M, P, uc, c, vc, ub, cbar, pbar);
    if (q == 10) {
      for (int i = 0; i < n; ++i) ybar[i] = ybar[i] + ub[i];
      break;
    }
    // direct size term of stage s and the base's cotangent
    double dk = 0.0;
    for (int i = 0; i < n; ++i) {
      dk = dk + Y[i] * st->k[t][i];
      bacc[i] = bacc[i] + ub[i];
    }
    hsub = hsub + wst[s] * dk;
    if (s >= 1) {
      // stage s's input was base + beta_s hs k_{s-1}
      const double beta = (s == 3) ? 1.0 : 0.5;
      double dkm = 0.0;
      for (int i = 0; i < n; ++i) {
        const double km = (s == 1 && sub < 2) ? k1[i] : st->k[t - 1][i];
        dkm = dkm + ub[i] * km;
        const double nk = hs * wst[s - 1] * Y[i] + beta * hs * ub[i];
        if (s == 1 && sub < 2) {
          k0s[i] = k0s[i] + nk;
        } else {
          kbn[i] = nk;
        }
      }
      hsub = hsub + beta * dkm;
      if (s == 1 && sub < 2) {
        // the shared k1's direct size term (w_1 / 6 Y . k1)
        double d1 = 0.0;
        for (int i = 0; i < n; ++i) d1 = d1 + Y[i] * k1[i];
        hsub = hsub + wst[0] * d1;
      }
    }
  }
  return hb;
}

// Partial derivatives of dp5_update's new step in (h, err) on the branch it
// takes (zero where a clamp or a constant is chosen).
KT_HD void sm_dp_ctl_partials(double err, double h, double* dh, double* de) {
  *dh = 0.0;
  *de = 0.0;
  if (!finite(err)) {
    if (finite(h) && h > 1e-10 && !(h * 0.5 < 1e-10)) *dh = 0.5;
    return;
  }
  if (err <= 1.0 || h < 1e-10) {
    const double fac = (err > 1e-12) ? 0.9 * ktm_pow(1.0 / err, 0.2) : 4.0;
    const double hnew = h * fac;
    if (!finite(hnew)) {
      if (h > 100.0 || h < 1e-10) return;
      *dh = 1.0;
      return;
    }
    if (hnew > 100.0 || hnew < 1e-10) return;
    *dh = fac;
    if (err > 1e-12) *de = -0.2 * hnew / err;
    return;
  }
  const double hnew = (h * 0.9) * ktm_pow(1.0 / err, 0.25);
  if (!finite(hnew)) {
    if (!(h * 0.5 < 1e-10)) *dh = 0.5;
    return;
  }
  if (hnew < 1e-10) return;
  *dh = hnew / h;
  *de = -0.25 * hnew / err;
}

// Reverse of one DOPRI5 attempt (the arguments as sm_attempt_bwd's; the
// passenger phi is not integrated).  The error norm feeds the controller:
// its cotangent reaches dy (and the scales' |y_i|), dy = h sum_j e_j k_j
// reaches every slope; y5 = y + h sum_{j<6} b5_j k_j gets yb_out plus k7's
// VJP; then the stage inputs u_s = y + h sum_{j<s} a_sj k_j, s = 5..1, walk
// back (each slope's cotangent complete before its VJP), and k1 = f(y) last.
template <class C>
KT_HD double sm_attempt_bwd_dp(const Frame& f, const SmPrm<double>& P, const double* c, const double* y,
                               double hh, double gout, const double* yb_out, double hbar_extra,
                               double* ybar, double* cbar, double* pbar, SmStages<C::kN>* st) {
  constexpr int n = C::kN;
  const double M = f.g.M;
  double k1[n], k1p, y5[n], dy[n];
  sm_rhs<C>(M, P, y, c, k1, &k1p);
  sm_dp_paths<C>(M, P, c, y, k1, hh, y5, dy, st);
  const double err = sm_dp_err(dy, y, f.tol, n);
  double dh, de;
  sm_dp_ctl_partials(err, hh, &dh, &de);
  const double eb = gout * de;
  double hb = gout * dh + hbar_extra;
  const bool ok = err > 0.0 && finite(err);
  double dyb[n];
  for (int i = 0; i < n; ++i) {
    const double sc = f.tol * (1.0 + fabs(y[i]));
    const double ratio = dy[i] / sc;
    const double rb = ok ? eb * ratio / ((double)n * err) : 0.0;  // d err / d ratio_i = ratio_i / (n err)
    dyb[i] = rb / sc;
    const double sg = y[i] > 0.0 ? 1.0 : (y[i] < 0.0 ? -1.0 : 0.0);
    ybar[i] = ybar[i] - rb * ratio * (f.tol * sg) / sc;  // through the scale tol (1 + |y_i|)
  }
  double kb[7][n];
  for (int j = 0; j < 7; ++j) {
    const double he = hh * dp5_e(j);
    double dk = 0.0;
    for (int i = 0; i < n; ++i) {
      kb[j][i] = he * dyb[i];
      dk = dk + dyb[i] * st->k[j][i];
    }
    hb = hb + dp5_e(j) * dk;
  }
  double w[n];
  sm_vjp_f<C>(M, P, st->u[6], c, kb[6], w, cbar, pbar);  // k7 = f(y5)
  for (int i = 0; i < n; ++i) w[i] = w[i] + (yb_out ? yb_out[i] : 0.0);
  KT_ROLLED
  for (int s = 6; s >= 1; --s) {
    if (s < 6) sm_vjp_f<C>(M, P, st->u[s], c, kb[s], w, cbar, pbar);  // w = cotangent of u_s
    for (int i = 0; i < n; ++i) ybar[i] = ybar[i] + w[i];
    for (int j = 0; j < s; ++j) {
      const double a = dp5_a(s, j);
      double dk = 0.0;
      for (int i = 0; i < n; ++i) {
        kb[j][i] = kb[j][i] + (hh * a) * w[i];
        dk = dk + w[i] * st->k[j][i];
      }
      hb = hb + a * dk;
    }
  }
  sm_vjp_f<C>(M, P, y, c, kb[0], w, cbar, pbar);  // k1 = f(y)
  for (int i = 0; i < n; ++i) ybar[i] = ybar[i] + w[i];
  return hb;
}

// The integrators of the smooth tracer: an attempt and its reverse.
struct SmRk4 {
  template <class C>
  KT_HD static int attempt(double M, const SmPrm<double>& P, double tol, const double* c, const double* y,
                           double pas, const double* k1, double k1p, double* h, double* yo,
                           double* paso) {
    return sm_attempt<C>(M, P, tol, c, y, pas, k1, k1p, h, yo, paso);
  }
  template <class C>
  KT_HD static double attempt_bwd(const Frame& f, const SmPrm<double>& P, const double* c,
                                  const double* y, double hh, double gout, const double* yb_out,
                                  double hbar_extra, double* ybar, double* cbar, double* pbar,
                                  SmStages<C::kN>* st) {
    return sm_attempt_bwd<C>(f, P, c, y, hh, gout, yb_out, hbar_extra, ybar, cbar, pbar, st);
  }
};
struct SmDp5 {
  template <class C>
  KT_HD static int attempt(double M, const SmPrm<double>& P, double tol, const double* c, const double* y,
                           double pas, const double* k1, double k1p, double* h, double* yo,
                           double* paso) {
    return sm_attempt_dp<C>(M, P, tol, c, y, pas, k1, k1p, h, yo, paso);
  }
  template <class C>
  KT_HD static double attempt_bwd(const Frame& f, const SmPrm<double>& P, const double* c,
                                  const double* y, double hh, double gout, const double* yb_out,
                                  double hbar_extra, double* ybar, double* cbar, double* pbar,
                                  SmStages<C::kN>* st) {
    return sm_attempt_bwd_dp<C>(f, P, c, y, hh, gout, yb_out, hbar_extra, ybar, cbar, pbar, st);
  }
};

constexpr int kSmMaxAttempts = 66;  // reject cap 64 + the accepted attempt

// Reverse of accepted step n from (y_n, H_n, attempts).  In: ybar =
// cotangent of y_{n+1}, *Hbar = cotangent of H_{n+1}, hbar_acc = extra
// cotangent of the accepted size (the event's).  Out: ybar = cotangent of
// y_n, *Hbar = of H_n.
template <class C, class I = SmRk4>
KT_HD void sm_step_bwd(const Frame& f, const SmPrm<double>& P, const double* c, const SmSt<C::kN>& st,
                       double hbar_acc, double* ybar, double* Hbar, double* cbar, double* pbar,
                       SmStages<C::kN>* stg) {
  const double M = f.g.M;
  double hs[kSmMaxAttempts];
  const int na = st.na < kSmMaxAttempts ? st.na : kSmMaxAttempts;
  hs[0] = st.H;
  if (na > 1) {
    // sizes of the attempts: the controller after each rejection
    double k1[C::kN], k1p, yo[C::kN], po;
    sm_rhs<C>(M, P, st.y, c, k1, &k1p);
    double h = st.H;
    KT_ROLLED
    for (int j = 0; j + 1 < na; ++j) {
      I::template attempt<C>(M, P, f.tol, c, st.y, 0.0, k1, k1p, &h, yo, &po);
      hs[j + 1] = h;
    }
  }
  double yb_out[C::kN];
  for (int i = 0; i < C::kN; ++i) {
    yb_out[i] = ybar[i];
    ybar[i] = 0.0;
  }
  double gout = *Hbar;
  KT_ROLLED
  for (int j = na - 1; j >= 0; --j) {
    const bool acc = (j == na - 1);
    gout = I::template attempt_bwd<C>(f, P, c, st.y, hs[j], gout, acc ? yb_out : nullptr,
                                      acc ? hbar_acc : 0.0, ybar, cbar, pbar, stg);
  }
  *Hbar = gout;
}

// Cotangents of the event step's inputs from (gbar, rbar, mbar): the hit state
// yh = Hermite(y_{N-1}, y_N, f_{N-1}, f_N; h, alpha*) feeds the outputs
// (r_hit; g through the disk redshift), differentiated in Dual over (yh,
// constants, a, Q, Lambda); alpha* moves with the inputs as
// d alpha* = -dq / q'(alpha*) (q the equator coordinate's interpolant minus
// its target), so the inputs also get lambda dq/dx with lambda = -alphabar/q';
// f_{N-1}, f_N pass their cotangents on through VJPs of the RHS.  A bundle's
// magnification |det J|, J = W_{N-1} + alpha* (W_N - W_{N-1}) over W's (r,
// theta) rows, sends mbar to both W's and to alpha*.
template <class C>
KT_HD void sm_event_bwd(const Frame& f, const SmPrm<double>& P, const double* c, const SmEvent<C::kN>& ev,
                        double gbar, double rbar, double mbar, double* ybp, double* ybN,
                        double* cbar, double* pbar, double* hbar) {
  constexpr int n = C::kN;
  constexpr int ng = C::kG;
  constexpr int ND = ng + C::kC + kSmPrm;
  typedef Dual<ND> D;
  const double M = f.g.M;
  double fe[2][n], pp;
  KT_ROLLED
  for (int w = 0; w < 2; ++w) sm_rhs<C>(M, P, w == 0 ? ev.yp : ev.y, c, fe[w], &pp);
  const double h = ev.h, al = ev.alpha;
  const double a2 = al * al, a3 = a2 * al;
  const double b00 = 2.0 * a3 - 3.0 * a2 + 1.0, b10 = a3 - 2.0 * a2 + al, b01 = 3.0 * a2 - 2.0 * a3,
               b11 = a3 - a2;
  const double d00 = 6.0 * a2 - 6.0 * al, d10 = 3.0 * a2 - 4.0 * al + 1.0, d01 = 6.0 * al - 6.0 * a2,
               d11 = 3.0 * a2 - 2.0 * al;
  D yh[ng], cd[C::kC];
  for (int i = 0; i < ng; ++i)
    yh[i] = D::var(b00 * ev.yp[i] + b10 * (h * fe[0][i]) + b01 * ev.y[i] + b11 * (h * fe[1][i]), i);
  for (int j = 0; j < C::kC; ++j) cd[j] = D::var(c[j], ng + j);
  SmPrm<D> Pd;
  Pd.a = D::var(P.a, ng + C::kC);
  Pd.Q = D::var(P.Q, ng + C::kC + 1);
  Pd.L = D::var(P.L, ng + C::kC + 2);
  const D r = C::radius(Pd.a, yh);
  D pph;
  if constexpr (n == 6)
    pph = yh[0] * yh[4] - yh[1] * yh[3];  // KS: L_z = X p_Y - Y p_X
  else
    pph = cd[C::kC - 1];
  D red;
  bool has;
  if constexpr (C::kBundle)
    has = sm_redshift_bundle<D>(M, Pd, r, cd[0], pph, &red) && ev.deriv;
  else
    has = sm_redshift<D>(M, Pd, r, cd[0], pph, &red) && ev.deriv;
  double yhb[ng];
  for (int i = 0; i < ng; ++i) yhb[i] = rbar * r.d[i] + (has ? gbar * red.d[i] : 0.0);
  for (int j = 0; j < C::kC; ++j) cbar[j] = cbar[j] + rbar * r.d[ng + j] + (has ? gbar * red.d[ng + j] : 0.0);
  for (int q = 0; q < kSmPrm; ++q)
    pbar[q] = pbar[q] + rbar * r.d[ng + C::kC + q] + (has ? gbar * red.d[ng + C::kC + q] : 0.0);
  // alpha
  double alb = 0.0;
  for (int i = 0; i < ng; ++i)
    alb = alb + yhb[i] * (d00 * ev.yp[i] + d10 * (h * fe[0][i]) + d01 * ev.y[i] + d11 * (h * fe[1][i]));
  double Jb[4] = {0.0, 0.0, 0.0, 0.0};
  if (C::kBundle && ev.mderiv && mbar != 0.0) {
    double J[4];
    for (int m = 0; m < 4; ++m) J[m] = ev.yp[4 + m] + al * (ev.y[4 + m] - ev.yp[4 + m]);
    const double sg = (J[0] * J[3] - J[1] * J[2]) < 0.0 ? -mbar : mbar;
    Jb[0] = sg * J[3];
    Jb[1] = -sg * J[2];
    Jb[2] = -sg * J[1];
    Jb[3] = sg * J[0];
    for (int m = 0; m < 4; ++m) alb = alb + Jb[m] * (ev.y[4 + m] - ev.yp[4 + m]);
  }
  const int e = C::kEq;
  const double dqda = d00 * ev.yp[e] + d10 * (h * fe[0][e]) + d01 * ev.y[e] + d11 * (h * fe[1][e]);
  const double lam = -alb / dqda;
  double fb[2][n];
  double hb = 0.0;
  for (int i = 0; i < n; ++i) {
    const double g = i < ng ? yhb[i] + (i == e ? lam : 0.0) : 0.0;
    ybp[i] = b00 * g;
    ybN[i] = b01 * g;
    fb[0][i] = b10 * h * g;
    fb[1][i] = b11 * h * g;
    hb = hb + (b10 * fe[0][i] + b11 * fe[1][i]) * g;
  }
  if (C::kBundle)
    for (int m = 0; m < 4; ++m) {
      ybp[4 + m] = ybp[4 + m] + (1.0 - al) * Jb[m];
      ybN[4 + m] = ybN[4 + m] + al * Jb[m];
    }
  double ub[n];
  KT_ROLLED
  for (int w = 0; w < 2; ++w) {
    sm_vjp_f<C>(M, P, w == 0 ? ev.yp : ev.y, c, fb[w], ub, cbar, pbar);
    for (int i = 0; i < n; ++i) {
      if (w == 0)
        ybp[i] = ybp[i] + ub[i];
      else
        ybN[i] = ybN[i] + ub[i];
    }
  }
  *hbar = hb;
}

// Scratch of one ray's adjoint (per thread, local memory).
template <int N>
struct SmScratch {
  SmCk<N> ck1[kSmCkCap];
  SmCk<N> ck2[kSmCkCap];
  SmSt<N> st[sm_ring_steps<N>()];  // the forward's ring; replays reuse st[0..31]
  SmStages<N> stages;
};

// Reverse sweep of a ray traced with recording (N accepted steps, the last
// one ending in the disk event `ev`, checkpoints every k1 steps in
// sc->ck1).  Returns the cotangents of the initial state, the constants
// and (a, Q, Lambda).  The initial dlam is a constant (step_init).
template <class C, class I = SmRk4>
KT_HD void sm_adjoint(const Frame& f, const SmPrm<double>& P, const double* c, const SmEvent<C::kN>& ev,
                      int N, int k1, double gbar, double rbar, double mbar, SmScratch<C::kN>* sc,
                      double* ybar, double* cbar, double* pbar) {
  double ybN[C::kN], yb_direct[C::kN], hbar_ev = 0.0;
  for (int j = 0; j < C::kC; ++j) cbar[j] = 0.0;
  for (int q = 0; q < kSmPrm; ++q) pbar[q] = 0.0;
  sm_event_bwd<C>(f, P, c, ev, gbar, rbar, mbar, yb_direct, ybN, cbar, pbar, &hbar_ev);
  // The walk starts at step N-1 with the cotangent of y_N (H_N unused); the
  // direct seed of y_{N-1} joins after that step.
  for (int i = 0; i < C::kN; ++i) ybar[i] = ybN[i];
  double Hbar = 0.0;
  bool last = true;
  // Steps from N - R on are still in the forward's ring (step t at st[t % R];
  // a sub-segment starts at a multiple of 32, so its entries are contiguous).
  // Older sub-segments are replayed into st[0..31]: the reverse reaches them
  // only after every ring entry has been used.
  constexpr int R = sm_ring_steps<C::kN>();
  const int in_ring = N - R;
  const int nseg = (N + k1 - 1) / k1;
  KT_ROLLED
  for (int sgi = nseg - 1; sgi >= 0; --sgi) {
    const int s0 = sgi * k1;
    const int len = (N - s0 < k1) ? N - s0 : k1;
    const int nsub = (len + kSmCkSteps - 1) / kSmCkSteps;
    if (nsub > 1 && s0 < in_ring)
      sm_replay<C, I>(f, P, c, sc->ck1[sgi], len, nullptr, sc->ck2, kSmCkSteps);
    KT_ROLLED
    for (int sub = nsub - 1; sub >= 0; --sub) {
      const int t0 = sub * kSmCkSteps;
      const int tl = (len - t0 < kSmCkSteps) ? len - t0 : kSmCkSteps;
      const SmSt<C::kN>* st = sc->st;
      if (s0 + t0 >= in_ring)
        st = sc->st + (s0 + t0) % R;
      else
        sm_replay<C, I>(f, P, c, nsub > 1 ? sc->ck2[sub] : sc->ck1[sgi], tl, sc->st, nullptr, 0);
      KT_ROLLED
      for (int m = tl - 1; m >= 0; --m) {
        sm_step_bwd<C, I>(f, P, c, st[m], last ? hbar_ev : 0.0, ybar, &Hbar, cbar, pbar,
                          &sc->stages);
        if (last) {
          for (int i = 0; i < C::kN; ++i) ybar[i] = ybar[i] + yb_direct[i];
          last = false;
        }
      }
    }
  }
}

}  // namespace kt

namespace kt {

// Where a disk-hit pixel's cotangents come from.
struct SmCot {
  int mode;  // 0: forward only; 1: arrays g, r (and m); 2: L2 loss against a target frame
  const double* g;
  const double* r;
  const uint8_t* t_out;
  const double* t_g;
  const double* t_r;
  double w_g, w_r;
  const double* m;    // cotangent of the magnification (mode 1; bundles)
  const double* t_m;  // target magnification (mode 2; bundles)
  double w_m;
};

// A launch of the smooth kernel with gradients: cotangent source, chart
// override (trace every ray in the BL chart), reverse sweep (tangent_dir < 0)
// or forward-mode tangent along one parameter (tangent_dir = kGA..kGRobs),
// the [kGSlots][n] output (indexed by pixel) and an optional pixel list.
struct SmJob {
  SmCot cot;
  int force_bl;
  int tangent_dir;
  double* contrib;
  const uint32_t* pix;  // trace only these pixels (n_pix of them), or all when NULL
  uint32_t n_pix;
};

// Gradient slots of one pixel (and of the frame after the sum): dL/d(a, Q,
// Lambda, theta_obs [rad], r_obs), the loss, and counts: pixels whose
// reverse sweep ran, pixels traced in the BL chart, disk hits with a
// cotangent but more than 131072 steps (no gradient).
enum : int {
  kGA = 0, kGQ = 1, kGLambda = 2, kGTheta = 3, kGRobs = 4, kGLoss = 5, kGNumGrad = 6, kGNumBL = 7,
  kGNumUnrecorded = 8, kGSlots = 9
};

// init_bundle (ray_bundle.hpp:278-298): W's columns are the central
// differences of the camera ray (r, theta, p_r, p_theta) over alpha and beta
// with the half-pixel step f.bundle_eps, here in T (the camera's own
// parameters carried as Duals for the chain to theta_obs, r_obs, a, Q, Lambda).
template <class T>
KT_HD void sm_bundle_w0(const Frame& f, double M, const SmPrm<T>& P, const T& r_obs, const T& th_obs,
                        double al, double be, T* W) {
  const double eps = f.bundle_eps;
  T yp[4], ym[4], cp[2], cm[2];
  KT_ROLLED
  for (int k = 0; k < 2; ++k) {
    sm_camera<T>(M, P, r_obs, th_obs, k == 0 ? al + eps : al, k == 0 ? be : be + eps, yp, cp);
    sm_camera<T>(M, P, r_obs, th_obs, k == 0 ? al - eps : al, k == 0 ? be : be - eps, ym, cm);
    for (int i = 0; i < 4; ++i) W[2 * i + k] = (yp[i] - ym[i]) / (2.0 * eps);
  }
}

// One pixel of the smooth tracer in chart C: outputs into *o; with a
// cotangent source, the pixel's loss, gradient (theta in radians) and counts
// into g[kGSlots].  In the KS chart a ray whose KS initialisation fails
// (init_ks_state, main.cpp:1533-1538) is not traced: returns false, and the
// caller hands it to the BL chart.
template <class C, bool kGrad, class I = SmRk4>
KT_HD bool sm_pixel(const Frame& f, uint32_t pix, const SmCot& cot, RayResult* o, double* g,
                    SmScratch<C::kN>* sc) {
  constexpr bool kKS = C::kN == 6;
  const int px = (int)(pix % (uint32_t)f.cam.W), py = (int)(pix / (uint32_t)f.cam.W);
  double al, be;
  pixel_angles(f.cam, px, py, &al, &be);
  const double M = f.g.M;
  const SmPrm<double> P = sm_prm<double>(f.g);
  double ybl[4], cbl[2], y0[C::kN], c0[C::kC];
  sm_camera<double>(M, P, f.cam.r_obs, f.cam.theta_obs, al, be, ybl, cbl);
  if (kKS) {
    double yk[6], ck[1];
    if (!sm_bl_to_ks<double>(M, P, ybl, cbl, f.cam.phi_obs, yk, ck)) return false;
    for (int i = 0; i < C::kN; ++i) y0[i] = yk[i];
    c0[0] = ck[0];
  } else {
    for (int i = 0; i < 4; ++i) y0[i] = ybl[i];
    for (int j = 0; j < C::kC; ++j) c0[j] = cbl[j];
    if constexpr (C::kBundle) sm_bundle_w0<double>(f, M, P, f.cam.r_obs, f.cam.theta_obs, al, be, y0 + 4);
  }
  SmEvent<C::kN> ev;
  int k1 = 0, nck = 0;
  SmCk<C::kN>* ck = kGrad ? sc->ck1 : nullptr;
  const int N = sm_trace<C, I>(f, P, y0, c0, kKS ? 0.0 : f.cam.phi_obs, o, &ev, ck, &k1, &nck,
                               kGrad ? sc->st : nullptr);
  if (!kGrad) return true;
  for (int q = 0; q < kGSlots; ++q) g[q] = 0.0;
  g[kGNumBL] = kKS ? 0.0 : 1.0;
  if (o->outcome != kOutDisk) return true;
  double gbar = 0.0, rbar = 0.0, mbar = 0.0;
  if (cot.mode == 1) {
    gbar = cot.g ? cot.g[pix] : 0.0;
    rbar = cot.r ? cot.r[pix] : 0.0;
    mbar = (C::kBundle && cot.m) ? cot.m[pix] : 0.0;
  } else if (cot.mode == 2) {
    if (cot.t_out[pix] != kOutDisk) return true;
    const double dg = o->red - cot.t_g[pix], dr = o->r - cot.t_r[pix];
    g[kGLoss] = cot.w_g * dg * dg + cot.w_r * dr * dr;
    gbar = 2.0 * cot.w_g * dg;
    rbar = 2.0 * cot.w_r * dr;
    if (C::kBundle && cot.t_m && cot.w_m != 0.0) {
      const double dm = o->magnif - cot.t_m[pix];
      g[kGLoss] = g[kGLoss] + cot.w_m * dm * dm;
      mbar = 2.0 * cot.w_m * dm;
    }
  }
  if (gbar == 0.0 && rbar == 0.0 && mbar == 0.0) return true;
  if (N == 0) {
    g[kGNumUnrecorded] = 1.0;
    return true;
  }
  g[kGNumGrad] = 1.0;
  double ybar[C::kN], cbar[C::kC], pbar[kSmPrm];
  sm_adjoint<C, I>(f, P, c0, ev, N, k1, gbar, rbar, mbar, sc, ybar, cbar, pbar);
  // chain through the camera ray: Dual over (a, Q, Lambda, theta_obs, r_obs)
  typedef Dual<5> D5;
  SmPrm<D5> Pd;
  Pd.a = D5::var(P.a, 0);
  Pd.Q = D5::var(P.Q, 1);
  Pd.L = D5::var(P.L, 2);
  const D5 thd = D5::var(f.cam.theta_obs, 3), rd = D5::var(f.cam.r_obs, 4);
  D5 yb5[4], cb5[2], y5[C::kN], c5[C::kC];
  sm_camera<D5>(M, Pd, rd, thd, al, be, yb5, cb5);
  if (kKS) {
    D5 yk[6], ck5[1];
    sm_bl_to_ks<D5>(M, Pd, yb5, cb5, f.cam.phi_obs, yk, ck5);
    for (int i = 0; i < C::kN; ++i) y5[i] = yk[i];
    c5[0] = ck5[0];
  } else {
    for (int i = 0; i < 4; ++i) y5[i] = yb5[i];
    for (int j = 0; j < C::kC; ++j) c5[j] = cb5[j];
    if constexpr (C::kBundle) sm_bundle_w0<D5>(f, M, Pd, rd, thd, al, be, y5 + 4);
  }
  for (int k = 0; k < 5; ++k) {
    double acc = k < kSmPrm ? pbar[k] : 0.0;
    for (int j = 0; j < C::kC; ++j) acc = acc + cbar[j] * c5[j].d[k];
    for (int i = 0; i < C::kN; ++i) acc = acc + ybar[i] * y5[i].d[k];
    g[k] = acc;
  }
  return true;
}

// ---- forward-mode tangent along one parameter -----------------------------
// The same tracer with every quantity a Dual<1>: the values are computed by
// the same operations in the same order as sm_trace's, so the trace (steps,
// events, outputs) is the smooth forward's bit for bit, and the tangents are
// the derivative of the discrete map along one parameter, the controller
// included (the derivative the reverse sweep gives for that parameter).
// Cost: one pass, no checkpoints; used where a single derivative is needed
// (a KS frame's Lambda entry, which lives in the BL chart).
typedef Dual<1> T1;

template <class C>
KT_HD_CALL void sm_paths_t(double M, const SmPrm<T1>& P, const T1* c, const T1* y, double pas,
                           const T1* k1, double k1p, const T1& hh, T1* yA, T1* yB, double* pB,
                           T1* dAB) {
  constexpr int n = C::kN;
  T1 base[n], kp[n], sum[n], yB1[n], u[n], k[n], kk, incA[n], incB1[n];
  double pbase = pas, sump = k1p, pB1 = pas;
  KT_ROLLED
  for (int t = 0; t < 10; ++t) {
    int sub, s;
    sm_stage_of(t, &sub, &s);
    const T1 hs = sub == 0 ? hh : 0.5 * hh;
    if (s == 1 && sub < 2) {
      for (int i = 0; i < n; ++i) {
        base[i] = y[i];
        kp[i] = k1[i];
        sum[i] = k1[i];
      }
      pbase = pas;
      sump = k1p;
    }
    if (s == 0) {
      for (int i = 0; i < n; ++i) {
        base[i] = yB1[i];
        u[i] = yB1[i];
      }
      pbase = pB1;
    } else {
      const T1 cs = (s == 3) ? hs : 0.5 * hs;
      for (int i = 0; i < n; ++i) u[i] = base[i] + cs * kp[i];
    }
    sm_rhs<C>(M, P, u, c, k, &kk);
    if (s == 0) {
      for (int i = 0; i < n; ++i) {
        kp[i] = k[i];
        sum[i] = k[i];
      }
      sump = kk.v;
      continue;
    }
    const double w = (s == 3) ? 1.0 : 2.0;
    for (int i = 0; i < n; ++i) {
      sum[i] = sum[i] + w * k[i];
      kp[i] = k[i];
    }
    sump = sump + w * kk.v;
    if (s == 3) {
      for (int i = 0; i < n; ++i) {
        const T1 inc = hs / 6.0 * sum[i];
        const T1 r = base[i] + inc;
        if (sub == 0) {
          yA[i] = r;
          incA[i] = inc;
        }
        if (sub == 1) {
          yB1[i] = r;
          incB1[i] = inc;
        }
        if (sub == 2) {
          yB[i] = r;
          dAB[i] = incA[i] - (incB1[i] + inc);
        }
      }
      const double pr = pbase + hs.v / 6.0 * sump;
      pB1 = sub == 1 ? pr : pB1;
      *pB = sub == 2 ? pr : *pB;
    }
  }
}

// doubling_update on Dual<1>: the same branches on the values; the new dlam's
// tangent from the step size's and the error's.
KT_HD int sm_update_t(const T1& err, double tol, T1* h) {
  if (!finite(err.v)) {
    const bool big = finite(h->v) && h->v > 1e-10;
    *h = big ? (*h) * 0.5 : T1(1e-6);
    if (h->v < 1e-10) *h = T1(1e-10);
    return -1;
  }
  const bool accepted = (err.v < tol || h->v < 1e-10);
  if (accepted) {
    T1 scale(4.0);
    if (err.v > 1e-14) {
      scale.v = 0.9 * ktm_pow(tol / err.v, 0.2);
      scale.d[0] = -0.2 * scale.v / err.v * err.d[0];
    }
    T1 hn = (*h) * scale;
    if (!finite(hn.v)) hn = *h;
    *h = hn;
    if (h->v > 100.0) *h = T1(100.0);
    if (h->v < 1e-10) *h = T1(1e-10);
  } else {
    const T1 half = (*h) * 0.5;
    const T1 h09 = (*h) * 0.9;
    const double pw = ktm_pow(tol / err.v, 0.25);
    T1 hn;
    hn.v = h09.v * pw;
    hn.d[0] = h09.d[0] * pw + h09.v * (-0.25 * pw / err.v * err.d[0]);
    if (!finite(hn.v)) hn = half;
    *h = hn;
    if (h->v > half.v) *h = half;
    if (h->v < 1e-10) *h = T1(1e-10);
  }
  return accepted ? 1 : 0;
}

template <class C>
KT_HD int sm_attempt_t(double M, const SmPrm<T1>& P, double tol, const T1* c, const T1* y, double pas,
                       const T1* k1, double k1p, T1* h, T1* yo, double* paso) {
  T1 yA[C::kN], yB[C::kN], dAB[C::kN];
  double pB = 0.0;
  sm_paths_t<C>(M, P, c, y, pas, k1, k1p, *h, yA, yB, &pB, dAB);
  T1 e2(0.0);
  for (int i = 0; i < C::kN; ++i) {
    const T1 d = dAB[i];
    e2 = e2 + d * d;
  }
  T1 err(sqrt(e2.v) / 15.0);
  if (e2.v > 0.0) err = sm_sqrt(e2) / 15.0;
  const int res = sm_update_t(err, tol, h);
  if (res == 1) {
    for (int i = 0; i < C::kN; ++i) yo[i] = yB[i];
    *paso = pB;
  }
  return res;
}

// sm_trace on Dual<1> (no recording).  On a disk hit: returns true with the
// hit radius and redshift carrying their tangents (*deriv = 0 where the
// redshift is a constant or clamped).
template <class C>
KT_HD bool sm_trace_t(const Frame& f, const SmPrm<T1>& P, const T1* y_in, const T1* c, double pas_in,
                      RayResult* o, T1* r_out, T1* g_out, int* deriv_out) {
  const double M = f.g.M;
  T1 y[C::kN], yp[C::kN], k1[C::kN], kprev[C::kN], kpT;
  double pas = pas_in, pasp, k1p, kprevp;
  for (int i = 0; i < C::kN; ++i) y[i] = y_in[i];
  T1 h(f.dlam0);
  uint32_t attempts = 0;
  sm_rhs<C>(M, P, y, c, k1, &kpT);
  k1p = kpT.v;
  double prev_r = C::radius(f.g.a, y).v;
  KT_ROLLED
  for (int it = 0;; ++it) {
    for (int i = 0; i < C::kN; ++i) {
      yp[i] = y[i];
      kprev[i] = k1[i];
    }
    pasp = pas;
    kprevp = k1p;
    T1 step_used = h;
    int rejects = 0;
    KT_ROLLED
    for (;;) {
      step_used = h;
      ++attempts;
      if (sm_attempt_t<C>(M, P, f.tol, c, yp, pasp, kprev, kprevp, &h, y, &pas) == 1) break;
      int status;
      if (reject_cap(h.v, &rejects, &status)) {
        double yv[C::kN];
        for (int i = 0; i < C::kN; ++i) yv[i] = yp[i].v;
        sm_stop<C>(f, yv, pasp, status, (uint32_t)it, attempts, o);
        return false;
      }
    }
    sm_rhs<C>(M, P, y, c, k1, &kpT);
    k1p = kpT.v;
    double yv[C::kN], ypv[C::kN];
    for (int i = 0; i < C::kN; ++i) {
      yv[i] = y[i].v;
      ypv[i] = yp[i].v;
    }
    const double r_now = C::radius(f.g.a, yv);
    double best_alpha = 2.0;
    int evt = kEvNone;
    T1 disk_r(0.0), disk_red(1.0);
    double disk_phi = 0.0;
    int deriv = 0;
    const int e = C::kEq;
    const double q0 = ypv[e] - C::kEqTarget, q1 = yv[e] - C::kEqTarget;
    if (sign_change(q0, q1) || dmin(fabs(q0), fabs(q1)) < 0.35) {
      double alpha = 0.0;
      if (sm_first_crossing(ypv[e], yv[e], kprev[e].v, k1[e].v, step_used.v, C::kEqTarget, &alpha)) {
        // alpha* moves with the parameter: d alpha = -dq / q'(alpha)
        const T1 q = sm_hermite_h(yp[e], y[e], kprev[e], k1[e], step_used, T1(alpha)) - C::kEqTarget;
        const double dqda = sm_hermite_da(ypv[e], yv[e], kprev[e].v, k1[e].v, step_used.v, alpha);
        T1 al(alpha);
        al.d[0] = -q.d[0] / dqda;
        T1 yh[C::kN];
        for (int i = 0; i < C::kN; ++i) yh[i] = sm_hermite_h(yp[i], y[i], kprev[i], k1[i], step_used, al);
        const T1 r_hit = C::radius(P.a, yh);
        if (r_hit.v >= f.r_in && r_hit.v <= f.r_out) {
          T1 pph;
          if constexpr (C::kN == 6)
            pph = yh[0] * yh[4] - yh[1] * yh[3];
          else
            pph = c[C::kC - 1];
          T1 red;
          deriv = sm_redshift<T1>(M, P, r_hit, c[0], pph, &red) ? 1 : 0;
          if (!(red.v > 0.0 && red.v < 20.0)) deriv = 0;
          disk_r = r_hit;
          disk_red = red;
          if (C::kN == 6) {
            double rr, tt;
            ks_to_bl(f.g, yh[0].v, yh[1].v, yh[2].v, &rr, &tt, &disk_phi);
          } else {
            disk_phi = pasp + alpha * (pas - pasp);
          }
          best_alpha = alpha;
          evt = kEvDisk;
        }
      }
    }
    horizon_escape(prev_r, r_now, f.rh_cut, f.r_esc, &best_alpha, &evt);
    if (evt != kEvNone) {
      o->steps = (uint32_t)it + 1;
      o->attempts = attempts;
      if (evt == kEvDisk) {
        set_result(o, kOutDisk, kStEvent, disk_r.v, dclamp(disk_red.v, 0.0, 20.0), 1.0, disk_phi, 0.0,
                   0.0);
        *r_out = disk_r;
        *g_out = disk_red;
        *deriv_out = deriv;
        return true;
      }
      if (evt == kEvHorizon) {
        set_result(o, kOutHorizon, kStEvent, prev_r + best_alpha * (r_now - prev_r), 0.0, 1.0, 0.0,
                   0.0, 0.0);
      } else if (C::kN == 6) {
        double xe[3];
        for (int i = 0; i < 3; ++i) xe[i] = ypv[i] + best_alpha * (yv[i] - ypv[i]);
        double re, te, pe;
        ks_to_bl(f.g, xe[0], xe[1], xe[2], &re, &te, &pe);
        set_result(o, kOutEscaped, kStEvent, re, 1.0, 1.0, te, pe, 0.0);
      } else {
        const double te = ypv[1] + best_alpha * (yv[1] - ypv[1]);
        const double pe = pasp + best_alpha * (pas - pasp);
        set_result(o, kOutEscaped, kStEvent, f.r_esc, 1.0, 1.0, te, pe, 0.0);
      }
      return false;
    }
    prev_r = r_now;
    if (it + 1 >= f.max_steps) {
      sm_stop<C>(f, yv, pas, kStStepCap, (uint32_t)(it + 1), attempts, o);
      return false;
    }
  }
}

// One pixel with the tangent along parameter `dir` (kGA..kGRobs): outputs
// into *o, g[kGSlots] as sm_pixel's with only g[dir] set among the
// derivatives.  Returns false where the KS initialisation fails (KS chart).
template <class C>
KT_HD bool sm_pixel_tangent(const Frame& f, uint32_t pix, int dir, const SmCot& cot, RayResult* o,
                            double* g, bool need_out = true) {
  constexpr bool kKS = C::kN == 6;
  if (!need_out) {
    // a pixel whose cotangent is zero whatever its trace gives contributes
    // nothing: a target pixel off the disk, or zero cotangent entries
    const bool zero = cot.mode == 2 ? cot.t_out[pix] != kOutDisk
                                    : (!cot.g || cot.g[pix] == 0.0) && (!cot.r || cot.r[pix] == 0.0);
    if (zero) {
      for (int q = 0; q < kGSlots; ++q) g[q] = 0.0;
      g[kGNumBL] = kKS ? 0.0 : 1.0;
      return true;
    }
  }
  const int px = (int)(pix % (uint32_t)f.cam.W), py = (int)(pix / (uint32_t)f.cam.W);
  double al, be;
  pixel_angles(f.cam, px, py, &al, &be);
  const double M = f.g.M;
  SmPrm<T1> Pd;
  Pd.a = T1(f.g.a);
  Pd.Q = T1(f.g.Q);
  Pd.L = T1(f.g.L);
  T1 th(f.cam.theta_obs), ro(f.cam.r_obs);
  if (dir == kGA) Pd.a.d[0] = 1.0;
  if (dir == kGQ) Pd.Q.d[0] = 1.0;
  if (dir == kGLambda) Pd.L.d[0] = 1.0;
  if (dir == kGTheta) th.d[0] = 1.0;
  if (dir == kGRobs) ro.d[0] = 1.0;
  T1 ybl[4], cbl[2], y0[C::kN], c0[C::kC];
  sm_camera<T1>(M, Pd, ro, th, al, be, ybl, cbl);
  if (kKS) {
    T1 yk[6], ck[1];
    if (!sm_bl_to_ks<T1>(M, Pd, ybl, cbl, f.cam.phi_obs, yk, ck)) return false;
    for (int i = 0; i < C::kN; ++i) y0[i] = yk[i];
    c0[0] = ck[0];
  } else {
    for (int i = 0; i < C::kN; ++i) y0[i] = ybl[i];
    for (int j = 0; j < C::kC; ++j) c0[j] = cbl[j];
  }
  T1 r_hit, g_hit;
  int deriv = 0;
  const bool disk = sm_trace_t<C>(f, Pd, y0, c0, kKS ? 0.0 : f.cam.phi_obs, o, &r_hit, &g_hit, &deriv);
  for (int q = 0; q < kGSlots; ++q) g[q] = 0.0;
  g[kGNumBL] = kKS ? 0.0 : 1.0;
  if (!disk) return true;
  double gbar = 0.0, rbar = 0.0;
  if (cot.mode == 1) {
    gbar = cot.g ? cot.g[pix] : 0.0;
    rbar = cot.r ? cot.r[pix] : 0.0;
  } else if (cot.mode == 2) {
    if (cot.t_out[pix] != kOutDisk) return true;
    const double dg = o->red - cot.t_g[pix], dr = o->r - cot.t_r[pix];
    g[kGLoss] = cot.w_g * dg * dg + cot.w_r * dr * dr;
    gbar = 2.0 * cot.w_g * dg;
    rbar = 2.0 * cot.w_r * dr;
  }
  if (gbar == 0.0 && rbar == 0.0) return true;
  g[kGNumGrad] = 1.0;
  g[dir] = rbar * r_hit.d[0] + (deriv ? gbar * g_hit.d[0] : 0.0);
  return true;
}

}  // namespace kt
