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
//     outputs are evaluated in Dual<2n + c + 3> over (y_{N-1}, y_N, constants,
//     a, Q, Lambda) with alpha* carrying that derivative;
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
//     inner checkpoints every 32 steps.
// VJP of the RHS f = J grad_y H (J = [[0, I], [-I, 0]]): v^T df/dy =
// H_yy (J^T v) and v^T df/dc = d/dc (grad_y H) . (J^T v) = the derivative of
// dH/dc along J^T v, so one Dual<1> evaluation of the full gradient of H along
// d = J^T v = (-v_p, v_x) gives the state, constant and parameter cotangents.
#pragma once

#include "kt_smooth.cuh"

namespace kt {

constexpr int kSmCkSteps = 32;  // accepted steps between checkpoints
constexpr int kSmCkCap = 64;    // checkpoints per level
constexpr int kSmMaxN = 6;
constexpr int kSmMaxDoublings = 6;  // k up to 32 * 2^6: 131072 accepted steps

struct SmCk {  // state at the start of an accepted step and dlam before its attempts
  double y[kSmMaxN];
  double h;
};

struct SmSt {  // state at the start of an accepted step and dlam before its attempts
  double y[kSmMaxN];
  double H;
};

// Data of the final (event) step kept for the adjoint.
struct SmEvent {
  double yp[kSmMaxN];  // y_{N-1}
  double y[kSmMaxN];   // y_N
  double H;            // dlam before the attempts of step N-1
  double h;            // accepted step size of step N-1
  double alpha;
  int deriv;           // 1: redshift has a derivative (not a constant or clamped)
};

// Primal RK4 step of size h from y with k1 = f(y); the passenger (BL phi)
// rides along.  Stage inputs y + h/2 k1, y + h/2 k2, y + h k3; result
// y + h/6 (k1 + 2 k2 + 2 k3 + k4) (rk4_step_ks, main.cpp:1456-1486).
template <class C>
KT_HD void sm_rk4(double M, const SmPrm<double>& P, const double* c, const double* y, double pas,
                  const double* k1, double k1p, double h, double* yo, double* paso) {
  double u[C::kN], k[C::kN], sum[C::kN], kp, sump = k1p;
  for (int i = 0; i < C::kN; ++i) {
    sum[i] = k1[i];
    u[i] = y[i] + 0.5 * h * k1[i];
  }
  sm_rhs<C>(M, P, u, c, k, &kp);
  for (int i = 0; i < C::kN; ++i) {
    sum[i] = sum[i] + 2.0 * k[i];
    u[i] = y[i] + 0.5 * h * k[i];
  }
  sump = sump + 2.0 * kp;
  sm_rhs<C>(M, P, u, c, k, &kp);
  for (int i = 0; i < C::kN; ++i) {
    sum[i] = sum[i] + 2.0 * k[i];
    u[i] = y[i] + h * k[i];
  }
  sump = sump + 2.0 * kp;
  sm_rhs<C>(M, P, u, c, k, &kp);
  for (int i = 0; i < C::kN; ++i) yo[i] = y[i] + h / 6.0 * (sum[i] + k[i]);
  *paso = pas + h / 6.0 * (sump + kp);
}

// One adaptive attempt from (y, pas) with k1 = f(y) and step *h: path A one
// step h, path B two steps h/2 (mid point ym), err = |A - B| / 15.  Returns
// doubling_update's result; on acceptance (yo, paso) = B.
template <class C>
KT_HD int sm_attempt(double M, const SmPrm<double>& P, double tol, const double* c, const double* y,
                     double pas, const double* k1, double k1p, double* h, double* yo, double* paso,
                     double* ym) {
  double yA[C::kN], yB1[C::kN], yB[C::kN], kb[C::kN], pA, pB1, pB, kbp;
  const double hh = *h;
  sm_rk4<C>(M, P, c, y, pas, k1, k1p, hh, yA, &pA);
  sm_rk4<C>(M, P, c, y, pas, k1, k1p, 0.5 * hh, yB1, &pB1);
  sm_rhs<C>(M, P, yB1, c, kb, &kbp);
  sm_rk4<C>(M, P, c, yB1, pB1, kb, kbp, 0.5 * hh, yB, &pB);
  double e2 = 0.0;
  for (int i = 0; i < C::kN; ++i) {
    const double d = yA[i] - yB[i];
    e2 = e2 + d * d;
  }
  const int res = doubling_update(sqrt(e2) / 15.0, tol, h);
  if (res == 1) {
    for (int i = 0; i < C::kN; ++i) {
      yo[i] = yB[i];
      if (ym) ym[i] = yB1[i];
    }
    *paso = pB;
  }
  return res;
}

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
  set_result(o, kOutEscaped, status, rr, 1.0, 1.0, tt, pp, 0.0);
}

// Trace one ray from (y, c, pas).  With ck != NULL, checkpoints are recorded
// (*ck_k = final interval, *ck_n = count).  On a disk hit `ev` receives the
// final step; returns the number of accepted steps N (0 if the ray ended
// otherwise or more than 131072 steps were taken with recording on).
template <class C>
KT_HD int sm_trace(const Frame& f, const SmPrm<double>& P, const double* y_in, const double* c,
                   double pas_in, RayResult* o, SmEvent* ev, SmCk* ck, int* ck_k, int* ck_n) {
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
    double step_used = h;
    int rejects = 0;
    KT_ROLLED
    for (;;) {
      step_used = h;
      ++attempts;
      if (sm_attempt<C>(M, P, f.tol, c, yp, pasp, kprev, kprevp, &h, y, &pas, nullptr) == 1) break;
      int status;
      if (reject_cap(h, &rejects, &status)) {
        sm_stop<C>(f, yp, pasp, status, (uint32_t)it, attempts, o);
        return 0;
      }
    }
    sm_rhs<C>(M, P, y, c, k1, &k1p);
    // events (main.cpp:1570-1657, 364-433)
    const double r_now = C::radius(f.g.a, y);
    double best_alpha = 2.0;
    int evt = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    int deriv = 0;
    const double q0 = yp[C::kEq] - C::kEqTarget, q1 = y[C::kEq] - C::kEqTarget;
    if (sign_change(q0, q1) || dmin(fabs(q0), fabs(q1)) < 0.35) {
      double alpha = 0.0;
      if (sm_first_crossing(yp[C::kEq], y[C::kEq], kprev[C::kEq], k1[C::kEq], step_used,
                            C::kEqTarget, &alpha)) {
        double yh[C::kN];
        for (int i = 0; i < C::kN; ++i) yh[i] = sm_hermite(yp[i], y[i], kprev[i], k1[i], step_used, alpha);
        const double r_hit = C::radius(f.g.a, yh);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          double red, pph;
          if (C::kN == 6) {
            pph = yh[0] * yh[4] - yh[1] * yh[3];
          } else {
            pph = c[C::kC - 1];
          }
          deriv = sm_redshift<double>(M, P, r_hit, c[0], pph, &red) ? 1 : 0;
          if (!(red > 0.0 && red < 20.0)) deriv = 0;
          disk_r = r_hit;
          disk_red = dclamp(red, 0.0, 20.0);
          if (C::kN == 6) {
            double rr, tt;
            ks_to_bl(f.g, yh[0], yh[1], yh[2], &rr, &tt, &disk_phi);
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
        set_result(o, kOutDisk, kStEvent, disk_r, disk_red, 1.0, disk_phi, 0.0, 0.0);
        if (ev) {
          for (int i = 0; i < C::kN; ++i) {
            ev->yp[i] = yp[i];
            ev->y[i] = y[i];
          }
          ev->H = H_start;
          ev->h = step_used;
          ev->alpha = best_alpha;
          ev->deriv = deriv;
        }
        if (ck_k) *ck_k = k;
        if (ck_n) *ck_n = nck;
        return (ck == nullptr || rec_ok) ? it + 1 : 0;
      }
      if (evt == kEvHorizon) {
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
// dlam, rejections included).  Stores each step's start (y_n, H_n) into
// st[0..n) and/or a checkpoint every k2 steps into ck2.
template <class C>
KT_HD void sm_replay(const Frame& f, const SmPrm<double>& P, const double* c, const SmCk& ck0, int n,
                     SmSt* st, SmCk* ck2, int k2) {
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
    int rejects = 0;
    KT_ROLLED
    for (;;) {
      if (sm_attempt<C>(M, P, f.tol, c, y, pas, k1, k1p, &h, y1, &pas1, nullptr) == 1) break;
      int status;
      if (reject_cap(h, &rejects, &status)) break;  // not reached: the forward accepted
    }
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
template <class C>
KT_HD void sm_vjp_f(double M, const SmPrm<double>& P, const double* u, const double* c, const double* v,
                    double* ubar, double* cbar, double* pbar) {
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

// Reverse of one RK4 step of size h from y (sm_rk4's arithmetic).  In:
// ybar = cotangent of the result.  Out: ybar = cotangent of y, hbar += the
// step size's, cbar/pbar += the constants' and parameters'.  Optionally
// returns the result of the step in yo.
template <class C>
KT_HD void sm_rk4_bwd(double M, const SmPrm<double>& P, const double* c, const double* y, double h,
                      double* ybar, double* hbar, double* cbar, double* pbar, double* yo) {
  double u[4][C::kN], k[4][C::kN], kp;
  for (int i = 0; i < C::kN; ++i) u[0][i] = y[i];
  sm_rhs<C>(M, P, u[0], c, k[0], &kp);
  for (int i = 0; i < C::kN; ++i) u[1][i] = y[i] + 0.5 * h * k[0][i];
  sm_rhs<C>(M, P, u[1], c, k[1], &kp);
  for (int i = 0; i < C::kN; ++i) u[2][i] = y[i] + 0.5 * h * k[1][i];
  sm_rhs<C>(M, P, u[2], c, k[2], &kp);
  for (int i = 0; i < C::kN; ++i) u[3][i] = y[i] + h * k[2][i];
  sm_rhs<C>(M, P, u[3], c, k[3], &kp);
  if (yo)
    for (int i = 0; i < C::kN; ++i)
      yo[i] = y[i] + h / 6.0 * (k[0][i] + 2.0 * k[1][i] + 2.0 * k[2][i] + k[3][i]);
  double kb[4][C::kN], ub[C::kN];
  const double w[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
  const double beta[4] = {0.0, 0.5, 0.5, 1.0};  // u_s = y + beta_s h k_{s-1}
  double hb = 0.0;
  for (int s = 0; s < 4; ++s) {
    double dot = 0.0;
    for (int i = 0; i < C::kN; ++i) {
      kb[s][i] = w[s] * h * ybar[i];
      dot = dot + ybar[i] * k[s][i];
    }
    hb = hb + w[s] * dot;
  }
  KT_ROLLED
  for (int s = 3; s >= 0; --s) {
    sm_vjp_f<C>(M, P, u[s], c, kb[s], ub, cbar, pbar);
    double dot = 0.0;
    for (int i = 0; i < C::kN; ++i) {
      ybar[i] = ybar[i] + ub[i];
      if (s > 0) {
        kb[s - 1][i] = kb[s - 1][i] + beta[s] * h * ub[i];
        dot = dot + ub[i] * k[s - 1][i];
      }
    }
    if (s > 0) hb = hb + beta[s] * dot;
  }
  *hbar = *hbar + hb;
}

// Reverse of one attempt from y with size h: cotangents Abar (of path A's
// result) and Bbar (of path B's).  ybar += .., returns the size's cotangent.
template <class C>
KT_HD double sm_attempt_bwd(double M, const SmPrm<double>& P, const double* c, const double* y, double h,
                            const double* Abar, const double* Bbar, double* ybar, double* cbar,
                            double* pbar) {
  double yb1[C::kN], k1[C::kN], k1p, pas1, t[C::kN], hb_half = 0.0, hb_full = 0.0;
  sm_rhs<C>(M, P, y, c, k1, &k1p);
  sm_rk4<C>(M, P, c, y, 0.0, k1, k1p, 0.5 * h, yb1, &pas1);
  for (int i = 0; i < C::kN; ++i) t[i] = Bbar[i];
  sm_rk4_bwd<C>(M, P, c, yb1, 0.5 * h, t, &hb_half, cbar, pbar, nullptr);  // second half step
  sm_rk4_bwd<C>(M, P, c, y, 0.5 * h, t, &hb_half, cbar, pbar, nullptr);    // first half step
  for (int i = 0; i < C::kN; ++i) ybar[i] = ybar[i] + t[i];
  for (int i = 0; i < C::kN; ++i) t[i] = Abar[i];
  sm_rk4_bwd<C>(M, P, c, y, h, t, &hb_full, cbar, pbar, nullptr);
  for (int i = 0; i < C::kN; ++i) ybar[i] = ybar[i] + t[i];
  return 0.5 * hb_half + hb_full;
}

// Paths A and B of an attempt and its error (sm_attempt's arithmetic).
template <class C>
KT_HD double sm_attempt_err(double M, const SmPrm<double>& P, const double* c, const double* y, double h,
                            double* d) {
  double yA[C::kN], yB1[C::kN], yB[C::kN], k1[C::kN], kb[C::kN], k1p, kbp, pa;
  sm_rhs<C>(M, P, y, c, k1, &k1p);
  sm_rk4<C>(M, P, c, y, 0.0, k1, k1p, h, yA, &pa);
  sm_rk4<C>(M, P, c, y, 0.0, k1, k1p, 0.5 * h, yB1, &pa);
  sm_rhs<C>(M, P, yB1, c, kb, &kbp);
  sm_rk4<C>(M, P, c, yB1, 0.0, kb, kbp, 0.5 * h, yB, &pa);
  double e2 = 0.0;
  for (int i = 0; i < C::kN; ++i) {
    d[i] = yA[i] - yB[i];
    e2 = e2 + d[i] * d[i];
  }
  return sqrt(e2) / 15.0;
}

constexpr int kSmMaxAttempts = 66;  // reject cap 64 + the accepted attempt

// Reverse of accepted step n from (y_n, H_n).  In: ybar = cotangent of
// y_{n+1}, *Hbar = cotangent of H_{n+1}, hbar_acc = extra cotangent of the
// accepted size (the event's).  Out: ybar = cotangent of y_n, *Hbar = of H_n.
template <class C>
KT_HD void sm_step_bwd(const Frame& f, const SmPrm<double>& P, const double* c, const SmSt& st,
                       double hbar_acc, double* ybar, double* Hbar, double* cbar, double* pbar) {
  const double M = f.g.M;
  double hs[kSmMaxAttempts], es[kSmMaxAttempts], d[C::kN];
  // replay the attempts: sizes and errors
  int na = 0;
  double h = st.H;
  KT_ROLLED
  for (;;) {
    hs[na] = h;
    es[na] = sm_attempt_err<C>(M, P, c, st.y, h, d);
    const double e = es[na];
    ++na;
    const int res = doubling_update(e, f.tol, &h);
    if (res == 1 || na == kSmMaxAttempts) break;
  }
  double yb_out[C::kN], Abar[C::kN], Bbar[C::kN];
  for (int i = 0; i < C::kN; ++i) {
    yb_out[i] = ybar[i];
    ybar[i] = 0.0;
  }
  // accepted attempt: H_{n+1} = sigma(h_R, e_R), y_{n+1} = B(y_n, h_R)
  double dh, de;
  sm_ctl_partials(es[na - 1], f.tol, hs[na - 1], &dh, &de);
  double hb = *Hbar * dh + hbar_acc;
  double eb = *Hbar * de;
  KT_ROLLED
  for (int j = na - 1; j >= 0; --j) {
    // cotangent of e_j -> paths A and B through d = A - B
    const double e = es[j];
    sm_attempt_err<C>(M, P, c, st.y, hs[j], d);
    const double kap = (e > 0.0 && finite(e)) ? eb / (225.0 * e) : 0.0;
    for (int i = 0; i < C::kN; ++i) {
      Abar[i] = kap * d[i];
      Bbar[i] = (j == na - 1 ? yb_out[i] : 0.0) - kap * d[i];
    }
    hb = hb + sm_attempt_bwd<C>(M, P, c, st.y, hs[j], Abar, Bbar, ybar, cbar, pbar);
    if (j > 0) {
      // h_j = rho(h_{j-1}, e_{j-1}) (a rejection)
      sm_ctl_partials(es[j - 1], f.tol, hs[j - 1], &dh, &de);
      eb = hb * de;
      hb = hb * dh;
    }
  }
  *Hbar = hb;
}

// Cotangents of the event step's inputs from (gbar, rbar):
// (y_{N-1}, y_N, constants, prm, h) -> ybar_prev, ybar_N, cbar, pbar, hbar.
template <class C>
KT_HD void sm_event_bwd(double M, const SmPrm<double>& P, const double* c, const SmEvent& ev,
                        double gbar, double rbar, double* ybp, double* ybN, double* cbar,
                        double* pbar, double* hbar) {
  constexpr int NE = 2 * C::kN + C::kC + kSmPrm + 1;
  typedef Dual<NE> D;
  D yp[C::kN], y[C::kN], cd[C::kC], fp[C::kN], fN[C::kN], fpp, fNp;
  for (int i = 0; i < C::kN; ++i) {
    yp[i] = D::var(ev.yp[i], i);
    y[i] = D::var(ev.y[i], C::kN + i);
  }
  for (int j = 0; j < C::kC; ++j) cd[j] = D::var(c[j], 2 * C::kN + j);
  SmPrm<D> Pd;
  Pd.a = D::var(P.a, 2 * C::kN + C::kC);
  Pd.Q = D::var(P.Q, 2 * C::kN + C::kC + 1);
  Pd.L = D::var(P.L, 2 * C::kN + C::kC + 2);
  const D hd = D::var(ev.h, NE - 1);
  sm_rhs<C>(M, Pd, yp, cd, fp, &fpp);
  sm_rhs<C>(M, Pd, y, cd, fN, &fNp);
  const int e = C::kEq;
  // implicit crossing parameter
  D q = sm_hermite_h(yp[e], y[e], fp[e], fN[e], hd, D(ev.alpha)) - C::kEqTarget;
  const double dqda = sm_hermite_da(yp[e].v, y[e].v, fp[e].v, fN[e].v, ev.h, ev.alpha);
  D al(ev.alpha);
  for (int k = 0; k < NE; ++k) al.d[k] = -q.d[k] / dqda;
  D r, pph;
  if (C::kN == 6) {
    D yh[C::kN];
    for (int i = 0; i < C::kN; ++i) yh[i] = sm_hermite_h(yp[i], y[i], fp[i], fN[i], hd, al);
    r = C::radius(Pd.a, yh);
    pph = yh[0] * yh[4] - yh[1] * yh[3];
  } else {
    r = sm_hermite_h(yp[0], y[0], fp[0], fN[0], hd, al);
    pph = cd[C::kC - 1];
  }
  D red;
  const bool has = sm_redshift<D>(M, Pd, r, cd[0], pph, &red) && ev.deriv;
  double s[NE];
  for (int k = 0; k < NE; ++k) s[k] = rbar * r.d[k] + (has ? gbar * red.d[k] : 0.0);
  for (int i = 0; i < C::kN; ++i) {
    ybp[i] = s[i];
    ybN[i] = s[C::kN + i];
  }
  for (int j = 0; j < C::kC; ++j) cbar[j] = cbar[j] + s[2 * C::kN + j];
  for (int q2 = 0; q2 < kSmPrm; ++q2) pbar[q2] = pbar[q2] + s[2 * C::kN + C::kC + q2];
  *hbar = s[NE - 1];
}

// Scratch of one ray's adjoint (per thread, local memory).
struct SmScratch {
  SmCk ck1[kSmCkCap];
  SmCk ck2[kSmCkCap];
  SmSt st[kSmCkSteps];
};

// Reverse sweep of a ray traced with recording (N accepted steps, the last
// one ending in the disk event `ev`, checkpoints every k1 steps in
// sc->ck1).  Returns the cotangents of the initial state, the constants
// and (a, Q, Lambda).  The initial dlam is a constant (step_init).
template <class C>
KT_HD void sm_adjoint(const Frame& f, const SmPrm<double>& P, const double* c, const SmEvent& ev,
                      int N, int k1, double gbar, double rbar, SmScratch* sc, double* ybar,
                      double* cbar, double* pbar) {
  const double M = f.g.M;
  double ybN[C::kN], yb_direct[C::kN], hbar_ev = 0.0;
  for (int j = 0; j < C::kC; ++j) cbar[j] = 0.0;
  for (int q = 0; q < kSmPrm; ++q) pbar[q] = 0.0;
  sm_event_bwd<C>(M, P, c, ev, gbar, rbar, yb_direct, ybN, cbar, pbar, &hbar_ev);
  // The walk starts at step N-1 with the cotangent of y_N (H_N unused); the
  // direct seed of y_{N-1} joins after that step.
  for (int i = 0; i < C::kN; ++i) ybar[i] = ybN[i];
  double Hbar = 0.0;
  bool last = true;
  const int nseg = (N + k1 - 1) / k1;
  KT_ROLLED
  for (int sgi = nseg - 1; sgi >= 0; --sgi) {
    const int s0 = sgi * k1;
    const int len = (N - s0 < k1) ? N - s0 : k1;
    const int nsub = (len + kSmCkSteps - 1) / kSmCkSteps;
    if (nsub > 1) sm_replay<C>(f, P, c, sc->ck1[sgi], len, nullptr, sc->ck2, kSmCkSteps);
    KT_ROLLED
    for (int sub = nsub - 1; sub >= 0; --sub) {
      const int t0 = sub * kSmCkSteps;
      const int tl = (len - t0 < kSmCkSteps) ? len - t0 : kSmCkSteps;
      sm_replay<C>(f, P, c, nsub > 1 ? sc->ck2[sub] : sc->ck1[sgi], tl, sc->st, nullptr, 0);
      KT_ROLLED
      for (int m = tl - 1; m >= 0; --m) {
        sm_step_bwd<C>(f, P, c, sc->st[m], last ? hbar_ev : 0.0, ybar, &Hbar, cbar, pbar);
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
  int mode;  // 0: forward only; 1: arrays g, r; 2: L2 loss against a target frame
  const double* g;
  const double* r;
  const uint8_t* t_out;
  const double* t_g;
  const double* t_r;
  double w_g, w_r;
};

// A launch of the smooth kernel with gradients: cotangent source, chart
// override (trace every ray in the BL chart) and the [kGSlots][n] output.
struct SmJob {
  SmCot cot;
  int force_bl;
  double* contrib;
};

// Gradient slots of one pixel (and of the frame after the sum): dL/d(a, Q,
// Lambda, theta_obs [rad], r_obs), the loss, and counts: pixels whose
// reverse sweep ran, pixels traced in the BL chart, disk hits with a
// cotangent but more than 131072 steps (no gradient).
enum : int {
  kGA = 0, kGQ = 1, kGLambda = 2, kGTheta = 3, kGRobs = 4, kGLoss = 5, kGNumGrad = 6, kGNumBL = 7,
  kGNumUnrecorded = 8, kGSlots = 9
};

// One pixel of the smooth tracer: outputs into *o; with a cotangent source,
// the pixel's loss and gradient into g[kGSlots] (theta in radians).
template <bool kGrad>
KT_HD void sm_pixel(const Frame& f, uint32_t pix, bool force_bl, const SmCot& cot, RayResult* o,
                    double* g, SmScratch* sc) {
  const int px = (int)(pix % (uint32_t)f.cam.W), py = (int)(pix / (uint32_t)f.cam.W);
  double al, be;
  pixel_angles(f.cam, px, py, &al, &be);
  const double M = f.g.M;
  const SmPrm<double> P = sm_prm<double>(f.g);
  double ybl[4], cbl[2];
  sm_camera<double>(M, P, f.cam.r_obs, f.cam.theta_obs, al, be, ybl, cbl);
  bool ks = (f.chart == 0) && !force_bl;
  double yks[6], cks[1];
  if (ks) ks = sm_bl_to_ks<double>(M, P, ybl, cbl, f.cam.phi_obs, yks, cks);
  SmEvent ev;
  int k1 = 0, nck = 0;
  SmCk* ck = kGrad ? sc->ck1 : nullptr;
  const int N = ks ? sm_trace<ChartKS>(f, P, yks, cks, 0.0, o, &ev, ck, &k1, &nck)
                   : sm_trace<ChartBL>(f, P, ybl, cbl, f.cam.phi_obs, o, &ev, ck, &k1, &nck);
  if (!kGrad) return;
  for (int q = 0; q < kGSlots; ++q) g[q] = 0.0;
  g[kGNumBL] = ks ? 0.0 : 1.0;
  if (o->outcome != kOutDisk) return;
  double gbar = 0.0, rbar = 0.0;
  if (cot.mode == 1) {
    gbar = cot.g ? cot.g[pix] : 0.0;
    rbar = cot.r ? cot.r[pix] : 0.0;
  } else if (cot.mode == 2) {
    if (cot.t_out[pix] != kOutDisk) return;
    const double dg = o->red - cot.t_g[pix], dr = o->r - cot.t_r[pix];
    g[kGLoss] = cot.w_g * dg * dg + cot.w_r * dr * dr;
    gbar = 2.0 * cot.w_g * dg;
    rbar = 2.0 * cot.w_r * dr;
  }
  if (gbar == 0.0 && rbar == 0.0) return;
  if (N == 0) {
    g[kGNumUnrecorded] = 1.0;
    return;
  }
  g[kGNumGrad] = 1.0;
  double ybar[kSmMaxN], cbar[2], pbar[kSmPrm];
  typedef Dual<5> D5;
  SmPrm<D5> Pd;
  Pd.a = D5::var(P.a, 0);
  Pd.Q = D5::var(P.Q, 1);
  Pd.L = D5::var(P.L, 2);
  const D5 thd = D5::var(f.cam.theta_obs, 3), rd = D5::var(f.cam.r_obs, 4);
  D5 yb5[4], cb5[2];
  sm_camera<D5>(M, Pd, rd, thd, al, be, yb5, cb5);
  double gi[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (ks) {
    sm_adjoint<ChartKS>(f, P, cks, ev, N, k1, gbar, rbar, sc, ybar, cbar, pbar);
    D5 y5[6], c5[1];
    sm_bl_to_ks<D5>(M, Pd, yb5, cb5, f.cam.phi_obs, y5, c5);
    for (int k = 0; k < 5; ++k) {
      double s = cbar[0] * c5[0].d[k];
      for (int i = 0; i < 6; ++i) s = s + ybar[i] * y5[i].d[k];
      gi[k] = s;
    }
  } else {
    sm_adjoint<ChartBL>(f, P, cbl, ev, N, k1, gbar, rbar, sc, ybar, cbar, pbar);
    for (int k = 0; k < 5; ++k) {
      double s = cbar[0] * cb5[0].d[k] + cbar[1] * cb5[1].d[k];
      for (int i = 0; i < 4; ++i) s = s + ybar[i] * yb5[i].d[k];
      gi[k] = s;
    }
  }
  for (int q = 0; q < kSmPrm; ++q) gi[q] = gi[q] + pbar[q];
  g[kGA] = gi[0];
  g[kGQ] = gi[1];
  g[kGLambda] = gi[2];
  g[kGTheta] = gi[3];
  g[kGRobs] = gi[4];
}

}  // namespace kt
