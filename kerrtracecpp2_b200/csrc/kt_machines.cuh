// kt_machines.cuh -- per-ray integrators as "one RHS per slot" machines.
//
// An adaptive attempt is a fixed sequence of kSlots right-hand-side
// evaluations (slots 0..kSlots-1).  input(slot) gives the point at which the
// slot's RHS is needed, consume(slot) takes the RHS there and does the
// bookkeeping (stage sums; after the last slot: error control,
// accept/reject, events, termination).  Slot -1 is an extra RHS a ray needs
// only sometimes: f(s) of a new ray, and for step doubling f at the end of
// an accepted step (the next attempt's first stage and the event test).
// The persistent kernel runs all lanes of a warp through the same slot
// sequence together, so the bookkeeping after each slot executes converged
// and the kernel holds a single copy of the RHS; rays that finished are
// replaced at the next attempt boundary.
//
// Arithmetic and control flow follow the reference renderer:
//   BL  RK4 step doubling : trace_single + rk4_adaptive (main.cpp:343-434,
//                           geodesic.hpp:169-257)
//   BL  DOPRI5            : trace_single + dopri5_adaptive (geodesic.hpp:284-414)
//   KS  RK4 step doubling : trace_single_ks (main.cpp:1456-1660)
//   BL  Jacobi bundle     : trace_bundle (ray_bundle.hpp:137-436)
// The reference evaluates f(s0) twice per step-doubling attempt and f at
// both ends of an accepted step for the event test; these are the same
// inputs, so the machines evaluate each once and reuse it (bit-identical).
#pragma once

#include "kt_physics.cuh"

namespace kt {

enum : int { kOutEscaped = 0, kOutDisk = 1, kOutHorizon = 2 };
enum : int { kStEvent = 0, kStStepCap = 1, kStRejectCap = 2, kStNonfinite = 3, kStCreep = 4 };
enum : int { kEvNone = 0, kEvDisk = 1, kEvHorizon = 2, kEvEscape = 3 };

struct Frame {
  Metric g;
  CamConst cam;
  Ang eq;  // bl_ang at theta = pi/2 (disk redshift)
  double r_in, r_out, r_esc, rh_cut;
  double dlam0, tol;
  double bundle_eps;
  double r_fp32;     // mixed precision: FP32 RHS beyond this radius (inf: never)
  double turn_frac;  // mixed precision: FP64 when |p_r| or |p_th|/r < turn_frac |p_t|
  double r_doom;     // bundles: a ray creeping ingoing below r_doom, or (mixed and
  double r_cdoom;    // smooth) outgoing beyond r_cdoom, ends as a horizon hit (+-inf: never)
  int max_steps;
  int chart, intg, bundles;
  int precision;     // KT_PREC_FP64 / KT_PREC_MIXED
  int solver;        // effective KT_SOLVER_STANDARD / KT_SOLVER_SEMI_ANALYTIC
};

struct RayResult {
  double r, red, magnif, phi_disk, th_esc, ph_esc;
  uint32_t steps, attempts;
  int outcome, status;
};

KT_HD void set_result(RayResult* o, int outcome, int status, double r, double red, double magnif,
                      double phi_disk, double th_esc, double ph_esc) {
  o->outcome = outcome;
  o->status = status;
  o->r = r;
  o->red = red;
  o->magnif = magnif;
  o->phi_disk = phi_disk;
  o->th_esc = th_esc;
  o->ph_esc = ph_esc;
}

// Step-size update shared by the step-doubling controllers (geodesic.hpp:226-256,
// main.cpp:1507-1527, ray_bundle.hpp:235-262): returns 1 accepted, 0
// rejected, -1 non-finite error.
KT_HD int doubling_update(double err, double tol, double* dlam) {
  if (!finite(err)) {
    *dlam = (finite(*dlam) && *dlam > 1e-10) ? *dlam * 0.5 : 1e-6;
    if (*dlam < 1e-10) *dlam = 1e-10;
    return -1;
  }
  const int accepted = (err < tol || *dlam < 1e-10);
  if (accepted) {
    const double scale = (err > 1e-14) ? 0.9 * ktm_pow(tol / err, 0.2) : 4.0;
    double hnew = *dlam * scale;
    if (!finite(hnew)) hnew = *dlam;
    *dlam = hnew;
    if (*dlam > 100.0) *dlam = 100.0;
    if (*dlam < 1e-10) *dlam = 1e-10;
  } else {
    const double half = *dlam * 0.5;
    double hnew = (*dlam * 0.9) * ktm_pow(tol / err, 0.25);
    if (!finite(hnew)) hnew = half;
    *dlam = hnew;
    if (*dlam > half) *dlam = half;
    if (*dlam < 1e-10) *dlam = 1e-10;
  }
  return accepted;
}

// After a rejected attempt: the reference's `!isfinite(dlam) || ++rejects > 64`.
KT_HD bool reject_cap(double h, int* rejects, int* status) {
  if (!finite(h)) {
    *status = kStNonfinite;
    return true;
  }
  if (++*rejects > 64) {
    *status = kStRejectCap;
    return true;
  }
  return false;
}

// Horizon and escape tests of one accepted step (main.cpp:398-418); updates
// best_alpha / ev when the crossing comes first.
KT_HD void horizon_escape(double r_prev, double r_now, double rh_cut, double r_esc,
                          double* best_alpha, int* ev) {
  if (r_now <= rh_cut) {
    const double denom_h = r_prev - r_now;
    double alpha_h = (fabs(denom_h) > 1e-12) ? ((r_prev - rh_cut) / denom_h) : 0.0;
    alpha_h = dclamp(alpha_h, 0.0, 1.0);
    if (alpha_h < *best_alpha) {
      *best_alpha = alpha_h;
      *ev = kEvHorizon;
    }
  }
  if (r_now >= r_esc) {
    const double denom_e = r_now - r_prev;
    double alpha_e = (fabs(denom_e) > 1e-12) ? ((r_esc - r_prev) / denom_e) : 1.0;
    alpha_e = dclamp(alpha_e, 0.0, 1.0);
    if (alpha_e < *best_alpha) {
      *best_alpha = alpha_e;
      *ev = kEvEscape;
    }
  }
}

// ------------------------------------------------------- BL, single ray
// Shared state of the BL single-ray machines.
struct BLBase {
  double r, th, ph, pr, pth, pt, pphi;  // GeodesicState
  double h;                             // dlam
  double step_used;
  int it, rejects;
  uint32_t attempts;
  bool need_k1;

  KT_HD void init_state(const Frame& f, const Geo& s) {
    r = s.r;
    th = s.th;
    ph = s.ph;
    pr = s.pr;
    pth = s.pth;
    pt = s.pt;
    pphi = s.pphi;
    h = f.dlam0;
    step_used = h;
    it = 0;
    rejects = 0;
    attempts = 0;
    need_k1 = true;
  }

  KT_HD bool needs_k1() const { return need_k1; }

  // Events of trace_single (main.cpp:364-433) for the accepted step
  // (sp_*) -> (current state), with f at both ends (k0_*, k1_*: dr and
  // dtheta).  Returns true when the ray stops.
  KT_HD bool events(const Frame& f, double sp_r, double sp_th, double sp_ph, double k0_r,
                    double k0_th, double k1_r, double k1_th, RayResult* o) {
    double best_alpha = 2.0;
    int ev = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    const double q0 = sp_th - kHalfPi;
    const double q1 = th - kHalfPi;
    if (sign_change(q0, q1) || (dmin(fabs(q0), fabs(q1)) < 0.35)) {
      double alpha = 0.0;
      if (first_event(sp_th, th, k0_th, k1_th, step_used, kHalfPi, &alpha)) {
        const double r_hit = hermite(sp_r, r, k0_r, k1_r, step_used, alpha);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          disk_r = r_hit;
          disk_red = dclamp(disk_redshift(f.g, f.eq, r_hit, pt, pphi), 0.0, 20.0);
          disk_phi = sp_ph + alpha * (ph - sp_ph);
          best_alpha = alpha;
          ev = kEvDisk;
        }
      }
    }
    horizon_escape(sp_r, r, f.rh_cut, f.r_esc, &best_alpha, &ev);
    if (ev == kEvNone) return false;
    o->steps = (uint32_t)it + 1;
    o->attempts = attempts;
    if (ev == kEvDisk) {
      set_result(o, kOutDisk, kStEvent, disk_r, disk_red, 1.0, disk_phi, 0.0, 0.0);
    } else if (ev == kEvHorizon) {
      set_result(o, kOutHorizon, kStEvent, sp_r + best_alpha * (r - sp_r), 0.0, 1.0, 0.0, 0.0, 0.0);
    } else {
      const double th_esc = sp_th + best_alpha * (th - sp_th);
      const double ph_esc = sp_ph + best_alpha * (ph - sp_ph);
      // TraceResult{ESCAPED, r_escape, 1.0, th_esc, ph_esc}: theta lands in
      // the phi_disk slot and phi in theta_esc (main.cpp:430-432).
      set_result(o, kOutEscaped, kStEvent, f.r_esc, 1.0, 1.0, th_esc, ph_esc, 0.0);
    }
    return true;
  }

  // {ESCAPED, s.r, 1.0, s.theta, s.phi} (main.cpp:359-360, 433).
  KT_HD void stop_here(int status, uint32_t steps, RayResult* o) {
    o->steps = steps;
    o->attempts = attempts;
    set_result(o, kOutEscaped, status, r, 1.0, 1.0, th, ph, 0.0);
  }

  // After an accepted step without event: next step or the step cap.
  KT_HD bool next_step(const Frame& f, RayResult* o) {
    ++it;
    rejects = 0;
    if (it >= f.max_steps) {
      stop_here(kStStepCap, (uint32_t)it, o);
      return true;
    }
    return false;
  }
};

// Stage coefficient and base of step-doubling slots 0..9 (h = step,
// hb = h/2): path A (0-2) = one step h from s, path B1 (3-5) = half step
// from s, path B2 (6-9) = half step from B1 (slot 6 is its first stage).
// Returns the multiplier c of the previous stage's k in y = base + c k.
KT_HD double doubling_coeff(int slot, double h) {
  const double hb = 0.5 * h;
  if (slot < 3) return (slot == 2) ? h : 0.5 * h;
  if (slot < 6) return (slot == 5) ? hb : 0.5 * hb;
  return (slot == 9) ? hb : 0.5 * hb;
}

// RK4 step doubling (rk4_adaptive, geodesic.hpp:204-257), kSlots = 10.
struct BLRk4 : BLBase {
  static constexpr int kSlots = 10;
  double k1[5];  // f(s) = {dr, dth, dpr, dpth, dphi}
  double sum[5];
  double kp[4];
  double A[4];   // path A result (r, th, pr, pth); after acceptance: s_prev
  double B1[5];  // r, th, ph, pr, pth
  double sp_ph;
  bool pending;  // accepted step waiting for f(s_new) and its events

  KT_HD void init(const Frame& f, const Geo& s) {
    init_state(f, s);
    pending = false;
  }

  KT_HD void input(int slot, double y[4]) const {
    if (slot < 0) {
      y[0] = r; y[1] = th; y[2] = pr; y[3] = pth;
      return;
    }
    if (slot == 6) {
      y[0] = B1[0]; y[1] = B1[1]; y[2] = B1[3]; y[3] = B1[4];
      return;
    }
    const double c = doubling_coeff(slot, h);
    const bool on_s = slot < 6;
    const bool use_k1 = (slot == 0 || slot == 3);
    y[0] = (on_s ? r : B1[0]) + c * (use_k1 ? k1[0] : kp[0]);
    y[1] = (on_s ? th : B1[1]) + c * (use_k1 ? k1[1] : kp[1]);
    y[2] = (on_s ? pr : B1[3]) + c * (use_k1 ? k1[2] : kp[2]);
    y[3] = (on_s ? pth : B1[4]) + c * (use_k1 ? k1[3] : kp[3]);
  }

  // Returns true when the ray is finished (o filled).
  KT_HD bool consume(const Frame& f, int slot, const double k[5], RayResult* o) {
    if (slot < 0) {
      for (int i = 0; i < 5; ++i) k1[i] = k[i];
      need_k1 = false;
      if (!pending) return false;
      pending = false;
      if (events(f, A[0], A[1], sp_ph, kp[0], kp[1], k1[0], k1[1], o)) return true;
      return next_step(f, o);
    }
    switch (slot) {
      case 0:
      case 3:
        for (int i = 0; i < 5; ++i) sum[i] = k1[i] + 2.0 * k[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        return false;
      case 1:
      case 4:
      case 7:
      case 8:
        for (int i = 0; i < 5; ++i) sum[i] = sum[i] + 2.0 * k[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        return false;
      case 6:
        for (int i = 0; i < 5; ++i) sum[i] = k[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        return false;
      case 2: {
        const double w = h / 6.0;
        A[0] = r + w * (sum[0] + k[0]);
        A[1] = th + w * (sum[1] + k[1]);
        A[2] = pr + w * (sum[2] + k[2]);
        A[3] = pth + w * (sum[3] + k[3]);
        return false;
      }
      case 5: {
        const double w = (0.5 * h) / 6.0;
        B1[0] = r + w * (sum[0] + k[0]);
        B1[1] = th + w * (sum[1] + k[1]);
        B1[2] = ph + w * (sum[4] + k[4]);
        B1[3] = pr + w * (sum[2] + k[2]);
        B1[4] = pth + w * (sum[3] + k[3]);
        return false;
      }
      default: {  // 9: path B2 done -> error control
        const double w = (0.5 * h) / 6.0;
        const double Br = B1[0] + w * (sum[0] + k[0]);
        const double Bth = B1[1] + w * (sum[1] + k[1]);
        const double Bph = B1[2] + w * (sum[4] + k[4]);
        const double Bpr = B1[3] + w * (sum[2] + k[2]);
        const double Bpth = B1[4] + w * (sum[3] + k[3]);
        const double e0 = A[0] - Br, e1 = A[1] - Bth, e2 = A[2] - Bpr, e3 = A[3] - Bpth;
        const double err = sqrt(((e0 * e0 + e1 * e1) + e2 * e2) + e3 * e3) / 15.0;
        step_used = h;
        ++attempts;
        const int acc = doubling_update(err, f.tol, &h);
        if (acc == 1) {
          A[0] = r;  // s_prev
          A[1] = th;
          sp_ph = ph;
          kp[0] = k1[0];  // f(s_prev): dr, dth
          kp[1] = k1[1];
          r = Br;
          th = Bth;
          ph = Bph;
          pr = Bpr;
          pth = Bpth;
          need_k1 = true;
          pending = true;
          return false;
        }
        int st;
        if (reject_cap(h, &rejects, &st)) {
          stop_here(st, (uint32_t)it, o);
          return true;
        }
        return false;
      }
    }
  }
};

// DOPRI5 (dopri5_adaptive, geodesic.hpp:284-414), kSlots = 6: slots 0..4
// -> k2..k6, slot 5 -> k7 = f(y5) then error control.  FSAL: after an
// accepted step k1 = k7, so only a new ray needs slot -1.  Phi is not
// advanced (the reference's `advance` updates r, theta, p_r, p_theta only).
struct BLDopri5 : BLBase {
  static constexpr int kSlots = 6;
  double kk[7][4];

  KT_HD void init(const Frame& f, const Geo& s) { init_state(f, s); }

  // advance (geodesic.hpp:300-310): y = s + sum_i (h w_i) k_i, in order.
  template <int N>
  KT_HD void adv(const double* w, double y[4]) const {
    y[0] = r; y[1] = th; y[2] = pr; y[3] = pth;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double hw = h * w[i];
      y[0] += hw * kk[i][0];
      y[1] += hw * kk[i][1];
      y[2] += hw * kk[i][2];
      y[3] += hw * kk[i][3];
    }
  }

  KT_HD void input(int slot, double y[4]) const {
    const double a2[1] = {1.0 / 5.0};
    const double a3[2] = {3.0 / 40.0, 9.0 / 40.0};
    const double a4[3] = {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0};
    const double a5[4] = {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0};
    const double a6[5] = {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0,
                          -5103.0 / 18656.0};
    const double b5[6] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0,
                          11.0 / 84.0};
    switch (slot) {
      case 0: adv<1>(a2, y); break;
      case 1: adv<2>(a3, y); break;
      case 2: adv<3>(a4, y); break;
      case 3: adv<4>(a5, y); break;
      case 4: adv<5>(a6, y); break;
      case 5: adv<6>(b5, y); break;
      default: y[0] = r; y[1] = th; y[2] = pr; y[3] = pth; break;
    }
  }

  KT_HD bool consume(const Frame& f, int slot, const double k[5], RayResult* o) {
    switch (slot) {  // constant indices keep kk in registers
      case -1:
        for (int i = 0; i < 4; ++i) kk[0][i] = k[i];
        need_k1 = false;
        return false;
      case 0: for (int i = 0; i < 4; ++i) kk[1][i] = k[i]; return false;
      case 1: for (int i = 0; i < 4; ++i) kk[2][i] = k[i]; return false;
      case 2: for (int i = 0; i < 4; ++i) kk[3][i] = k[i]; return false;
      case 3: for (int i = 0; i < 4; ++i) kk[4][i] = k[i]; return false;
      case 4: for (int i = 0; i < 4; ++i) kk[5][i] = k[i]; return false;
      default: break;
    }
    for (int i = 0; i < 4; ++i) kk[6][i] = k[i];
    const double b5[6] = {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0,
                          11.0 / 84.0};
    const double b4[7] = {5179.0 / 57600.0, 0.0, 7571.0 / 16695.0, 393.0 / 640.0,
                          -92097.0 / 339200.0, 187.0 / 2100.0, 1.0 / 40.0};
    double y5[4], y4[4];
    adv<6>(b5, y5);
    adv<7>(b4, y4);
    const double ref[4] = {r, th, pr, pth};
    double err2 = 0.0;
    for (int i = 0; i < 4; ++i) {
      const double ratio = (y5[i] - y4[i]) / (f.tol * (1.0 + fabs(ref[i])));
      err2 += ratio * ratio;
    }
    const double err = sqrt(err2 / 4.0);
    step_used = h;
    ++attempts;
    if (!finite(err)) {
      h = (finite(h) && h > 1e-10) ? h * 0.5 : 1e-6;
      if (h < 1e-10) h = 1e-10;
    } else if (err <= 1.0 || h < 1e-10) {
      const double fac = (err > 1e-12) ? 0.9 * ktm_pow(1.0 / err, 0.2) : 4.0;
      double hnew = h * fac;
      if (!finite(hnew)) hnew = h;
      if (hnew > 100.0) hnew = 100.0;
      if (hnew < 1e-10) hnew = 1e-10;
      h = hnew;
      const double sp_r = r, sp_th = th;
      const double k0_r = kk[0][0], k0_th = kk[0][1];
      r = y5[0];
      th = y5[1];
      pr = y5[2];
      pth = y5[3];
      for (int i = 0; i < 4; ++i) kk[0][i] = kk[6][i];  // FSAL
      if (events(f, sp_r, sp_th, ph, k0_r, k0_th, kk[0][0], kk[0][1], o)) return true;
      return next_step(f, o);
    } else {
      double hnew = (h * 0.9) * ktm_pow(1.0 / err, 0.25);
      if (!finite(hnew)) hnew = h * 0.5;
      h = dmax(hnew, 1e-10);
    }
    int st;
    if (reject_cap(h, &rejects, &st)) {
      stop_here(st, (uint32_t)it, o);
      return true;
    }
    return false;
  }
};

// ------------------------------------------------------------- KS chart
// trace_single_ks (main.cpp:1530-1660), RK4 step doubling in (X,Y,Z,p),
// kSlots = 10 as BLRk4.
struct KSRk4 {
  static constexpr int kSlots = 10;
  double s[6];   // X, Y, Z, pX, pY, pZ
  double pT;
  double h;
  double k1[6];
  double sum[6], kp[6];
  double A[6];   // path A; after acceptance: s_prev
  double B1[6];
  double step_used;
  double prev_r;  // r_KS at the start of the step
  int it, rejects;
  uint32_t attempts;
  bool need_k1, pending;

  // Returns false when init_ks_state fails: the reference then traces the
  // ray in the BL chart (main.cpp:1537-1538).
  KT_HD bool init(const Frame& f, const Geo& sb) {
    KSState k;
    if (!init_ks_state(f.g, sb, &k)) return false;
    s[0] = k.X; s[1] = k.Y; s[2] = k.Z; s[3] = k.pX; s[4] = k.pY; s[5] = k.pZ;
    pT = k.pT;
    h = f.dlam0;
    step_used = h;
    prev_r = r_ks(f.g, s[0], s[1], s[2]);
    it = 0;
    rejects = 0;
    attempts = 0;
    need_k1 = true;
    pending = false;
    return true;
  }

  KT_HD bool needs_k1() const { return need_k1; }

  KT_HD void input(int slot, double y[6]) const {
    if (slot < 0) {
      for (int i = 0; i < 6; ++i) y[i] = s[i];
      return;
    }
    if (slot == 6) {
      for (int i = 0; i < 6; ++i) y[i] = B1[i];
      return;
    }
    const double c = doubling_coeff(slot, h);
    const bool on_s = slot < 6;
    const bool use_k1 = (slot == 0 || slot == 3);
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] = (on_s ? s[i] : B1[i]) + c * (use_k1 ? k1[i] : kp[i]);
  }

  KT_HD void stop_at(const Frame& f, const double* x, int status, uint32_t steps, RayResult* o) {
    double rr, tt, pp;
    ks_to_bl(f.g, x[0], x[1], x[2], &rr, &tt, &pp);
    o->steps = steps;
    o->attempts = attempts;
    // TraceResult{ESCAPED, r, 1.0, th, ph}: slot quirk as in the BL tracer.
    set_result(o, kOutEscaped, status, rr, 1.0, 1.0, tt, pp, 0.0);
  }

  // Events of an accepted step (main.cpp:1570-1657); A = s_prev, kp = f(s_prev).
  KT_HD bool events(const Frame& f, RayResult* o) {
    const double* sp = A;
    const double* d0 = kp;
    const double r_now = r_ks(f.g, s[0], s[1], s[2]);
    double best_alpha = 2.0;
    int ev = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    if (sign_change(sp[2], s[2]) || (dmin(fabs(sp[2]), fabs(s[2])) < 0.35)) {
      double alpha = 0.0;
      bool hit = first_event(sp[2], s[2], d0[2], k1[2], step_used, 0.0, &alpha);
      if (!hit && sign_change(sp[2], s[2])) {
        const double denom = sp[2] - s[2];
        alpha = (fabs(denom) > 1e-12) ? (sp[2] / denom) : 0.5;
        alpha = dclamp(alpha, 0.0, 1.0);
        hit = true;
      }
      if (hit) {
        double xh[6];
        for (int i = 0; i < 6; ++i) xh[i] = hermite(sp[i], s[i], d0[i], k1[i], step_used, alpha);
        double r_hit, th_hit, ph_hit;
        ks_to_bl(f.g, xh[0], xh[1], xh[2], &r_hit, &th_hit, &ph_hit);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          const double pphi_bl = ks_pphi_bl(r_hit, th_hit, ph_hit, f.g.a, xh[3], xh[4], xh[5]);
          disk_r = r_hit;
          disk_red = dclamp(disk_redshift(f.g, f.eq, r_hit, pT, pphi_bl), 0.0, 20.0);
          disk_phi = ph_hit;
          best_alpha = alpha;
          ev = kEvDisk;
        }
      }
    }
    horizon_escape(prev_r, r_now, f.rh_cut, f.r_esc, &best_alpha, &ev);
    if (ev != kEvNone) {
      o->steps = (uint32_t)it + 1;
      o->attempts = attempts;
      if (ev == kEvDisk) {
        set_result(o, kOutDisk, kStEvent, disk_r, disk_red, 1.0, disk_phi, 0.0, 0.0);
      } else if (ev == kEvHorizon) {
        set_result(o, kOutHorizon, kStEvent, prev_r + best_alpha * (r_now - prev_r), 0.0, 1.0, 0.0,
                   0.0, 0.0);
      } else {
        double xe[3];
        for (int i = 0; i < 3; ++i) xe[i] = sp[i] + best_alpha * (s[i] - sp[i]);
        double re, te, pe;
        ks_to_bl(f.g, xe[0], xe[1], xe[2], &re, &te, &pe);
        set_result(o, kOutEscaped, kStEvent, re, 1.0, 1.0, te, pe, 0.0);
      }
      return true;
    }
    prev_r = r_now;
    ++it;
    rejects = 0;
    if (it >= f.max_steps) {
      stop_at(f, s, kStStepCap, (uint32_t)it, o);
      return true;
    }
    return false;
  }

  KT_HD bool consume(const Frame& f, int slot, const double k[6], RayResult* o) {
    if (slot < 0) {
      for (int i = 0; i < 6; ++i) k1[i] = k[i];
      need_k1 = false;
      if (!pending) return false;
      pending = false;
      return events(f, o);
    }
    switch (slot) {
      case 0:
      case 3:
        for (int i = 0; i < 6; ++i) {
          sum[i] = k1[i] + 2.0 * k[i];
          kp[i] = k[i];
        }
        return false;
      case 1:
      case 4:
      case 7:
      case 8:
        for (int i = 0; i < 6; ++i) {
          sum[i] = sum[i] + 2.0 * k[i];
          kp[i] = k[i];
        }
        return false;
      case 6:
        for (int i = 0; i < 6; ++i) {
          sum[i] = k[i];
          kp[i] = k[i];
        }
        return false;
      case 2: {
        const double w = h / 6.0;
        for (int i = 0; i < 6; ++i) A[i] = s[i] + w * (sum[i] + k[i]);
        return false;
      }
      case 5: {
        const double w = (0.5 * h) / 6.0;
        for (int i = 0; i < 6; ++i) B1[i] = s[i] + w * (sum[i] + k[i]);
        return false;
      }
      default: {  // 9
        const double w = (0.5 * h) / 6.0;
        double B[6];
        for (int i = 0; i < 6; ++i) B[i] = B1[i] + w * (sum[i] + k[i]);
        const double e0 = A[0] - B[0], e1 = A[1] - B[1], ez = A[2] - B[2];
        const double e3 = A[3] - B[3], e4 = A[4] - B[4], e5 = A[5] - B[5];
        const double err =
            sqrt(((((e0 * e0 + e1 * e1) + ez * ez) + e3 * e3) + e4 * e4) + e5 * e5) / 15.0;
        step_used = h;
        ++attempts;
        const int acc = doubling_update(err, f.tol, &h);
        if (acc == 1) {
          for (int i = 0; i < 6; ++i) {
            A[i] = s[i];    // s_prev
            kp[i] = k1[i];  // f(s_prev)
            s[i] = B[i];
          }
          need_k1 = true;
          pending = true;
          return false;
        }
        int st;
        if (reject_cap(h, &rejects, &st)) {
          stop_at(f, s, st, (uint32_t)it, o);
          return true;
        }
        return false;
      }
    }
  }
};

// ------------------------------------- mixed-precision constraint reprojection
// Hamiltonian-constraint reprojection (FP64) of the mixed-precision tracer.
// After an accepted step in the FP32 regime (the new point beyond r_fp32,
// which is infinite unless the tolerance lets the FP32 right-hand side run),
// the momenta the integrator evolves are scaled by the lambda that puts the
// point back on H = 0 -- BL: (p_r, p_theta), with p_t and p_phi constants of
// motion; KS: (p_X, p_Y, p_Z), with p_T -- when that correction is below
// 1e-4 (larger ones are not rounding drift).  Returns true when it scaled.
KT_HD_CALL bool bl_reproject(const Frame& f, double r, double th, double* pr, double* pth,
                             double pt, double pphi) {
  if (!(r > f.r_fp32)) return false;
  const Inv U = bl_inv_mx(f.g, r, th);
  const double kin = U.rr * (*pr) * (*pr) + U.hh * (*pth) * (*pth);
  const double pot = -((U.tt * pt * pt + 2.0 * U.tp * pt * pphi) + U.pp * pphi * pphi);
  if (!(kin > 0.0 && pot > 0.0)) return false;
  const double lam2 = pot / kin;
  if (!(fabs(lam2 - 1.0) < 2e-4)) return false;
  const double lam = sqrt(lam2);
  *pr *= lam;
  *pth *= lam;
  return true;
}

// KS: 2H(lambda) = -p_T^2 + lambda^2 |p|^2 - F (-p_T + lambda m)^2 with
// m = l_i p_i (the spatial part of l.p), i.e. A lambda^2 + B lambda + C = 0,
// A = |p|^2 - F m^2, B = 2 F p_T m, C = -p_T^2 (1 + F); the root nearer 1.
KT_HD_CALL bool ks_reproject(const Frame& f, double s[6], double pT) {
  const Metric& g = f.g;
  const double X = s[0], Y = s[1], Z = s[2];
  const double b = ((X * X + Y * Y) + Z * Z) - g.a2;
  const double r = sqrt(0.5 * (b + sqrt(b * b + 4.0 * g.a2 * Z * Z)));
  if (!(r > f.r_fp32)) return false;
  const double ir = mx_rcp(r), iD = mx_rcp(r * r + g.a2);
  const double rho2 = r * r + g.a2 * Z * Z * ir * ir;
  const double F = (g.twoM * r - g.Q2) * mx_rcp(rho2);
  const double m = ((r * X + g.a * Y) * s[3] + (r * Y - g.a * X) * s[4]) * iD + Z * s[5] * ir;
  const double P2 = (s[3] * s[3] + s[4] * s[4]) + s[5] * s[5];
  const double A = P2 - F * m * m, B = 2.0 * F * pT * m, C = -pT * pT * (1.0 + F);
  const double disc = B * B - 4.0 * A * C;
  if (!(A != 0.0 && disc >= 0.0)) return false;
  const double q = -0.5 * (B + copysign(sqrt(disc), B));  // roots q/A and C/q
  const double l1 = q / A, l2 = (q != 0.0) ? C / q : l1;
  const double lam = (fabs(l1 - 1.0) < fabs(l2 - 1.0)) ? l1 : l2;
  if (!(fabs(lam - 1.0) < 1e-4)) return false;
  s[3] *= lam;
  s[4] *= lam;
  s[5] *= lam;
  return true;
}

// The mixed tracer's step hook: after consume(slot) returned false, with
// `it0` the step count before it.  RK4 doubling accepts at slot 9 and then
// evaluates f at the new point (slot -1), which sees the scaled momenta;
// DOPRI5 accepts at slot 5 and carries f(y5) over (FSAL), so a scaled point
// has f evaluated again.
KT_HD void mixed_after_slot(const Frame& f, BLRk4* m, int slot, int) {
  if (slot == 9 && m->pending) bl_reproject(f, m->r, m->th, &m->pr, &m->pth, m->pt, m->pphi);
}
KT_HD void mixed_after_slot(const Frame& f, BLDopri5* m, int slot, int it0) {
  if (slot == 5 && m->it != it0 &&
      bl_reproject(f, m->r, m->th, &m->pr, &m->pth, m->pt, m->pphi))
    m->need_k1 = true;
}
KT_HD void mixed_after_slot(const Frame& f, KSRk4* m, int slot, int) {
  if (slot == 9 && m->pending) ks_reproject(f, m->s, m->pT);
}

// ---------------------------------------------------- BL Jacobi bundle
// trace_bundle (ray_bundle.hpp:301-436): RK4 step doubling of the geodesic
// and the 4x2 deviation matrix W; error control on the geodesic only.
struct Bundle {
  static constexpr int kSlots = 10;
  double r, th, ph, pr, pth, pt, pphi;
  double W[8];
  double h;
  double k1[5], kW1[8];  // f(s, W)
  double sum[5], sumW[8], kp[4], kpW[8];
  double A[4];            // path A geodesic; after acceptance: s_prev (r, th)
  double B1[5], B1W[8];
  double Wprev[8];
  double step_used, sp_ph;
  int it, rejects;
  uint32_t attempts;
  bool need_k1, pending;

  KT_HD void init(const Frame& f, int px, int py) {
    double al, be;
    pixel_angles(f.cam, px, py, &al, &be);
    const Geo s = angle_ray(f.cam, al, be);
    r = s.r; th = s.th; ph = s.ph; pr = s.pr; pth = s.pth; pt = s.pt; pphi = s.pphi;
    // init_bundle (ray_bundle.hpp:278-298)
    const double eps = f.bundle_eps;
    const Geo ap = angle_ray(f.cam, al + eps, be);
    const Geo am = angle_ray(f.cam, al - eps, be);
    const Geo bp = angle_ray(f.cam, al, be + eps);
    const Geo bm = angle_ray(f.cam, al, be - eps);
    W[0] = (ap.r - am.r) / (2.0 * eps);
    W[2] = (ap.th - am.th) / (2.0 * eps);
    W[4] = (ap.pr - am.pr) / (2.0 * eps);
    W[6] = (ap.pth - am.pth) / (2.0 * eps);
    W[1] = (bp.r - bm.r) / (2.0 * eps);
    W[3] = (bp.th - bm.th) / (2.0 * eps);
    W[5] = (bp.pr - bm.pr) / (2.0 * eps);
    W[7] = (bp.pth - bm.pth) / (2.0 * eps);
    h = f.dlam0;
    step_used = h;
    it = 0;
    rejects = 0;
    attempts = 0;
    need_k1 = true;
    pending = false;
  }

  KT_HD bool needs_k1() const { return need_k1; }

  // point (geodesic y[4] and W yW[8]) of the slot's bundle RHS
  KT_HD void input(int slot, double y[4], double yW[8]) const {
    if (slot < 0) {
      y[0] = r; y[1] = th; y[2] = pr; y[3] = pth;
#pragma unroll
      for (int i = 0; i < 8; ++i) yW[i] = W[i];
      return;
    }
    if (slot == 6) {
      y[0] = B1[0]; y[1] = B1[1]; y[2] = B1[3]; y[3] = B1[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) yW[i] = B1W[i];
      return;
    }
    const double c = doubling_coeff(slot, h);
    const bool on_s = slot < 6;
    const bool use_k1 = (slot == 0 || slot == 3);
    y[0] = (on_s ? r : B1[0]) + c * (use_k1 ? k1[0] : kp[0]);
    y[1] = (on_s ? th : B1[1]) + c * (use_k1 ? k1[1] : kp[1]);
    y[2] = (on_s ? pr : B1[3]) + c * (use_k1 ? k1[2] : kp[2]);
    y[3] = (on_s ? pth : B1[4]) + c * (use_k1 ? k1[3] : kp[3]);
#pragma unroll
    for (int i = 0; i < 8; ++i) yW[i] = (on_s ? W[i] : B1W[i]) + c * (use_k1 ? kW1[i] : kpW[i]);
  }

  // Events of an accepted bundle step (ray_bundle.hpp:337-434).
  KT_HD bool events(const Frame& f, RayResult* o) {
    const double sp_r = A[0], sp_th = A[1];
    double best_alpha = 2.0;
    int ev = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_det = 1.0, disk_phi = 0.0;
    bool skip = false;
    const double q0 = sp_th - kHalfPi;
    const double q1 = th - kHalfPi;
    if (sign_change(q0, q1) || (dmin(fabs(q0), fabs(q1)) < 0.35)) {
      double alpha = 0.0;
      if (!first_event(sp_th, th, kp[1], k1[1], step_used, kHalfPi, &alpha)) {
        skip = true;  // ray_bundle.hpp:352-356 `continue`: no horizon/escape test this step
      } else {
        const double r_hit = hermite(sp_r, r, kp[0], k1[0], step_used, alpha);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          const double J00 = Wprev[0] + alpha * (W[0] - Wprev[0]);
          const double J01 = Wprev[1] + alpha * (W[1] - Wprev[1]);
          const double J10 = Wprev[2] + alpha * (W[2] - Wprev[2]);
          const double J11 = Wprev[3] + alpha * (W[3] - Wprev[3]);
          double det = fabs(J00 * J11 - J01 * J10);
          det = det < 1e-12 ? 1e-12 : det;
          disk_r = r_hit;
          disk_red = bundle_redshift(f.g, f.eq, r_hit, pt, pphi);
          disk_det = det;
          disk_phi = sp_ph + alpha * (ph - sp_ph);
          best_alpha = alpha;
          ev = kEvDisk;
        }
      }
    }
    if (skip && ((r <= f.r_doom && k1[0] < 0.0) || (r >= f.r_cdoom && k1[0] > 0.0))) {
      // The step near the equator skipped the horizon and escape tests, and
      // the ray is ingoing within 1e-4 r_+ of the outer horizon (inside every
      // photon orbit, below the disk's inner edge and rh_cut), or (mixed
      // precision only) outgoing within 1e-4 r_c of the cosmological one: it
      // can only creep onto that horizon in BL coordinates, theta frozen,
      // until the controller gives up (the reference's reject cap, or its
      // step cap), or leave the band and meet the horizon test at once --
      // every ending gives the record BundleResult{} gives (trace_bundle,
      // ray_bundle.hpp:320, 418-435; the frame loop writes r = 0 for every
      // ray that misses the disk, main.cpp:2103-2110).  It ends here with
      // that record and status kStCreep; its counters stop here.
      o->steps = (uint32_t)it + 1;
      o->attempts = attempts;
      set_result(o, kOutEscaped, kStCreep, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
      return true;
    }
    if (!skip) {
      horizon_escape(sp_r, r, f.rh_cut, f.r_esc, &best_alpha, &ev);
      if (ev != kEvNone) {
        o->steps = (uint32_t)it + 1;
        o->attempts = attempts;
        if (ev == kEvDisk) {
          set_result(o, kOutDisk, kStEvent, disk_r, disk_red, disk_det, disk_phi, 0.0, 0.0);
        } else if (ev == kEvHorizon) {
          // BundleResult{}: the pixel reads as escaped toward (0, 0)
          set_result(o, kOutEscaped, kStEvent, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
        } else {
          const double th_esc = sp_th + best_alpha * (th - sp_th);
          const double ph_esc = sp_ph + best_alpha * (ph - sp_ph);
          set_result(o, kOutEscaped, kStEvent, 0.0, 1.0, 1.0, 0.0, th_esc, ph_esc);
        }
        return true;
      }
    }
    ++it;
    rejects = 0;
    if (it >= f.max_steps) {
      o->steps = (uint32_t)it;
      o->attempts = attempts;
      set_result(o, kOutEscaped, kStStepCap, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
      return true;
    }
    return false;
  }

  KT_HD bool consume(const Frame& f, int slot, const double k[5], const double kW[8],
                     RayResult* o) {
    if (slot < 0) {
      for (int i = 0; i < 5; ++i) k1[i] = k[i];
      for (int i = 0; i < 8; ++i) kW1[i] = kW[i];
      need_k1 = false;
      if (!pending) return false;
      pending = false;
      return events(f, o);
    }
    switch (slot) {
      case 0:
      case 3:
        for (int i = 0; i < 5; ++i) sum[i] = k1[i] + 2.0 * k[i];
        for (int i = 0; i < 8; ++i) sumW[i] = kW1[i] + 2.0 * kW[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        for (int i = 0; i < 8; ++i) kpW[i] = kW[i];
        return false;
      case 1:
      case 4:
      case 7:
      case 8:
        for (int i = 0; i < 5; ++i) sum[i] = sum[i] + 2.0 * k[i];
        for (int i = 0; i < 8; ++i) sumW[i] = sumW[i] + 2.0 * kW[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        for (int i = 0; i < 8; ++i) kpW[i] = kW[i];
        return false;
      case 6:
        for (int i = 0; i < 5; ++i) sum[i] = k[i];
        for (int i = 0; i < 8; ++i) sumW[i] = kW[i];
        for (int i = 0; i < 4; ++i) kp[i] = k[i];
        for (int i = 0; i < 8; ++i) kpW[i] = kW[i];
        return false;
      case 2: {
        const double w = h / 6.0;
        A[0] = r + w * (sum[0] + k[0]);
        A[1] = th + w * (sum[1] + k[1]);
        A[2] = pr + w * (sum[2] + k[2]);
        A[3] = pth + w * (sum[3] + k[3]);
        return false;
      }
      case 5: {
        const double w = (0.5 * h) / 6.0;
        B1[0] = r + w * (sum[0] + k[0]);
        B1[1] = th + w * (sum[1] + k[1]);
        B1[2] = ph + w * (sum[4] + k[4]);
        B1[3] = pr + w * (sum[2] + k[2]);
        B1[4] = pth + w * (sum[3] + k[3]);
        for (int i = 0; i < 8; ++i) B1W[i] = W[i] + w * (sumW[i] + kW[i]);
        return false;
      }
      default: {  // 9
        const double w = (0.5 * h) / 6.0;
        const double Br = B1[0] + w * (sum[0] + k[0]);
        const double Bth = B1[1] + w * (sum[1] + k[1]);
        const double Bph = B1[2] + w * (sum[4] + k[4]);
        const double Bpr = B1[3] + w * (sum[2] + k[2]);
        const double Bpth = B1[4] + w * (sum[3] + k[3]);
        const double e0 = A[0] - Br, e1 = A[1] - Bth, e2 = A[2] - Bpr, e3 = A[3] - Bpth;
        const double err = sqrt(((e0 * e0 + e1 * e1) + e2 * e2) + e3 * e3) / 15.0;
        step_used = h;
        ++attempts;
        const int acc = doubling_update(err, f.tol, &h);
        if (acc == 1) {
          A[0] = r;
          A[1] = th;
          sp_ph = ph;
          kp[0] = k1[0];
          kp[1] = k1[1];
          for (int i = 0; i < 8; ++i) {
            Wprev[i] = W[i];
            W[i] = B1W[i] + w * (sumW[i] + kW[i]);
          }
          r = Br;
          th = Bth;
          ph = Bph;
          pr = Bpr;
          pth = Bpth;
          need_k1 = true;
          pending = true;
          return false;
        }
        int st;
        if (reject_cap(h, &rejects, &st)) {
          // trace_bundle returns BundleResult{} (ray_bundle.hpp:320)
          o->steps = (uint32_t)it;
          o->attempts = attempts;
          set_result(o, kOutEscaped, st, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
          return true;
        }
        return false;
      }
    }
  }
};

// -------------------------------------------------- separable Kerr (BL)
// The semi-analytic solver, trace_single_separable_kerr with
// rk4_adaptive_separable_kerr and rk4_step_separable_kerr (main.cpp:506-703):
// RK4 step doubling on (r, theta, phi) with the separated right-hand side
// (sep_rhs), kSlots = 10 as in BLRk4 (f(s) shared by both paths, f at the
// end of an accepted step shared by the events and the next attempt).  A
// stage whose right-hand side or end state is not finite fails the attempt
// (h halved).  The ray gives up -- and is traced again from the camera by
// the standard BL tracer with RK4 step doubling -- when the constants of
// motion cannot be formed, after 65 rejected attempts of one step, on a
// non-finite step size, or when f at the end of a step near the equator
// is not finite; `fallback` is then set.
struct SepRk4 {
  static constexpr int kSlots = 10;
  SepConst c;
  double pt, pphi;   // camera covector (disk redshift)
  double r, th, ph;  // SeparableState
  double h, step_used;
  double k1[3];      // f(s) = {dr, dth, dph}
  double kp[3];      // previous stage; after acceptance f(s_prev) (dr, dth)
  double sum[3];
  double A[3];       // path A result; after acceptance s_prev
  double B1[3];
  double prevR, prevT;  // R, Theta at the start of the step
  double Rn, Tn;        // ... at its end
  double kin[2];        // (r, theta) at which k1 was evaluated
  int kin_sr, kin_sth;  // ... and the branch signs
  int sr, sth;
  int it, rejects;
  uint32_t attempts;
  uint32_t fb_key, out_slot;
  bool need_k1, pending, k1_ok, fail, fallback;

  KT_HD bool needs_k1() const { return need_k1; }

  // false: the constants cannot be formed (init_separable_consts).
  KT_HD bool init(const Frame& f, const Geo& s, uint32_t key, uint32_t slot) {
    fb_key = key;
    out_slot = slot;
    fallback = false;
    if (!sep_init(f.g, s.th, s.pth, s.pt, s.pphi, &c)) return false;
    // branch signs from the BL velocities dr = g^rr p_r, dth = g^thth p_th
    const Inv U = bl_inv(f.g, s.r, bl_ang(f.g, s.th));
    sr = (U.rr * s.pr >= 0.0) ? 1 : -1;
    sth = (U.hh * s.pth >= 0.0) ? 1 : -1;
    pt = s.pt;
    pphi = s.pphi;
    r = s.r;
    th = s.th;
    ph = s.ph;
    h = f.dlam0;
    step_used = h;
    prevR = sep_R(c, r);
    prevT = sep_Theta(c, th);
    kin[0] = kin[1] = ktm_nan();
    kin_sr = kin_sth = 0;
    it = 0;
    rejects = 0;
    attempts = 0;
    need_k1 = true;
    pending = false;
    return true;
  }

  KT_HD void input(int slot, double y[2]) const {
    if (slot < 0) {
      y[0] = r; y[1] = th;
      return;
    }
    if (slot == 6) {
      y[0] = B1[0]; y[1] = B1[1];
      return;
    }
    const double cf = doubling_coeff(slot, h);
    const bool on_s = slot < 6;
    const bool use_k1 = (slot == 0 || slot == 3);
    y[0] = (on_s ? r : B1[0]) + cf * (use_k1 ? k1[0] : kp[0]);
    y[1] = (on_s ? th : B1[1]) + cf * (use_k1 ? k1[1] : kp[1]);
  }

  // The right-hand side at the slot's input y (sep_rhs, a function of
  // (r, theta, sr, sth) alone).  When y and the signs are those of k1 it is
  // k1: a ray whose radial and polar velocities are both zero stays at that
  // point, every stage of its attempts has the same input, and only phi
  // advances -- the solver's rays with a radial turning point end that way
  // and run to the step cap.  (-0 == +0 here: sep_rhs gives the same
  // values for either zero.)
  KT_HD bool rhs(int slot, const double y[2], double k[3]) {
    if (y[0] == kin[0] && y[1] == kin[1] && sr == kin_sr && sth == kin_sth) {
      k[0] = k1[0];
      k[1] = k1[1];
      k[2] = k1[2];
      return k1_ok;
    }
    const bool ok = sep_rhs(c, y[0], y[1], sr, sth, k);
    if (slot < 0) {
      kin[0] = y[0];
      kin[1] = y[1];
      kin_sr = sr;
      kin_sth = sth;
    }
    return ok;
  }

  // After an accepted step without event: the next step or the step cap.
  KT_HD bool end_step(const Frame& f, RayResult* o) {
    ++it;
    rejects = 0;
    if (it >= f.max_steps) {
      o->steps = (uint32_t)it;
      o->attempts = attempts;
      set_result(o, kOutEscaped, kStStepCap, r, 1.0, 1.0, th, ph, 0.0);
      return true;
    }
    return false;
  }

  // At an attempt boundary: f(s) is finite with dr = dth = 0 (k1 belongs to
  // the current point, kin).  r + c * (+-0) = r and th + c * (+-0) = th for
  // r, th != 0, so every stage input of every later attempt is this point,
  // every right-hand side is k1, and only phi moves.
  KT_HD bool parked() const {
    return k1_ok && k1[0] == 0.0 && k1[1] == 0.0 && r != 0.0 && th != 0.0;
  }

  // Up to kParkedBudget attempts of a parked ray, each with the arithmetic
  // of slots 0..9 and -1 written out for stages that all return k1: the
  // stage sums of r and theta are +-0 (A, B1, B2 keep r and theta), those
  // of phi are ((c + 2c) + 2c) + c with c = k1[2]; the step ends where it
  // started, so R and Theta equal prevR and prevT (no branch flip) and
  // f(s_new) is k1.  Two shortcuts, both exact:
  //  - with r, theta fixed and dr = dth = 0 the event tests see the same
  //    numbers at every step (the Hermite terms in h * dy vanish), so once
  //    they find nothing they are not repeated;
  //  - at h = 100 (the cap) with err <= tol / 2 the new step is the cap
  //    again: sc = 0.9 (tol / err)^0.2 >= 0.9 * 2^0.2 > 1.03 (4 for
  //    err <= 1e-14), so pow is not needed.
  static constexpr int kParkedBudget = 256;
  KT_HD_CALL bool parked_steps(const Frame& f, RayResult* o) {
    const double cph = k1[2];
    const double t = ((cph + 2.0 * cph) + 2.0 * cph) + cph;
    const double tol = f.tol;
    double hh = h, p = ph;
    int n_it = it, rej = rejects;
    uint32_t n_att = attempts;
    bool quiet = false;
    double wh = hh, w = hh / 6.0, wb = (0.5 * hh) / 6.0;  // stage weights of step wh
    for (int n = 0; n < kParkedBudget; ++n) {
      if (hh != wh) {
        wh = hh;
        w = hh / 6.0;
        wb = (0.5 * hh) / 6.0;
      }
      const double Aph = p + w * t;
      const double B1ph = p + wb * t;
      const double Bph = B1ph + wb * t;
      const double used = hh;
      ++n_att;
      bool accepted = false;
      if (!(finite(Aph) && finite(B1ph) && finite(Bph))) {
        hh = dmax(hh * 0.5, 1e-10);
      } else {
        const double e2 = Aph - Bph;
        const double err = sqrt(e2 * e2) / 15.0;  // (0*0 + 0*0) + e2*e2 = e2*e2
        if (!finite(err)) {
          hh = dmax(hh * 0.5, 1e-10);
        } else if (err < tol || hh < 1e-10) {
          accepted = true;
          if (!(hh == 100.0 && (err <= 1e-14 || err <= 0.5 * tol))) {
            const double sc = (err > 1e-14) ? 0.9 * ktm_pow(tol / err, 0.2) : 4.0;
            hh = dclamp(hh * sc, 1e-10, 100.0);
          }
        } else {
          hh = dmax((hh * 0.9) * ktm_pow(tol / err, 0.25), 1e-10);
        }
      }
      if (!accepted) {
        if (!finite(hh) || ++rej > 64) {
          it = n_it;
          attempts = n_att;
          return give_up(o);
        }
        continue;
      }
      const double p_prev = p;
      p = Bph;
      if (!quiet) {
        A[0] = r;
        A[1] = th;
        A[2] = p_prev;
        kp[0] = k1[0];
        kp[1] = k1[1];
        step_used = used;
        ph = p;
        it = n_it;
        attempts = n_att;
        if (events(f, o)) return true;
        quiet = true;
      }
      ++n_it;
      rej = 0;
      if (n_it >= f.max_steps) {
        o->steps = (uint32_t)n_it;
        o->attempts = n_att;
        set_result(o, kOutEscaped, kStStepCap, r, 1.0, 1.0, th, p, 0.0);
        return true;
      }
    }
    h = hh;
    ph = p;
    it = n_it;
    rejects = rej;
    attempts = n_att;
    return false;
  }

  KT_HD bool give_up(RayResult* o) {
    fallback = true;
    o->steps = (uint32_t)it;
    o->attempts = attempts;
    set_result(o, kOutEscaped, kStEvent, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0);
    return true;
  }

  // Events of the accepted step s_prev = A -> (r, th, ph) (main.cpp:633-699).
  KT_HD bool events(const Frame& f, RayResult* o) {
    double best_alpha = 2.0;
    int ev = kEvNone;
    double disk_r = 0.0, disk_red = 1.0, disk_phi = 0.0;
    const double q0 = A[1] - kHalfPi;
    const double q1 = th - kHalfPi;
    if (sign_change(q0, q1) || (dmin(fabs(q0), fabs(q1)) < 0.35)) {
      if (!k1_ok) return give_up(o);  // f(s_prev) was finite: the attempt used it
      double alpha = 0.0;
      if (first_event(A[1], th, kp[1], k1[1], step_used, kHalfPi, &alpha)) {
        const double r_hit = hermite(A[0], r, kp[0], k1[0], step_used, alpha);
        if (r_hit >= f.r_in && r_hit <= f.r_out) {
          disk_r = r_hit;
          disk_red = dclamp(disk_redshift(f.g, f.eq, r_hit, pt, pphi), 0.0, 20.0);
          disk_phi = A[2] + alpha * (ph - A[2]);
          best_alpha = alpha;
          ev = kEvDisk;
        }
      }
    }
    horizon_escape(A[0], r, f.rh_cut, f.r_esc, &best_alpha, &ev);
    if (ev == kEvNone) return false;
    o->steps = (uint32_t)it + 1;
    o->attempts = attempts;
    if (ev == kEvDisk) {
      set_result(o, kOutDisk, kStEvent, disk_r, disk_red, 1.0, disk_phi, 0.0, 0.0);
    } else if (ev == kEvHorizon) {
      set_result(o, kOutHorizon, kStEvent, A[0] + best_alpha * (r - A[0]), 0.0, 1.0, 0.0, 0.0, 0.0);
    } else {
      const double th_esc = A[1] + best_alpha * (th - A[1]);
      const double ph_esc = A[2] + best_alpha * (ph - A[2]);
      // {ESCAPED, r_escape, 1.0, th_esc, ph_esc}: the phi_disk and theta_esc slots
      set_result(o, kOutEscaped, kStEvent, f.r_esc, 1.0, 1.0, th_esc, ph_esc, 0.0);
    }
    return true;
  }

  // k: f at the slot's input; ok: sep_rhs found it finite.  Returns true
  // when the ray is finished (o filled; fallback set if it gave up).
  KT_HD bool consume(const Frame& f, int slot, const double k[3], bool ok, RayResult* o) {
    if (slot < 0) {
      for (int i = 0; i < 3; ++i) k1[i] = k[i];
      k1_ok = ok;
      need_k1 = false;
      if (!pending) return false;
      pending = false;
      if (events(f, o)) return true;
      prevR = Rn;
      prevT = Tn;
      if (end_step(f, o)) return true;
      if (parked()) return parked_steps(f, o);
      return false;
    }
    switch (slot) {
      case 0:
      case 3:
        if (slot == 0) fail = !k1_ok;
        fail = fail || !ok;
        for (int i = 0; i < 3; ++i) sum[i] = k1[i] + 2.0 * k[i];
        for (int i = 0; i < 2; ++i) kp[i] = k[i];
        return false;
      case 1:
      case 4:
      case 7:
      case 8:
        fail = fail || !ok;
        for (int i = 0; i < 3; ++i) sum[i] = sum[i] + 2.0 * k[i];
        for (int i = 0; i < 2; ++i) kp[i] = k[i];
        return false;
      case 6:
        fail = fail || !ok;
        for (int i = 0; i < 3; ++i) sum[i] = k[i];
        for (int i = 0; i < 2; ++i) kp[i] = k[i];
        return false;
      case 2: {
        const double w = h / 6.0;
        A[0] = r + w * (sum[0] + k[0]);
        A[1] = th + w * (sum[1] + k[1]);
        A[2] = ph + w * (sum[2] + k[2]);
        fail = fail || !ok || !(finite(A[0]) && finite(A[1]) && finite(A[2]));
        return false;
      }
      case 5: {
        const double w = (0.5 * h) / 6.0;
        B1[0] = r + w * (sum[0] + k[0]);
        B1[1] = th + w * (sum[1] + k[1]);
        B1[2] = ph + w * (sum[2] + k[2]);
        fail = fail || !ok || !(finite(B1[0]) && finite(B1[1]) && finite(B1[2]));
        return false;
      }
      default: {  // 9: path B2 done -> error control
        const double w = (0.5 * h) / 6.0;
        const double Br = B1[0] + w * (sum[0] + k[0]);
        const double Bth = B1[1] + w * (sum[1] + k[1]);
        const double Bph = B1[2] + w * (sum[2] + k[2]);
        fail = fail || !ok || !(finite(Br) && finite(Bth) && finite(Bph));
        step_used = h;
        ++attempts;
        bool accepted = false;
        if (fail) {
          h = dmax(h * 0.5, 1e-10);
        } else {
          const double e0 = A[0] - Br, e1 = A[1] - Bth, e2 = A[2] - Bph;
          const double err = sqrt((e0 * e0 + e1 * e1) + e2 * e2) / 15.0;
          if (!finite(err)) {
            h = dmax(h * 0.5, 1e-10);
          } else if (err < f.tol || h < 1e-10) {
            const double sc = (err > 1e-14) ? 0.9 * ktm_pow(f.tol / err, 0.2) : 4.0;
            h = dclamp(h * sc, 1e-10, 100.0);
            accepted = true;
          } else {
            h = dmax((h * 0.9) * ktm_pow(f.tol / err, 0.25), 1e-10);
          }
        }
        if (!accepted) {
          if (!finite(h) || ++rejects > 64) return give_up(o);
          return false;
        }
        A[0] = r;  // s_prev
        A[1] = th;
        A[2] = ph;
        kp[0] = k1[0];  // f(s_prev): dr, dth
        kp[1] = k1[1];
        r = Br;
        th = Bth;
        ph = Bph;
        // theta kept in [0, pi], then the turning points of R and Theta flip
        // the branch signs (main.cpp:615-628)
        if (th < 0.0) {
          th = -th;
          sth = -sth;
        } else if (th > kPi) {
          th = 2.0 * kPi - th;
          sth = -sth;
        }
        Rn = sep_R(c, r);
        Tn = sep_Theta(c, th);
        if (Rn <= 1e-9 && prevR > 1e-9) sr = -sr;
        if (Tn <= 1e-11 && prevT > 1e-11) sth = -sth;
        need_k1 = true;
        pending = true;
        return false;
      }
    }
  }
};

}  // namespace kt
