// kt_frame.cpp -- host-side frame preparation (the per-frame part of the
// reference's trace_geodesics, main.cpp:2014-2082).
//
// Validates a kt_frame_desc, applies the reference's chart fallback rules and
// argument clamps, and computes the frame constants the kernels use: outer
// horizon r_+ (knds_metric.hpp:237-315), ISCO (knds_metric.hpp:318-349),
// disk bounds, escape radius, and the observer's metric for the camera.  The
// arithmetic is the reference's, evaluated with the renderer's libm so that
// every derived constant is bit-identical to what the reference computes.
// Compile with -ffp-contract=off.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#include <unistd.h>
#endif

#include "kt_frame.h"

namespace kt {

// f(0) .. f(n-1), independent of one another: the samples of the horizon
// scan and the ISCO search (each the same arithmetic as in a serial loop;
// the pass that reads them is serial).  Up to 16 host threads; serial in a
// process forked from the one whose OpenMP thread pool exists, where that
// pool is unusable.
template <class F>
static void for_each_sample(int n, F&& f) {
  int threads = 1;
#ifdef _OPENMP
  static const pid_t owner = getpid();
  if (getpid() == owner) {
    threads = omp_get_max_threads();
    if (threads > 16) threads = 16;
  }
  if (threads > 1 && n > 1) {
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
#endif
  for (int i = 0; i < n; ++i) f(i);
}

static double delta_r(const Metric& g, double r) { return bl_delta_r(g, r, r * r + g.a2); }

// The roots of Delta_r for Lambda != 0 as r_horizon finds them
// (knds_metric.hpp:244-314): a 20000-point logarithmic scan with 160-step
// bisection; sorted, at most 16.
static int knds_roots(const Metric& g, double roots[16]) {
  const double M = g.M, a = g.a, Q = g.Q, L = g.L;
  const double scale = dmax(fabs(M), 1.0);
  const double rmin = dmax(1e-6 * scale, 1e-9);
  double rmax;
  if (L > 0.0)
    rmax = dmax(20.0 * scale, 1.25 * sqrt(3.0 / L));
  else
    rmax = (200.0 * scale + 20.0 * fabs(a)) + 20.0 * fabs(Q);
  if (!(rmax > rmin)) rmax = rmin * 10.0;

  auto bisect = [&](double lo, double hi) -> double {
    double flo = delta_r(g, lo), fhi = delta_r(g, hi);
    if (!finite(flo) || !finite(fhi)) return ktm_nan();
    for (int i = 0; i < 160; ++i) {
      const double mid = 0.5 * (lo + hi);
      const double fmid = delta_r(g, mid);
      if (!finite(fmid)) break;
      if ((flo > 0.0 && fmid < 0.0) || (flo < 0.0 && fmid > 0.0)) {
        hi = mid;
        fhi = fmid;
      } else {
        lo = mid;
        flo = fmid;
      }
    }
    (void)fhi;
    return 0.5 * (lo + hi);
  };
  int nroots = 0;
  auto push_root = [&](double rr) {
    if (!finite(rr) || rr <= 0.0) return;
    for (int i = 0; i < nroots; ++i) {
      double rel = 1.0;
      if (rel < fabs(roots[i])) rel = fabs(roots[i]);
      if (rel < fabs(rr)) rel = fabs(rr);
      if (fabs(roots[i] - rr) <= 1e-8 * rel) return;
    }
    if (nroots < 16) roots[nroots++] = rr;
  };
  const int samples = 20000;
  const double log_span = ktm_log(rmax / rmin);
  std::vector<double> rs(samples + 1), fs(samples + 1);
  rs[0] = rmin;
  fs[0] = delta_r(g, rmin);
  for_each_sample(samples, [&](int j) {
    const int i = j + 1;
    const double t = (double)i / (double)samples;
    rs[i] = rmin * ktm_exp(log_span * t);
    fs[i] = delta_r(g, rs[i]);
  });
  double prev_r = rs[0];
  double prev_f = fs[0];
  for (int i = 1; i <= samples; ++i) {
    const double r = rs[i];
    const double f = fs[i];
    if (finite(prev_f) && finite(f)) {
      if (prev_f == 0.0) push_root(prev_r);
      if (f == 0.0) push_root(r);
      if ((prev_f > 0.0 && f < 0.0) || (prev_f < 0.0 && f > 0.0)) push_root(bisect(prev_r, r));
    }
    prev_r = r;
    prev_f = f;
  }
  std::sort(roots, roots + nroots);
  return nroots;
}

// r_horizon (knds_metric.hpp:237-315): closed form for Lambda = 0, else the
// largest root of Delta_r, or for Lambda > 0 (the largest is cosmological)
// the next one.
double host_r_horizon(const Metric& g) {
  const double M = g.M, a = g.a, Q = g.Q, L = g.L;
  if (fabs(L) < 1e-15) {
    const double disc = (M * M - a * a) - Q * Q;
    return M + sqrt(dmax(disc, 0.0));
  }
  double roots[16];
  const int nroots = knds_roots(g, roots);
  if (nroots == 0) {
    const double disc = (M * M - a * a) - Q * Q;
    return M + sqrt(dmax(disc, 0.0));
  }
  if (L > 0.0 && nroots >= 2) return roots[nroots - 2];
  return roots[nroots - 1];
}

// The cosmological horizon for Lambda > 0 (the largest root), else +inf.
double host_r_cosmo(const Metric& g) {
  if (!(g.L > 0.0) || fabs(g.L) < 1e-15) return ktm_inf();
  double roots[16];
  const int nroots = knds_roots(g, roots);
  return nroots >= 2 ? roots[nroots - 1] : ktm_inf();
}

// r_isco (knds_metric.hpp:318-349): Bardeen-Press-Teukolsky closed form for
// Kerr; otherwise the first radius (1e-4 M steps from 1.05 r_+) where the
// circular-orbit angular momentum stops decreasing.
double host_r_isco(const Metric& g, double rh) {
  const double M = g.M, a = g.a;
  if (fabs(g.L) < 1e-15 && fabs(g.Q) < 1e-15) {
    if (fabs(a) < 1e-10) return 6.0 * M;
    const double ap = a / M;
    const double z1 = 1.0 + ktm_cbrt(1.0 - ap * ap) * (ktm_cbrt(1.0 + ap) + ktm_cbrt(1.0 - ap));
    const double z2 = sqrt((3.0 * ap) * ap + z1 * z1);
    return M * ((3.0 + z2) - sqrt((3.0 - z1) * ((3.0 + z1) + 2.0 * z2)));
  }
  const Ang eq = bl_ang(g, kHalfPi);
  auto L_circ = [&](double rr) -> double {
    const double Om = kepler_omega(g, rr);
    const Cov G = bl_cov(g, rr, eq);
    const double N2 = -((G.tt + (2.0 * G.tp) * Om) + (G.pp * Om) * Om);
    if (N2 <= 0.0) return -1e30;
    const double ut = 1.0 / sqrt(N2);
    return -(G.tp + G.pp * Om) * ut;
  };
  // The reference's loop: r from 1.05 r_+ in steps of dr (accumulated),
  // return r at the first step where L(r + dr) < L(r) > 0, else the r that
  // ends the loop at 30 M.  Here the loop's r values are generated serially
  // in chunks, L at each r + dr evaluated in parallel, then scanned in order.
  double r = rh * 1.05;
  const double dr = 1e-4 * M;
  double L_prev = L_circ(r);
  const int chunk = 2048;
  std::vector<double> rv(chunk), Lv(chunk);
  while (r < 30.0 * M) {
    int n = 0;
    for (double x = r; n < chunk && x < 30.0 * M; x += dr) rv[n++] = x;
    for_each_sample(n, [&](int j) { Lv[j] = L_circ(rv[j] + dr); });
    for (int j = 0; j < n; ++j) {
      if (Lv[j] < L_prev && L_prev > 0.0) return rv[j];
      L_prev = Lv[j];
    }
    r = rv[n - 1] + dr;
  }
  return r;
}

static bool all_finite(std::initializer_list<double> xs) {
  for (double x : xs)
    if (!finite(x)) return false;
  return true;
}

kt_status prepare_frame(const kt_frame_desc* d, Frame* f, kt_frame_derived* dv, std::string* err) {
  if (d == nullptr) {
    *err = "frame descriptor is NULL";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->width < 1 || d->height < 1) {
    *err = "width and height must be >= 1";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if ((int64_t)d->width * (int64_t)d->height > (int64_t)0x7fffffff) {
    *err = "width*height exceeds 2^31-1 pixels";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (!all_finite({d->M, d->a, d->Q, d->Lambda, d->theta_deg, d->phi_deg, d->r_obs, d->disk_out,
                   d->fov_deg, d->pixel_offset_x, d->pixel_offset_y, d->step_init, d->tol})) {
    *err = "non-finite frame parameter";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->chart != KT_CHART_KS && d->chart != KT_CHART_BL) {
    *err = "chart must be KT_CHART_KS or KT_CHART_BL";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->integrator != KT_RK4_DOUBLING && d->integrator != KT_DOPRI5) {
    *err = "integrator must be KT_RK4_DOUBLING or KT_DOPRI5";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->bundles != 0 && d->bundles != 1) {
    *err = "bundles must be 0 or 1";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->solver_mode != KT_SOLVER_STANDARD && d->solver_mode != KT_SOLVER_SEMI_ANALYTIC &&
      d->solver_mode != KT_SOLVER_ELLIPTIC_CLOSED) {
    *err = "solver_mode must be KT_SOLVER_STANDARD, _SEMI_ANALYTIC or _ELLIPTIC_CLOSED";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (d->precision != KT_PREC_FP64 && d->precision != KT_PREC_MIXED &&
      d->precision != KT_PREC_SMOOTH) {
    *err = "precision must be KT_PREC_FP64, KT_PREC_MIXED or KT_PREC_SMOOTH";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if ((d->flags & ~(uint32_t)(KT_FLAG_ANGLES_RADIANS | KT_FLAG_BUNDLE_FULL_CREEP)) != 0) {
    *err = "unknown bits in flags";
    return KT_ERR_INVALID_ARGUMENT;
  }
  if (!(d->r_obs > 0.0) || !(d->M > 0.0)) {
    *err = "r_obs and M must be positive";
    return KT_ERR_INVALID_ARGUMENT;
  }

  Frame fr;
  memset(&fr, 0, sizeof fr);
  fr.g = make_metric(d->M, d->a, d->Q, d->Lambda);
  // Chart fallback rules (main.cpp:2033-2049).
  int chart = d->chart;
  if (chart == KT_CHART_KS && fabs(d->Lambda) > 1e-15) chart = KT_CHART_BL;
  if (d->bundles && chart == KT_CHART_KS) chart = KT_CHART_BL;
  fr.chart = chart;
  fr.intg = d->integrator;
  fr.bundles = d->bundles;
  // select_solver_mode (main.cpp:235-276) on the effective chart: bundles,
  // and the KS chart for the semi-analytic solver, take the standard
  // tracers; both other solvers need Kerr (Q = Lambda = 0).
  int solver = d->solver_mode;
  const bool kerr = fabs(d->Q) <= 1e-15 && fabs(d->Lambda) <= 1e-15;
  if (d->bundles && solver != KT_SOLVER_STANDARD) solver = KT_SOLVER_STANDARD;
  if (solver == KT_SOLVER_SEMI_ANALYTIC && (chart != KT_CHART_BL || !kerr)) solver = KT_SOLVER_STANDARD;
  if (solver == KT_SOLVER_ELLIPTIC_CLOSED && !kerr) solver = KT_SOLVER_STANDARD;
  if (solver != KT_SOLVER_STANDARD && d->precision != KT_PREC_FP64) {
    *err = "the semi-analytic and elliptic-closed solvers run in FP64 only";
    return KT_ERR_UNSUPPORTED;
  }
  fr.solver = solver;
  // Camera (camera.hpp:32-35): degrees -> radians as theta_deg * M_PI / 180.
  double th, ph, fov;
  if (d->flags & KT_FLAG_ANGLES_RADIANS) {
    th = d->theta_deg;
    ph = d->phi_deg;
    fov = d->fov_deg;
  } else {
    th = (d->theta_deg * kPi) / 180.0;
    ph = (d->phi_deg * kPi) / 180.0;
    fov = (d->fov_deg * kPi) / 180.0;
  }
  fr.cam = make_camera(fr.g, d->r_obs, th, ph, fov, d->width, d->height, d->pixel_offset_x,
                       d->pixel_offset_y);
  fr.eq = bl_ang(fr.g, kHalfPi);
  // Controls with main()'s clamps (main.cpp:2683-2686) and the tracers' own
  // max(step_init, 1e-10) / max(1, max_steps).
  fr.max_steps = std::max(1, (int)d->max_steps);
  fr.dlam0 = dmax(dmax(1e-10, d->step_init), 1e-10);
  fr.tol = dmax(1e-10, d->tol);
  const double rh = host_r_horizon(fr.g);
  const double r_isco = host_r_isco(fr.g, rh);
  fr.rh_cut = rh * 1.03;
  fr.r_in = r_isco;
  fr.r_out = d->disk_out;
  fr.r_esc = d->r_obs * 1.05;
  fr.bundle_eps = (fov / (double)d->width) * 0.5;
  // Mixed precision: the FP32 RHS carries ~1e-7 relative rounding noise, which
  // the step controller sees as error; it is used only when the tolerance is
  // looser than 1e-8, beyond max(4M, 2 r_+), away from turning points.
  fr.precision = d->precision;
  fr.r_fp32 = (d->precision == KT_PREC_MIXED && fr.tol >= 1e-8) ? dmax(4.0 * d->M, 2.0 * rh)
                                                                  : ktm_inf();
  fr.turn_frac = 0.05;
  // Bundles: rays whose step skipped the horizon and escape tests (near the
  // equator, no crossing found) and that creep onto a horizon in BL
  // coordinates end with the record the controller's eventual failure gives
  // them (status KT_RAY_CREEP).  Ingoing within 1e-4 r_+ of r_+, in every
  // precision: r decreases monotonically there (inside every photon orbit),
  // below rh_cut and -- checked here, with a margin for the Hermite
  // interpolant -- below the disk's inner edge, so no ending of the ray can
  // be a disk hit or an escape and its record is BundleResult{}'s whatever
  // it does next.  Outgoing within 1e-4 r_c of the cosmological horizon:
  // mixed and smooth only (an FP64 ray there may still leave the band
  // beyond r_escape and record an escape).  KT_FLAG_BUNDLE_FULL_CREEP traces
  // them on, as the reference does, for its step and attempt counts.
  const double r_doom = rh * (1.0 + 1e-4);
  const bool creep_end = d->bundles && !(d->flags & KT_FLAG_BUNDLE_FULL_CREEP);
  fr.r_doom = (creep_end && r_isco > 1.01 * r_doom) ? r_doom : -ktm_inf();
  fr.r_cdoom = (creep_end && d->precision != KT_PREC_FP64) ? host_r_cosmo(fr.g) * (1.0 - 1e-4)
                                                          : ktm_inf();
  *f = fr;
  if (dv) {
    memset(dv, 0, sizeof *dv);
    dv->chart = chart;
    dv->integrator = (chart == KT_CHART_KS) ? KT_RK4_DOUBLING : d->integrator;
    dv->r_horizon = rh;
    dv->rh_cut = fr.rh_cut;
    dv->r_isco = r_isco;
    dv->r_disk_in = fr.r_in;
    dv->r_disk_out = fr.r_out;
    dv->r_escape = fr.r_esc;
    dv->r_obs = d->r_obs;
    dv->theta_obs = th;
    dv->phi_obs = ph;
    dv->fov_h = fov;
    dv->dlam0 = fr.dlam0;
    dv->max_steps = fr.max_steps;
    dv->solver = fr.solver;
    dv->tol = fr.tol;
    dv->bundle_eps = fr.bundle_eps;
    dv->r_fp32 = fr.r_fp32;
  }
  return KT_OK;
}

ColourConst make_colour(const Frame& f, const kt_color_params& cp) {
  ColourConst cc;
  cc.M = f.g.M;
  cc.r_isco = f.r_in;
  cc.exposure = cp.exposure;
  cc.gamma = cp.gamma;
  cc.temp_scale = cp.temp_scale;
  cc.log10_50 = ktm_log10(4e4 / 800.0);  // blackbody's log10(4e4/800.0), main.cpp:1665
  cc.pt_peak = page_thorne(3.0 * f.r_in, f.r_in);
  cc.palette = cp.palette;
  cc.rings = cp.disk_rings;
  cc.sectors = cp.disk_sectors;
  cc.pad0 = 0;
  cc.sigma = cp.disk_sigma;
  cc.hue_offset = cp.disk_hue_offset;
  cc.r_in = f.r_in;
  cc.r_out = f.r_out;
  return cc;
}

}  // namespace kt
