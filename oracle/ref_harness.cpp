// ref_harness.cpp -- TEST INFRASTRUCTURE (oracle), never part of the product.
//
// Compiles the reference renderer itself: the reference's main.cpp (and the
// headers it includes) from a copy of the reference tree made by
// oracle/build.py (one token patched, geodesic.hpp:326, so that g++ 13
// accepts it), with `main` renamed.  The functions below call the
// reference's own static tracers and return their results in float64, so the
// tests can compare the CUDA kernels with the reference on the same inputs.
//
// Two flavours are built from this file:
//   strict : -O2 -ffp-contract=off, the reference's calls to sin, cos, pow,
//            exp, log, log10, cbrt, atan2 and acos bound to the renderer's own
//            libm (ref_libm_interpose.c) -> the bit-exact parity oracle;
//   stock  : the reference's own flags (-O3 -ffast-math, -march=x86-64-v3
//            instead of -march=native so it runs on any AVX2 host) and glibc's
//            libm -> the reference as shipped, the timed CPU baseline.
#define main kt_reference_main
#include "main.cpp"
#undef main

#include <cstdint>
#include <omp.h>

#include "../include/kerrtrace.h"

namespace {

// Result of one ray as the reference computes it before GeoPixel's float
// cast (main.cpp:2111-2149).
struct RayOut {
  uint8_t outcome;
  double r, redshift, magnif, phi_disk, theta_esc, phi_esc;
};

RaySolverMode solver_of(const kt_frame_desc* d) {
  return d->solver_mode == KT_SOLVER_SEMI_ANALYTIC ? RaySolverMode::SEMI_ANALYTIC
         : d->solver_mode == KT_SOLVER_ELLIPTIC_CLOSED ? RaySolverMode::ELLIPTIC_CLOSED
                                                      : RaySolverMode::STANDARD;
}

struct FrameSetup {
  KNdSMetric g;
  Camera cam;
  CoordinateChart eff_chart;
  RaySolverMode solver;  // after select_solver_mode
  Integrator intg;
  IntegratorControls ctl;
  bool bundles;
  double r_disk_in, r_disk_out, r_escape;
  double offx, offy;
};

// The per-frame part of trace_geodesics (main.cpp:2033-2082) and main's
// argument clamps (main.cpp:2683-2686).
FrameSetup setup_frame(const kt_frame_desc* d) {
  KNdSMetric g(d->M, d->a, d->Q, d->Lambda);
  Camera cam(d->r_obs, d->theta_deg, d->phi_deg, d->fov_deg, d->width, d->height);
  CoordinateChart chart = (d->chart == KT_CHART_KS) ? CoordinateChart::KS : CoordinateChart::BL;
  if (chart == CoordinateChart::KS && std::abs(d->Lambda) > 1e-15) chart = CoordinateChart::BL;
  if (d->bundles && chart == CoordinateChart::KS) chart = CoordinateChart::BL;
  IntegratorControls ctl;
  ctl.max_steps = std::max(1, (int)d->max_steps);
  ctl.step_init = std::max(1e-10, d->step_init);
  ctl.tol = std::max(1e-10, d->tol);
  const double r_isco = g.r_isco();
  const RaySolverMode solver =
      select_solver_mode(solver_of(d), d->bundles != 0, chart, d->Q, d->Lambda).effective;
  return FrameSetup{g, cam, chart, solver,
                    d->integrator == KT_DOPRI5 ? Integrator::DOPRI5 : Integrator::RK4_DOUBLING,
                    ctl, d->bundles != 0, r_isco, d->disk_out, cam.r_obs * 1.05,
                    d->pixel_offset_x, d->pixel_offset_y};
}

RayOut trace_one(const FrameSetup& f, int px, int py) {
  RayOut o{};
  if (f.bundles) {
    auto res = trace_bundle(px, py, f.cam, f.g, f.r_disk_in, f.r_disk_out, f.r_escape,
                            f.ctl.max_steps, f.ctl.step_init, f.ctl.tol, f.offx, f.offy);
    o.outcome = res.disk_hit ? 1 : 0;
    o.r = res.disk_hit ? res.r_hit : 0.0;
    o.redshift = res.redshift;
    o.magnif = res.magnif;
    o.phi_disk = res.phi_disk;
    o.theta_esc = res.theta_esc;
    o.phi_esc = res.phi_esc;
    return o;
  }
  auto s = f.cam.pixel_ray(px, py, f.g, f.offx, f.offy);
  TraceResult res{};
  if (f.solver == RaySolverMode::ELLIPTIC_CLOSED) {
    EllipticFallbackReason why = EllipticFallbackReason::NONE;
    res = trace_single_elliptic_closed(s, f.g, f.r_disk_in, f.r_disk_out, f.r_escape, &why,
                                       f.eff_chart, f.intg, f.ctl);
  } else if (f.eff_chart == CoordinateChart::KS)
    res = trace_single_ks(s, f.g, f.r_disk_in, f.r_disk_out, f.r_escape, f.intg, f.ctl);
  else if (f.solver == RaySolverMode::SEMI_ANALYTIC)
    res = trace_single_separable_kerr(s, f.g, f.r_disk_in, f.r_disk_out, f.r_escape, f.ctl);
  else
    res = trace_single(s, f.g, f.r_disk_in, f.r_disk_out, f.r_escape, f.intg, f.ctl);
  o.outcome = (res.out == Outcome::DISK_HIT) ? 1 : (res.out == Outcome::HORIZON) ? 2
            : (res.out == Outcome::ESCAPED_B) ? 3 : 0;
  o.r = res.r;
  o.redshift = res.redshift;
  o.magnif = 1.0;
  o.phi_disk = res.phi_disk;
  o.theta_esc = res.theta_esc;
  o.phi_esc = res.phi_esc;
  return o;
}

}  // namespace

extern "C" {

// Which libm the reference code in this build calls: std::cos as the
// reference's own translation unit sees it.
double ref_libm_probe_cos(double x) { return std::cos(x); }
double ref_libm_probe_pow(double x, double y) { return std::pow(x, y); }

// The elliptic-closed solver's fallback reason (EllipticFallbackReason,
// 0 = the closed form was used or checked) per pixel, from the reference's
// own trace_single_elliptic_closed, for a frame whose effective solver it is.
void ref_elliptic_reasons(const kt_frame_desc* d, int64_t n, const uint32_t* pix, uint8_t* reason,
                          int nthreads) {
  const FrameSetup f = setup_frame(d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const int px = (int)(pix[i] % (uint32_t)d->width);
    const int py = (int)(pix[i] / (uint32_t)d->width);
    auto s = f.cam.pixel_ray(px, py, f.g, f.offx, f.offy);
    EllipticFallbackReason why = EllipticFallbackReason::NONE;
    trace_single_elliptic_closed(s, f.g, f.r_disk_in, f.r_disk_out, f.r_escape, &why, f.eff_chart,
                                 f.intg, f.ctl);
    reason[i] = (uint8_t)why;
  }
}

// Trace pixels pix[i] (= py*width+px) through the reference's per-ray
// tracers, with the dispatch of trace_geodesics; float64 SoA out.
void ref_trace_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix,
                      uint8_t* outcome, double* r, double* redshift, double* magnif,
                      double* phi_disk, double* theta_esc, double* phi_esc, int nthreads) {
  const FrameSetup f = setup_frame(d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const int px = (int)(pix[i] % (uint32_t)d->width);
    const int py = (int)(pix[i] / (uint32_t)d->width);
    const RayOut o = trace_one(f, px, py);
    outcome[i] = o.outcome;
    r[i] = o.r;
    redshift[i] = o.redshift;
    magnif[i] = o.magnif;
    phi_disk[i] = o.phi_disk;
    theta_esc[i] = o.theta_esc;
    phi_esc[i] = o.phi_esc;
  }
}

// The reference's own frame tracer (trace_geodesics), GeoPixel records out
// (28 bytes each, float32 fields).  Checks the dispatch and the float cast.
void ref_trace_geodesics(const kt_frame_desc* d, void* geopixels, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  FrameParams fp;
  fp.a = d->a;
  fp.theta = d->theta_deg;
  fp.phi = d->phi_deg;
  fp.r_obs = d->r_obs;
  fp.disk_out = d->disk_out;
  fp.fov = d->fov_deg;
  IntegratorControls ctl;
  ctl.max_steps = std::max(1, (int)d->max_steps);
  ctl.step_init = std::max(1e-10, d->step_init);
  ctl.tol = std::max(1e-10, d->tol);
  auto geo = trace_geodesics(d->width, d->height, fp, d->bundles != 0, solver_of(d),
                             d->chart == KT_CHART_KS ? CoordinateChart::KS : CoordinateChart::BL,
                             d->integrator == KT_DOPRI5 ? Integrator::DOPRI5 : Integrator::RK4_DOUBLING,
                             ctl, d->pixel_offset_x, d->pixel_offset_y, d->M, d->Q, d->Lambda);
  std::memcpy(geopixels, geo.data(), geo.size() * sizeof(GeoPixel));
}

// colorize_buffer (main.cpp:1817) on GeoPixel records with a background
// given as raw RGB8 (bg may be NULL); rgb out is W*H*3 bytes.
void ref_colorize(const void* geopixels, int W, int H, double exposure, double gamma,
                  double temp_scale, const uint8_t* bg, int bg_w, int bg_h, double M_bh,
                  double r_isco, double r_disk_in, double r_disk_out, uint8_t* rgb) {
  std::vector<GeoPixel> geo((size_t)W * H);
  std::memcpy(geo.data(), geopixels, geo.size() * sizeof(GeoPixel));
  ColorParams cp;
  cp.exposure = exposure;
  cp.gamma = gamma;
  cp.temp_scale = temp_scale;
  BackgroundImage img;
  if (bg && bg_w > 0 && bg_h > 0) {
    img.w = bg_w;
    img.h = bg_h;
    img.px.assign(bg, bg + (size_t)bg_w * bg_h * 3);
  }
  auto out = colorize_buffer(geo, W, H, cp, img, M_bh, r_isco, r_disk_in, r_disk_out);
  std::memcpy(rgb, out.data(), out.size() * 3);
}

static ColorParams to_cp(const kt_color_params* c) {
  ColorParams cp;
  cp.exposure = c->exposure;
  cp.gamma = c->gamma;
  cp.temp_scale = c->temp_scale;
  cp.palette = c->palette == 1 ? DiskPalette::INTERSTELLAR : DiskPalette::BLACKBODY;
  cp.disk_rings = c->disk_rings;
  cp.disk_sectors = c->disk_sectors;
  cp.disk_sigma = c->disk_sigma;
  cp.disk_hue_offset = c->disk_hue_offset;
  return cp;
}

static BackgroundImage to_bg(const uint8_t* bg, int bg_w, int bg_h) {
  BackgroundImage img;
  if (bg && bg_w > 0 && bg_h > 0) {
    img.w = bg_w;
    img.h = bg_h;
    img.px.assign(bg, bg + (size_t)bg_w * bg_h * 3);
  }
  return img;
}

// colorize_buffer with every ColorParams field (both palettes).
void ref_colorize_cp(const void* geopixels, int W, int H, const kt_color_params* c,
                     const uint8_t* bg, int bg_w, int bg_h, double M_bh, double r_isco,
                     double r_disk_in, double r_disk_out, uint8_t* rgb) {
  std::vector<GeoPixel> geo((size_t)W * H);
  std::memcpy(geo.data(), geopixels, geo.size() * sizeof(GeoPixel));
  auto out = colorize_buffer(geo, W, H, to_cp(c), to_bg(bg, bg_w, bg_h), M_bh, r_isco, r_disk_in,
                             r_disk_out);
  std::memcpy(rgb, out.data(), out.size() * 3);
}

// render_image (main.cpp:2209-2478, CPU branch) with camera_spp passes.
void ref_render_image(const kt_frame_desc* d, const kt_color_params* c, const uint8_t* bg, int bg_w,
                      int bg_h, int camera_spp, int nthreads, uint8_t* rgb) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  FrameParams fp;
  fp.a = d->a;
  fp.theta = d->theta_deg;
  fp.phi = d->phi_deg;
  fp.r_obs = d->r_obs;
  fp.disk_out = d->disk_out;
  fp.fov = d->fov_deg;
  IntegratorControls ctl;
  ctl.max_steps = std::max(1, (int)d->max_steps);
  ctl.step_init = std::max(1e-10, d->step_init);
  ctl.tol = std::max(1e-10, d->tol);
  auto out = render_image(d->width, d->height, fp, to_bg(bg, bg_w, bg_h), d->bundles != 0,
                          solver_of(d),
                          d->chart == KT_CHART_KS ? CoordinateChart::KS : CoordinateChart::BL,
                          d->integrator == KT_DOPRI5 ? Integrator::DOPRI5 : Integrator::RK4_DOUBLING,
                          ctl, camera_spp, d->M, d->Q, d->Lambda, IntersectionMode::HERMITE, 0, false,
                          false, false, to_cp(c), nullptr, false, d->pixel_offset_x,
                          d->pixel_offset_y);
  std::memcpy(rgb, out.data(), out.size() * 3);
}

// Per-frame scalars as the reference computes them.
double ref_r_horizon(double M, double a, double Q, double L) { return KNdSMetric(M, a, Q, L).r_horizon(); }
double ref_r_isco(double M, double a, double Q, double L) { return KNdSMetric(M, a, Q, L).r_isco(); }
double ref_keplerian_omega(double M, double a, double Q, double L, double r) {
  return KNdSMetric(M, a, Q, L).keplerian_omega(r);
}

// Metric tensors (for the known-answer tests of tests/core_tests.cpp).
void ref_covariant_BL(double M, double a, double Q, double L, double r, double th, double* g16) {
  double g[4][4];
  KNdSMetric(M, a, Q, L).covariant_BL(r, th, g);
  std::memcpy(g16, g, sizeof g);
}
void ref_contravariant_BL(double M, double a, double Q, double L, double r, double th, double* g16) {
  double g[4][4];
  KNdSMetric(M, a, Q, L).contravariant_BL(r, th, g);
  std::memcpy(g16, g, sizeof g);
}
void ref_contravariant_KS(double M, double a, double Q, double X, double Y, double Z, double* g16) {
  double g[4][4];
  KNdSMetric(M, a, Q, 0.0).contravariant_KS(0.0, X, Y, Z, KS_INGOING, g);
  std::memcpy(g16, g, sizeof g);
}
double ref_hamiltonian(double M, double a, double Q, double L, const double* s7) {
  return KNdSMetric(M, a, Q, L).hamiltonian(s7[0], s7[1], s7[3], s7[4], s7[5], s7[6]);
}

// Camera::angle_ray / pixel_ray: GeodesicState {r, th, phi, pr, pth, pt, pphi}.
void ref_angle_ray(double M, double a, double Q, double L, double r_obs, double th_deg,
                   double ph_deg, double fov_deg, int W, int H, double alpha, double beta,
                   double* s7) {
  KNdSMetric g(M, a, Q, L);
  Camera cam(r_obs, th_deg, ph_deg, fov_deg, W, H);
  GeodesicState s = cam.angle_ray(alpha, beta, g);
  const double v[7] = {s.r, s.theta, s.phi, s.pr, s.ptheta, s.pt, s.pphi};
  std::memcpy(s7, v, sizeof v);
}

// One adaptive attempt (adaptive_step, geodesic.hpp:423) on a state; returns
// accepted and updates s7 and h.  fsal4 is the DOPRI5 FSAL vector.
int ref_adaptive_step(double M, double a, double Q, double L, double* s7, double* h, int dopri5,
                      double* fsal4, double tol) {
  KNdSMetric g(M, a, Q, L);
  GeodesicState s{s7[0], s7[1], s7[2], s7[3], s7[4], s7[5], s7[6]};
  Vec4d f;
  for (int i = 0; i < 4; ++i) f.v[i] = fsal4[i];
  bool acc = adaptive_step(g, s, *h, dopri5 ? Integrator::DOPRI5 : Integrator::RK4_DOUBLING, f, tol);
  const double v[7] = {s.r, s.theta, s.phi, s.pr, s.ptheta, s.pt, s.pphi};
  std::memcpy(s7, v, sizeof v);
  for (int i = 0; i < 4; ++i) fsal4[i] = f.v[i];
  return acc ? 1 : 0;
}

void ref_bl_to_ks(double r, double th, double ph, double a, double* xyz) {
  KNdSMetric::BL_to_KS_spatial(r, th, ph, a, xyz[0], xyz[1], xyz[2]);
}
void ref_ks_to_bl(double X, double Y, double Z, double a, double* rtp) {
  KNdSMetric::KS_to_BL_spatial(X, Y, Z, a, rtp[0], rtp[1], rtp[2]);
}
double ref_r_ks(double X, double Y, double Z, double a) { return KNdSMetric::r_KS(X, Y, Z, a); }

// disk_colour (main.cpp:1799) and BackgroundImage::sample (main.cpp:153).
void ref_disk_colour(double r, double red, double magnif, double M, double r_isco,
                     double exposure, double gamma, double temp_scale, uint8_t* rgb3) {
  ColorParams cp;
  cp.exposure = exposure;
  cp.gamma = gamma;
  cp.temp_scale = temp_scale;
  RGB c = disk_colour(r, red, magnif, M, r_isco, cp);
  rgb3[0] = c.r;
  rgb3[1] = c.g;
  rgb3[2] = c.b;
}

}  // extern "C"
