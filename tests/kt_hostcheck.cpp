// kt_hostcheck.cpp -- TEST-ONLY host build of the GPU kernels' per-ray code.
//
// The kernels' state machines (kt_machines.cuh) are written for host and
// device.  This file runs them on the CPU, one ray after another, exactly as
// the persistent kernel does for one lane, so the CPU test suite can check
// their arithmetic against the oracle without a GPU.  It is not a fallback:
// the product library has no CPU tracing path and nothing outside tests/
// loads this library.  Built by tests/conftest.py with -ffp-contract=off.
#include <stdint.h>

#include <string>

#include "../include/kerrtrace.h"
#include "../kerrtracecpp2_b200/csrc/kt_frame.h"
#include "../kerrtracecpp2_b200/csrc/kt_internal.h"
#include "../kerrtracecpp2_b200/csrc/kt_elliptic.cuh"
#include "../kerrtracecpp2_b200/csrc/kt_smray.cuh"

using namespace kt;

namespace {

Geo camera_ray(const Frame& f, uint32_t pix) {
  const int px = (int)(pix % (uint32_t)f.cam.W);
  const int py = (int)(pix / (uint32_t)f.cam.W);
  double al, be;
  pixel_angles(f.cam, px, py, &al, &be);
  return angle_ray(f.cam, al, be);
}

// The mixed-precision right-hand sides of kt_mixed.cu for one lane (the
// kernel decides FP32 per warp; a single lane decides for itself).
void bl_rhs_mixed_host(const Frame& f, const double y[4], double pt, double pphi, double k[5]) {
  const double lim = f.turn_frac * fabs(pt);
  if (y[0] > f.r_fp32 && fabs(y[2]) > lim && fabs(y[3]) > lim * y[0])
    bl_rhs_analytic<float>(f.g, y[0], y[1], y[2], y[3], pt, pphi, k);
  else
    bl_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], pt, pphi, k);
}

void ks_rhs_mixed_host(const Frame& f, const double y[6], double pT, double k[6]) {
  const double rr = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
  const double prad = (y[0] * y[3] + y[1] * y[4] + y[2] * y[5]) / rr;
  if (rr > f.r_fp32 && fabs(prad) > f.turn_frac * fabs(pT))
    ks_rhs_analytic<float>(f.g, y[0], y[1], y[2], y[3], y[4], y[5], pT, k);
  else
    ks_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], y[4], y[5], pT, k);
}

// One lane of the kernel: the slot sequence of k_trace for a single ray.
template <class M>
RayResult run_bl(const Frame& f, const Geo& s) {
  M m;
  m.init(f, s);
  RayResult res;
  for (;;) {
    for (int slot = -1; slot < M::kSlots; ++slot) {
      if (slot < 0 && !m.needs_k1()) continue;
      double y[4], k[5];
      m.input(slot, y);
      if (f.precision == KT_PREC_MIXED)
        bl_rhs_mixed_host(f, y, m.pt, m.pphi, k);
      else
        bl_rhs(f.g, y[0], y[1], y[2], y[3], m.pt, m.pphi, k);
      const int it0 = m.it;
      if (m.consume(f, slot, k, &res)) return res;
      if (f.precision == KT_PREC_MIXED) mixed_after_slot(f, &m, slot, it0);
    }
  }
}

RayResult run_ray_standard(const Frame& f, uint32_t pix);

// The elliptic-closed solver as the kernels run it: the standard trace,
// then the closed-form disk hit unless the standard trace ends at the horizon.
RayResult run_ray(const Frame& f, uint32_t pix) {
  RayResult res = run_ray_standard(f, pix);
  if (f.solver != KT_SOLVER_ELLIPTIC_CLOSED || res.outcome == kOutHorizon) return res;
  double r, g;
  int why;
  if (elliptic_closed_form(f, camera_ray(f, pix), &r, &g, &why))
    set_result(&res, kOutDisk, res.status, r, g, 1.0, 0.0, 0.0, 0.0);
  return res;
}

// Bundle RHS through the two-lane split (bundle_rhs_half for both lanes,
// then bundle_rhs_combine), as the paired bundle kernel evaluates it.
int g_bundle_split = 0;  // 1: the rolled code shape, 2: the unrolled one

void bundle_rhs_split(const Metric& g, const double y[4], double pt, double pphi,
                      const double W[8], double k[5], double kW[8]) {
  BundleHalf E, O;
  if (g_bundle_split == 2) {
    bundle_rhs_half<false>(g, y[0], y[1], y[2], y[3], pt, pphi, false, &E);
    bundle_rhs_half<false>(g, y[0], y[1], y[2], y[3], pt, pphi, true, &O);
  } else {
    bundle_rhs_half<true>(g, y[0], y[1], y[2], y[3], pt, pphi, false, &E);
    bundle_rhs_half<true>(g, y[0], y[1], y[2], y[3], pt, pphi, true, &O);
  }
  bundle_rhs_combine(E, O, y[0], y[2], y[3], W, k, kW);
}

RayResult run_ray_standard(const Frame& f, uint32_t pix) {
  if (f.bundles) {
    Bundle m;
    m.init(f, (int)(pix % (uint32_t)f.cam.W), (int)(pix / (uint32_t)f.cam.W));
    RayResult res;
    for (;;) {
      for (int slot = -1; slot < Bundle::kSlots; ++slot) {
        if (slot < 0 && !m.needs_k1()) continue;
        double y[4], yW[8], k[5], kW[8];
        m.input(slot, y, yW);
        if (f.precision == KT_PREC_MIXED)
          bundle_rhs_analytic(f.g, y, m.pt, m.pphi, yW, k, kW);
        else if (g_bundle_split)
          bundle_rhs_split(f.g, y, m.pt, m.pphi, yW, k, kW);
        else
          bundle_rhs(f.g, y[0], y[1], y[2], y[3], m.pt, m.pphi, yW, k, kW);
        if (m.consume(f, slot, k, kW, &res)) return res;
      }
    }
  }
  const Geo s = camera_ray(f, pix);
  if (f.solver == KT_SOLVER_SEMI_ANALYTIC) {
    SepRk4 m;
    if (m.init(f, s, pix, pix)) {
      RayResult res;
      for (;;) {
        bool done = false;
        for (int slot = -1; slot < SepRk4::kSlots && !done; ++slot) {
          if (slot < 0 && !m.needs_k1()) continue;
          double y[2], k[3];
          m.input(slot, y);
          const bool ok = m.rhs(slot, y, k);
          done = m.consume(f, slot, k, ok, &res);
        }
        if (done) {
          if (!m.fallback) return res;
          break;
        }
      }
    }
    return run_bl<BLRk4>(f, s);  // the separable tracer gave up: standard BL, RK4
  }
  if (f.chart == KT_CHART_KS) {
    KSRk4 m;
    if (m.init(f, s)) {
      RayResult res;
      for (;;) {
        for (int slot = -1; slot < KSRk4::kSlots; ++slot) {
          if (slot < 0 && !m.needs_k1()) continue;
          double y[6], k[6];
          m.input(slot, y);
          if (f.precision == KT_PREC_MIXED)
            ks_rhs_mixed_host(f, y, m.pT, k);
          else
            ks_rhs(f.g, y[0], y[1], y[2], y[3], y[4], y[5], m.pT, k);
          const int it0 = m.it;
          if (m.consume(f, slot, k, &res)) return res;
          if (f.precision == KT_PREC_MIXED) mixed_after_slot(f, &m, slot, it0);
        }
      }
    }
  }
  return f.intg == KT_DOPRI5 ? run_bl<BLDopri5>(f, s) : run_bl<BLRk4>(f, s);
}

}  // namespace

// The mixed tracer's constraint reprojection on one state: the camera ray
// of pixel `pix` with its evolved momenta scaled by (1 + eps), reprojected;
// returns 1 when it scaled, and the Hamiltonian (BL: g^{mu nu} of the exact
// path; KS: the reference's hamiltonian_KS form) before and after, over the
// scale p_t^2 (BL) or p_T^2 (KS).
extern "C" int hc_reproject(const kt_frame_desc* d, uint32_t pix, double eps, double* h_before,
                            double* h_after) {
  Frame f;
  std::string err;
  if (prepare_frame(d, &f, nullptr, &err) != KT_OK) return -1;
  const Geo s = camera_ray(f, pix);
  if (f.chart == KT_CHART_BL) {
    double pr = s.pr * (1.0 + eps), pth = s.pth * (1.0 + eps);
    auto ham = [&](double a_pr, double a_pth) {
      const Inv U = bl_inv(f.g, s.r, bl_ang(f.g, s.th));
      return bl_ham(U, a_pr, a_pth, s.pt, s.pphi) / (s.pt * s.pt);
    };
    *h_before = ham(pr, pth);
    const int done = bl_reproject(f, s.r, s.th, &pr, &pth, s.pt, s.pphi) ? 1 : 0;
    *h_after = ham(pr, pth);
    return done;
  }
  KSState k;
  if (!init_ks_state(f.g, s, &k)) return -2;
  double st[6] = {k.X, k.Y, k.Z, k.pX * (1.0 + eps), k.pY * (1.0 + eps), k.pZ * (1.0 + eps)};
  auto ham = [&](const double* x) {
    double G[16];
    ks_inv(f.g, x[0], x[1], x[2], G);
    const double p[4] = {k.pT, x[3], x[4], x[5]};
    return ks_ham(G, p) / (k.pT * k.pT);
  };
  *h_before = ham(st);
  const int done = ks_reproject(f, st, k.pT) ? 1 : 0;
  *h_after = ham(st);
  return done;
}

static int trace_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix, uint8_t* outcome,
                        double* r, double* red, double* magnif, double* phi_disk, double* th_esc,
                        double* ph_esc, uint8_t* status, uint32_t* steps, uint32_t* attempts,
                        bool fp64_rhs, double tol) {
  Frame f;
  std::string err;
  if (prepare_frame(d, &f, nullptr, &err) != KT_OK) return 1;
  if (fp64_rhs) f.r_fp32 = INFINITY;
  if (tol > 0.0) f.tol = tol;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t i = 0; i < n; ++i) {
    const RayResult o = run_ray(f, pix[i]);
    outcome[i] = (uint8_t)o.outcome;
    r[i] = o.r;
    red[i] = o.red;
    magnif[i] = o.magnif;
    phi_disk[i] = o.phi_disk;
    th_esc[i] = o.th_esc;
    ph_esc[i] = o.ph_esc;
    if (status) status[i] = (uint8_t)o.status;
    if (steps) steps[i] = o.steps;
    if (attempts) attempts[i] = o.attempts;
  }
  return 0;
}

// FP64 bundle frames take the two-lane split of the bundle RHS: 1 in its
// rolled code shape, 2 unrolled; 0 the single-lane bundle_rhs.
extern "C" void hc_set_bundle_split(int mode) { g_bundle_split = mode; }

extern "C" int hc_trace_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix,
                               uint8_t* outcome, double* r, double* red, double* magnif,
                               double* phi_disk, double* th_esc, double* ph_esc, uint8_t* status,
                               uint32_t* steps, uint32_t* attempts) {
  return trace_pixels(d, n, pix, outcome, r, red, magnif, phi_disk, th_esc, ph_esc, status, steps,
                      attempts, false, 0.0);
}

// The mixed tracer (KT_PREC_MIXED frames) with its FP32 right-hand side and
// constraint reprojection switched off: the analytic FP64 Hamiltonian
// gradient, on the host with correctly rounded reciprocals and the
// renderer's sincos, no contraction.  Separates the mixed kernels' own error
// (FP32, approximate reciprocals and sincos, FMA) from the difference
// between the analytic gradient and the reference's finite differences.
// tol > 0 replaces the frame's tolerance after the set-up (which clamps it to
// 1e-10 as main.cpp:2683-2716 does), for traces tighter than any frame's.
extern "C" int hc_trace_pixels_fp64_rhs(const kt_frame_desc* d, int64_t n, const uint32_t* pix,
                                        uint8_t* outcome, double* r, double* red, double* magnif,
                                        double* phi_disk, double* th_esc, double* ph_esc,
                                        uint8_t* status, uint32_t* steps, uint32_t* attempts,
                                        double tol) {
  return trace_pixels(d, n, pix, outcome, r, red, magnif, phi_disk, th_esc, ph_esc, status, steps,
                      attempts, true, tol);
}

// The smooth tracer and its adjoint on the host (kt_smray.cuh compiled by
// g++ with the kernels' floating-point flags): pixels pix[0..n) of the
// frame; cotangent mode 0 (forward only), 1 (arrays over the frame's pixels)
// or 2 (L2 against target arrays); contrib[kGSlots][n] per listed pixel.
// Bundle frames take the bundle tracer (cot_m / t_m, w_m: the
// magnification's cotangent or target; magnif may be NULL).
extern "C" int hc_smooth_pixels_m(const kt_frame_desc* d, int64_t n, const uint32_t* pix, int mode,
                                  int force_bl, int tangent_dir, const double* cot_g,
                                  const double* cot_r, const double* cot_m, const uint8_t* t_out,
                                  const double* t_g, const double* t_r, const double* t_m,
                                  double w_g, double w_r, double w_m, uint8_t* outcome, double* r,
                                  double* red, double* magnif, double* phi_disk, double* th_esc,
                                  double* ph_esc, uint32_t* steps, uint32_t* attempts,
                                  double* contrib) {
  kt_frame_desc dd = *d;
  dd.precision = KT_PREC_SMOOTH;
  Frame f;
  std::string err;
  if (prepare_frame(&dd, &f, nullptr, &err) != KT_OK) return 1;
  SmCot cot;
  memset(&cot, 0, sizeof cot);
  cot.mode = mode;
  cot.g = cot_g;
  cot.r = cot_r;
  cot.t_out = t_out;
  cot.t_g = t_g;
  cot.t_r = t_r;
  cot.w_g = w_g;
  cot.w_r = w_r;
  cot.m = cot_m;
  cot.t_m = t_m;
  cot.w_m = w_m;
  // BL frames with DOPRI5 take the smooth DOPRI5 integrator, bundles the
  // bundle tracer, as the kernels do (no forward-mode tangent for either)
  const bool bundle = f.bundles != 0;
  const bool dp5 = !bundle && f.intg == KT_DOPRI5 && f.chart == KT_CHART_BL;
  if ((dp5 || bundle) && mode != 0 && tangent_dir >= 0) return 2;
#pragma omp parallel
  {
    SmScratch<6>* sk = new SmScratch<6>;
    SmScratch<4>* sb = new SmScratch<4>;
    SmScratch<12>* sw = bundle ? new SmScratch<12> : nullptr;
#pragma omp for schedule(dynamic, 2)
    for (int64_t i = 0; i < n; ++i) {
      RayResult o;
      double g[kGSlots];
      const bool ks = f.chart == KT_CHART_KS && !force_bl;
      bool done = false;
      if (bundle) {
        if (mode == 0)
          sm_pixel<ChartBLB, false>(f, pix[i], cot, &o, g, nullptr);
        else
          sm_pixel<ChartBLB, true>(f, pix[i], cot, &o, g, sw);
        done = true;
      } else if (mode != 0 && tangent_dir >= 0) {
        if (ks) done = sm_pixel_tangent<ChartKS>(f, pix[i], tangent_dir, cot, &o, g);
        if (!done) sm_pixel_tangent<ChartBL>(f, pix[i], tangent_dir, cot, &o, g);
        done = true;
      } else if (ks)
        done = mode == 0 ? sm_pixel<ChartKS, false>(f, pix[i], cot, &o, g, nullptr)
                         : sm_pixel<ChartKS, true>(f, pix[i], cot, &o, g, sk);
      if (!done) {
        if (dp5) {
          if (mode == 0)
            sm_pixel<ChartBL, false, SmDp5>(f, pix[i], cot, &o, g, nullptr);
          else
            sm_pixel<ChartBL, true, SmDp5>(f, pix[i], cot, &o, g, sb);
        } else if (mode == 0) {
          sm_pixel<ChartBL, false>(f, pix[i], cot, &o, g, nullptr);
        } else {
          sm_pixel<ChartBL, true>(f, pix[i], cot, &o, g, sb);
        }
      }
      outcome[i] = (uint8_t)o.outcome;
      r[i] = o.r;
      red[i] = o.red;
      if (magnif) magnif[i] = o.magnif;
      phi_disk[i] = o.phi_disk;
      th_esc[i] = o.th_esc;
      ph_esc[i] = o.ph_esc;
      steps[i] = o.steps;
      attempts[i] = o.attempts;
      if (mode != 0 && contrib)
        for (int q = 0; q < kGSlots; ++q) contrib[q * n + i] = g[q];
    }
    delete sk;
    delete sb;
    delete sw;
  }
  return 0;
}

extern "C" int hc_smooth_pixels(const kt_frame_desc* d, int64_t n, const uint32_t* pix, int mode,
                                int force_bl, int tangent_dir, const double* cot_g, const double* cot_r,
                                const uint8_t* t_out, const double* t_g, const double* t_r,
                                double w_g, double w_r, uint8_t* outcome, double* r, double* red,
                                double* phi_disk, double* th_esc, double* ph_esc, uint32_t* steps,
                                uint32_t* attempts, double* contrib) {
  return hc_smooth_pixels_m(d, n, pix, mode, force_bl, tangent_dir, cot_g, cot_r, nullptr, t_out, t_g,
                            t_r, nullptr, w_g, w_r, 0.0, outcome, r, red, nullptr, phi_disk, th_esc,
                            ph_esc, steps, attempts, contrib);
}

// The centre-out order's input map (ring_item, kt_internal.h) on the host:
// for every item e of a W x H frame, its pixel p[e] and ring c[e].
extern "C" void hc_ring_items(int W, int H, uint32_t* p, int32_t* c) {
  const RingGeom g = ring_geom(W, H);
  const uint32_t n = (uint32_t)W * (uint32_t)H;
  for (uint32_t e = 0; e < n; ++e) {
    int cc;
    ring_item(g, e, &p[e], &cc);
    c[e] = cc;
  }
}
