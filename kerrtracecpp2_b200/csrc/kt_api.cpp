// kt_api.cpp -- the C ABI (include/kerrtrace.h) over the CUDA kernels.
//
// No exceptions cross the boundary: every entry point returns a kt_status
// and records a message readable with kt_last_error().  There is no CPU
// tracing path: without a CUDA device the trace calls fail with
// KT_ERR_NO_DEVICE.
#include <cmath>
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <new>
#include <string>
#include <vector>

#include "../../include/kerrtrace.h"
#include "kt_adjoint.h"
#include "kt_context.h"
#include "kt_frame.h"
#include "kt_internal.h"

using namespace ktc;

namespace {

kt_status shape(kt_context* ctx, kt::Mode m, kt::LaunchShape* s) {
  if (!ctx->shape_ok[m]) {
    KT_CUDA(ctx, kt::launch_shape(m, ctx->device, &ctx->shapes[m]), "occupancy query");
    ctx->shape_ok[m] = true;
  }
  *s = ctx->shapes[m];
  return KT_OK;
}

// Launch the trace of rl (and, in the KS chart, the BL pass over the rays
// whose KS initialisation failed, main.cpp:1537-1538).
static kt_status run_trace_list(kt_context* ctx, const kt::Frame& f, const kt::OutSoA& out,
                                const kt::RayList& rl, uint64_t n_max, cudaStream_t st);

// A whole frame of at least kOrderMinPixels pixels is traced in centre-out
// order (kt_kernels.cu, launch_ring_order: three small launches on the same
// stream before the trace), each ray written at its own pixel.  Smaller
// frames and pixel lists take the row-major order.
kt_status run_trace(kt_context* ctx, const kt::Frame& f, const kt::OutSoA& out,
                    const kt::RayList& rl, uint64_t n_max, cudaStream_t st) {
  const int W = f.cam.W, H = f.cam.H;
  const uint64_t n = (uint64_t)W * (uint64_t)H;
  if (rl.pix || rl.slot || rl.n_dev || rl.n != n || n < kt::kOrderMinPixels)
    return run_trace_list(ctx, f, out, rl, n_max, st);
  const size_t words = (size_t)n + kt::ring_scratch_words(n);
  kt_status r = ensure(ctx, (void**)&ctx->d_order, &ctx->order_cap, words * sizeof(uint32_t),
                       "ray order");
  if (r != KT_OK) return r;
  KT_CUDA(ctx, kt::launch_ring_order(W, H, 0, ctx->d_order + n, ctx->d_order, st), "ray order");
  if (f.precision == KT_PREC_SMOOTH) {
    // the smooth tracer takes the order as its list of rays
    r = ensure(ctx, (void**)&ctx->d_fb, &ctx->fb_cap, 2 * n_max * sizeof(uint32_t), "fallback list");
    if (r != KT_OK) return r;
    KT_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
    KT_CUDA(ctx, kt::launch_smooth(f, out, (uint32_t)n, nullptr, ctx->d_counters, ctx->d_fb, ctx->device,
                                   st, ctx->d_order),
            "smooth kernel launch");
    return KT_OK;
  }
  const kt::RayList ord = {ctx->d_order, ctx->d_order, nullptr, (uint32_t)n};
  return run_trace_list(ctx, f, out, ord, n_max, st);
}

static kt_status run_trace_list(kt_context* ctx, const kt::Frame& f, const kt::OutSoA& out,
                                const kt::RayList& rl, uint64_t n_max, cudaStream_t st) {
  if (f.precision == KT_PREC_SMOOTH) {
    if (rl.pix || rl.slot || rl.n_dev)
      return fail(ctx, KT_ERR_UNSUPPORTED, "the smooth tracer traces whole frames only");
    kt_status r = ensure(ctx, (void**)&ctx->d_fb, &ctx->fb_cap, 2 * n_max * sizeof(uint32_t), "fallback list");
    if (r != KT_OK) return r;
    KT_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
    KT_CUDA(ctx, kt::launch_smooth(f, out, rl.n, nullptr, ctx->d_counters, ctx->d_fb, ctx->device, st),
            "smooth kernel launch");
    return KT_OK;
  }
  const kt::Mode m = kt::frame_mode(f);
  kt::LaunchShape s;
  kt_status r = shape(ctx, m, &s);
  if (r != KT_OK) return r;
  KT_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
  kt::Fallback fb = {nullptr, nullptr, ctx->d_counters + 2};
  if (kt::has_fallback(m)) {
    r = ensure(ctx, (void**)&ctx->d_fb, &ctx->fb_cap, 2 * n_max * sizeof(uint32_t), "fallback list");
    if (r != KT_OK) return r;
    fb.pix = ctx->d_fb;
    fb.slot = ctx->d_fb + n_max;
  }
  KT_CUDA(ctx, kt::launch_trace(m, f, out, rl, ctx->d_counters, fb, s, st), "trace kernel launch");
  if (kt::has_fallback(m)) {
    const kt::Mode bm = kt::fallback_mode(f);
    kt::LaunchShape bs;
    r = shape(ctx, bm, &bs);
    if (r != KT_OK) return r;
    kt::RayList fl = {fb.pix, fb.slot, fb.count, 0};
    KT_CUDA(ctx, kt::launch_trace(bm, f, out, fl, ctx->d_counters + 1, fb, bs, st),
            "fallback kernel launch");
  }
  if (f.solver == KT_SOLVER_ELLIPTIC_CLOSED)
    KT_CUDA(ctx, kt::launch_elliptic(f, out, rl, st), "elliptic kernel launch");
  return KT_OK;
}

// The jitter offsets of render_image's camera_spp branch (main.cpp:2238-2279):
// spp = 2 splits horizontally; otherwise the centre for odd spp, then +/-
// pairs from a fixed table, then +/- pairs on a golden-angle spiral of
// radius 0.49 sqrt((m + 1) / (spp + 1)).
void spp_offsets(int spp, double* xy) {
  if (spp <= 1) {
    xy[0] = xy[1] = 0.0;
    return;
  }
  if (spp == 2) {
    xy[0] = -0.35; xy[1] = 0.0;
    xy[2] = 0.35; xy[3] = 0.0;
    return;
  }
  static const double kPairs[7][2] = {{0.35, 0.00}, {0.00, 0.35}, {0.25, 0.25}, {0.45, 0.20},
                                      {0.20, 0.45}, {0.40, 0.00}, {0.00, 0.40}};
  int k = 0;
  if (spp % 2 == 1) {
    xy[0] = xy[1] = 0.0;
    k = 1;
  }
  for (int j = 0; j < 7 && k + 2 <= spp; ++j, k += 2) {
    xy[2 * k] = kPairs[j][0];
    xy[2 * k + 1] = kPairs[j][1];
    xy[2 * k + 2] = -kPairs[j][0];
    xy[2 * k + 3] = -kPairs[j][1];
  }
  const double golden = 2.39996322972865332;
  for (int m = 1; k < spp; ++m) {
    const double rad = 0.49 * sqrt((double)m / (double)(spp + 1));
    const double ang = golden * (double)m;
    const double x = rad * ktm_cos(ang), y = rad * ktm_sin(ang);
    xy[2 * k] = x;
    xy[2 * k + 1] = y;
    if (++k < spp) {
      xy[2 * k] = -x;
      xy[2 * k + 1] = -y;
      ++k;
    }
  }
}

}  // namespace

extern "C" {

int kt_abi_version(void) { return KT_ABI_VERSION; }

const char* kt_status_string(kt_status s) {
  switch (s) {
    case KT_OK: return "ok";
    case KT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case KT_ERR_UNSUPPORTED: return "unsupported";
    case KT_ERR_CUDA: return "CUDA error";
    case KT_ERR_OUT_OF_MEMORY: return "out of device memory";
    case KT_ERR_NO_DEVICE: return "no CUDA device";
    case KT_ERR_IO: return "I/O error";
    case KT_ERR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

int kt_abi_struct_sizes(size_t* sizes, int n) {
  const size_t v[7] = {sizeof(kt_frame_desc),    sizeof(kt_frame_derived),
                       sizeof(kt_geo_soa),       sizeof(kt_color_params),
                       sizeof(kt_batch_options), sizeof(kt_batch_group_info),
                       sizeof(kt_grad_stats)};
  int k = 0;
  for (; k < n && k < 7; ++k) sizes[k] = v[k];
  return k;
}

void kt_frame_desc_defaults(kt_frame_desc* d) {
  if (!d) return;
  memset(d, 0, sizeof *d);
  // main.cpp:2505-2517 and 2709-2716
  d->M = 1.0;
  d->a = 0.998;
  d->theta_deg = 80.0;
  d->r_obs = 40.0;
  d->disk_out = 12.0;
  d->fov_deg = 30.0;
  d->width = 1920;
  d->height = 1080;
  d->chart = KT_CHART_KS;
  d->integrator = KT_RK4_DOUBLING;
  d->max_steps = 500000;
  d->step_init = 1.0;
  d->tol = 1e-7;
}

void kt_color_params_defaults(kt_color_params* cp) {
  if (!cp) return;
  memset(cp, 0, sizeof *cp);
  cp->exposure = 1.0;
  cp->gamma = 2.2;
  cp->temp_scale = 1.0;
  // ColorParams' defaults (main.cpp:76-80)
  cp->disk_rings = 7;
  cp->disk_sectors = 14;
  cp->disk_sigma = 0.5;
  cp->disk_hue_offset = 0.0;
}

kt_status kt_frame_derive(const kt_frame_desc* desc, kt_frame_derived* out) {
  if (!out) return KT_ERR_INVALID_ARGUMENT;
  kt::Frame f;
  std::string err;
  return kt::prepare_frame(desc, &f, out, &err);
}

kt_status kt_create(kt_context** pctx, int device) {
  if (!pctx) return KT_ERR_INVALID_ARGUMENT;
  *pctx = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return KT_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return KT_ERR_INVALID_ARGUMENT;
  kt_context* ctx = new (std::nothrow) kt_context();
  if (!ctx) return KT_ERR_OUT_OF_MEMORY;
  ctx->device = device;
  DeviceGuard g(device);
  if (!g.ok) {
    delete ctx;
    return KT_ERR_NO_DEVICE;
  }
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
  if (major != 10) {
    delete ctx;
    return KT_ERR_UNSUPPORTED;  // kernels are built for sm_100a only
  }
  if (cudaMalloc((void**)&ctx->d_counters, 4 * sizeof(uint32_t)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    kt_destroy(ctx);
    return KT_ERR_OUT_OF_MEMORY;
  }
  *pctx = ctx;
  return KT_OK;
}

void kt_destroy(kt_context* ctx) {
  if (!ctx) return;
  DeviceGuard g(ctx->device);
  if (ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  cudaFree(ctx->d_counters);
  cudaFree(ctx->d_fb);
  cudaFree(ctx->d_stage);
  cudaFree(ctx->d_order);
  cudaFree(ctx->d_bg);
  cudaFree(ctx->d_grad);
  cudaFree(ctx->d_gsum);
  delete ctx;
}

const char* kt_last_error(const kt_context* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

kt_status kt_trace(kt_context* ctx, const kt_frame_desc* desc, const kt_geo_soa* out,
                   void* stream) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!out_complete(out)) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_trace: output pointer is NULL");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const uint64_t n = (uint64_t)desc->width * (uint64_t)desc->height;
  kt::RayList rl = {nullptr, nullptr, nullptr, (uint32_t)n};
  return run_trace(ctx, f, to_out(out), rl, n, (cudaStream_t)stream);
}

kt_status kt_trace_pixels(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                          int64_t n, const kt_geo_soa* out, void* stream) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (n < 0 || n > 0x7fffffff) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_trace_pixels: bad n");
  if (n > 0 && (!pix_dev || !out_complete(out)))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_trace_pixels: NULL pointer");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  if (n == 0) return KT_OK;
  DeviceGuard g(ctx->device);
  kt::RayList rl = {pix_dev, nullptr, nullptr, (uint32_t)n};
  return run_trace(ctx, f, to_out(out), rl, (uint64_t)n, (cudaStream_t)stream);
}

// The device address of a page-locked host buffer mapped into `device`'s
// address space (cudaHostAlloc, or cudaHostRegister'd memory), else nullptr.
static void* mapped_host_ptr(void* p, int device) {
  if (!p) return nullptr;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return (a.type == cudaMemoryTypeHost && a.device == device) ? a.devicePointer : nullptr;
}

kt_status kt_trace_host(kt_context* ctx, const kt_frame_desc* desc, const kt_geo_soa* out_host) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!out_complete(out_host)) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_trace_host: NULL output");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const size_t n = (size_t)desc->width * (size_t)desc->height;
  // Page-locked, mapped host buffers: the kernels write every ray's record
  // straight into them, so the transfer overlaps the trace.  Otherwise the
  // records go to a device staging area and are copied after the trace.
  {
    kt_geo_soa m = *out_host;
    void** fields[] = {(void**)&m.outcome, (void**)&m.r, (void**)&m.redshift, (void**)&m.magnif,
                       (void**)&m.phi_disk, (void**)&m.theta_esc, (void**)&m.phi_esc,
                       (void**)&m.status, (void**)&m.steps, (void**)&m.attempts};
    bool direct = true;
    for (void** fp : fields) {
      if (!*fp) continue;
      void* dp = mapped_host_ptr(*fp, ctx->device);
      if (!dp) {
        direct = false;
        break;
      }
      *fp = dp;
    }
    if (direct) {
      kt::RayList rl = {nullptr, nullptr, nullptr, (uint32_t)n};
      r = run_trace(ctx, f, to_out(&m), rl, n, ctx->stream);
      if (r != KT_OK) return r;
      KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "trace");
      return KT_OK;
    }
  }
  // 6 float64 arrays, attempts, steps, outcome, status
  const size_t need = n * (6 * 8 + 4 + 4 + 1 + 1) + 256;
  r = ensure(ctx, (void**)&ctx->d_stage, &ctx->stage_cap, need, "staging buffer");
  if (r != KT_OK) return r;
  unsigned char* p = ctx->d_stage;
  kt_geo_soa d;
  d.r = (double*)p; p += 8 * n;
  d.redshift = (double*)p; p += 8 * n;
  d.magnif = (double*)p; p += 8 * n;
  d.phi_disk = (double*)p; p += 8 * n;
  d.theta_esc = (double*)p; p += 8 * n;
  d.phi_esc = (double*)p; p += 8 * n;
  d.steps = (uint32_t*)p; p += 4 * n;
  d.attempts = (uint32_t*)p; p += 4 * n;
  d.outcome = p; p += n;
  d.status = p;
  if (!out_host->status) d.status = nullptr;
  if (!out_host->steps) d.steps = nullptr;
  if (!out_host->attempts) d.attempts = nullptr;
  kt::RayList rl = {nullptr, nullptr, nullptr, (uint32_t)n};
  r = run_trace(ctx, f, to_out(&d), rl, n, ctx->stream);
  if (r != KT_OK) return r;
  struct { void* dst; const void* src; size_t bytes; } cp[] = {
      {out_host->outcome, d.outcome, n}, {out_host->r, d.r, 8 * n},
      {out_host->redshift, d.redshift, 8 * n}, {out_host->magnif, d.magnif, 8 * n},
      {out_host->phi_disk, d.phi_disk, 8 * n}, {out_host->theta_esc, d.theta_esc, 8 * n},
      {out_host->phi_esc, d.phi_esc, 8 * n}, {out_host->status, d.status, n},
      {out_host->steps, d.steps, 4 * n}, {out_host->attempts, d.attempts, 4 * n}};
  for (auto& c : cp)
    if (c.dst && c.src)
      KT_CUDA(ctx, cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, ctx->stream),
              "copy results to host");
  KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "trace");
  return KT_OK;
}

kt_status kt_colorize(kt_context* ctx, const kt_frame_desc* desc, const kt_geo_soa* geo,
                      const kt_color_params* cp, const uint8_t* bg_rgb, int32_t bg_w,
                      int32_t bg_h, uint8_t* rgb_out, void* stream) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!geo || !geo->outcome || !geo->r || !geo->redshift || !geo->magnif || !geo->theta_esc ||
      !geo->phi_esc || !cp || !rgb_out)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize: NULL pointer");
  if (bg_rgb && (bg_w < 1 || bg_h < 1))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize: background size must be >= 1");
  if (cp->palette != 0 && cp->palette != 1)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize: palette must be 0 (blackbody) or 1 (interstellar)");
  if (cp->palette == 1 && !geo->phi_disk)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize: the interstellar palette needs phi_disk");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const kt::ColourConst cc = kt::make_colour(f, *cp);
  const int64_t n = (int64_t)desc->width * desc->height;
  KT_CUDA(ctx, kt::launch_colorize(cc, n, geo->outcome, geo->r, geo->redshift, geo->magnif,
                                   geo->phi_disk, geo->theta_esc, geo->phi_esc, bg_rgb, bg_w, bg_h,
                                   rgb_out,
                                   (cudaStream_t)stream),
          "colorize kernel launch");
  return KT_OK;
}

kt_status kt_render_host(kt_context* ctx, const kt_frame_desc* desc, const kt_color_params* cp,
                         const uint8_t* bg_rgb_host, int32_t bg_w, int32_t bg_h,
                         uint8_t* rgb_out_host) {
  return kt_render_spp_host(ctx, desc, cp, 1, bg_rgb_host, bg_w, bg_h, rgb_out_host);
}

kt_status kt_render_spp_host(kt_context* ctx, const kt_frame_desc* desc, const kt_color_params* cp,
                             int32_t camera_spp, const uint8_t* bg_rgb_host, int32_t bg_w,
                             int32_t bg_h, uint8_t* rgb_out_host) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!desc || !cp || !rgb_out_host) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_render_host: NULL pointer");
  if (bg_rgb_host && (bg_w < 1 || bg_h < 1))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_render_host: background size must be >= 1");
  if (cp->palette != 0 && cp->palette != 1)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_render_host: palette must be 0 or 1");
  const int spp = camera_spp < 1 ? 1 : camera_spp;
  if (spp > KT_MAX_CAMERA_SPP)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_render_spp_host: camera_spp above KT_MAX_CAMERA_SPP");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const size_t n = (size_t)desc->width * (size_t)desc->height;
  const uint8_t* d_bg = nullptr;
  if (bg_rgb_host) {
    const size_t bb = (size_t)bg_w * (size_t)bg_h * 3;
    r = ensure(ctx, (void**)&ctx->d_bg, &ctx->bg_cap, bb, "background buffer");
    if (r != KT_OK) return r;
    KT_CUDA(ctx, cudaMemcpyAsync(ctx->d_bg, bg_rgb_host, bb, cudaMemcpyHostToDevice, ctx->stream),
            "copy background");
    d_bg = ctx->d_bg;
  }
  const kt::ColourConst cc = kt::make_colour(f, *cp);
  if (spp == 1) {
    // render_image (main.cpp:2209-2478): trace + colorize
    const size_t need = n * (6 * 8 + 1 + 3) + 256;
    r = ensure(ctx, (void**)&ctx->d_stage, &ctx->stage_cap, need, "staging buffer");
    if (r != KT_OK) return r;
    unsigned char* p = ctx->d_stage;
    kt_geo_soa d;
    memset(&d, 0, sizeof d);
    d.r = (double*)p; p += 8 * n;
    d.redshift = (double*)p; p += 8 * n;
    d.magnif = (double*)p; p += 8 * n;
    d.phi_disk = (double*)p; p += 8 * n;
    d.theta_esc = (double*)p; p += 8 * n;
    d.phi_esc = (double*)p; p += 8 * n;
    d.outcome = p; p += n;
    uint8_t* d_rgb = p;
    kt::RayList rl = {nullptr, nullptr, nullptr, (uint32_t)n};
    r = run_trace(ctx, f, to_out(&d), rl, n, ctx->stream);
    if (r != KT_OK) return r;
    KT_CUDA(ctx, kt::launch_colorize(cc, (int64_t)n, d.outcome, d.r, d.redshift, d.magnif, d.phi_disk,
                                     d.theta_esc, d.phi_esc, d_bg, bg_w, bg_h, d_rgb, ctx->stream),
            "colorize kernel launch");
    KT_CUDA(ctx, cudaMemcpyAsync(rgb_out_host, d_rgb, 3 * n, cudaMemcpyDeviceToHost, ctx->stream),
            "copy image to host");
    KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "render");
    return KT_OK;
  }
  // camera_spp > 1 (main.cpp:2232-2322): every pass is a full render at the
  // frame's pixel offset plus the pass's jitter.  The passes differ only in
  // their camera, so they share one kernel mode: one batch launch traces all
  // of them (lanes refill across pass boundaries), one kernel colours them
  // and averages in linear light.
  if (f.precision == KT_PREC_SMOOTH)
    return fail(ctx, KT_ERR_UNSUPPORTED, "kt_render_spp_host: the smooth tracer renders one pass");
  if ((uint64_t)n * (uint64_t)spp > 0x7fffffffULL)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_render_spp_host: more than 2^31 rays");
  double offs[2 * KT_MAX_CAMERA_SPP];
  spp_offsets(spp, offs);
  std::vector<kt::Frame> frames((size_t)spp);
  for (int s = 0; s < spp; ++s) {
    kt_frame_desc ds = *desc;
    ds.pixel_offset_x = desc->pixel_offset_x + offs[2 * s];
    ds.pixel_offset_y = desc->pixel_offset_y + offs[2 * s + 1];
    r = kt::prepare_frame(&ds, &frames[(size_t)s], nullptr, &ctx->err);
    if (r != KT_OK) return r;
  }
  const kt::Mode m = kt::frame_mode(f);
  // staging: Frame[spp] | OutSoA[spp] | offsets[spp + 1] | 6 f64 fields
  // [spp][n] | outcome [spp][n] | rgb [3n]
  auto a256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t nt = n * (size_t)spp;
  const size_t off_outs = a256(spp * sizeof(kt::Frame));
  const size_t off_offs = off_outs + a256(spp * sizeof(kt::OutSoA));
  const size_t off_f64 = off_offs + a256((spp + 1) * sizeof(uint64_t));
  const size_t off_oc = off_f64 + a256(6 * 8 * nt);
  const size_t off_rgb = off_oc + a256(nt);
  r = ensure(ctx, (void**)&ctx->d_stage, &ctx->stage_cap, off_rgb + 3 * n + 256, "staging buffer");
  if (r != KT_OK) return r;
  if (kt::has_fallback(m)) {
    r = ensure(ctx, (void**)&ctx->d_fb, &ctx->fb_cap, nt * sizeof(uint32_t), "fallback list");
    if (r != KT_OK) return r;
  }
  unsigned char* base = ctx->d_stage;
  double* f64 = (double*)(base + off_f64);
  uint8_t* oc = base + off_oc;
  uint8_t* d_rgb = base + off_rgb;
  kt::SppPasses P = {oc, f64, f64 + nt, f64 + 2 * nt, f64 + 3 * nt, f64 + 4 * nt, f64 + 5 * nt};
  std::vector<kt::OutSoA> outs((size_t)spp);
  std::vector<uint64_t> offsets((size_t)spp + 1);
  for (int s = 0; s < spp; ++s) {
    const size_t o = (size_t)s * n;
    outs[(size_t)s] = kt::OutSoA{oc + o, f64 + o, f64 + nt + o, f64 + 2 * nt + o, f64 + 3 * nt + o,
                                 f64 + 4 * nt + o, f64 + 5 * nt + o, nullptr, nullptr, nullptr};
    offsets[(size_t)s] = o;
  }
  offsets[(size_t)spp] = nt;
  KT_CUDA(ctx, cudaMemcpyAsync(base, frames.data(), spp * sizeof(kt::Frame), cudaMemcpyHostToDevice,
                               ctx->stream), "pass frames");
  KT_CUDA(ctx, cudaMemcpyAsync(base + off_outs, outs.data(), spp * sizeof(kt::OutSoA),
                               cudaMemcpyHostToDevice, ctx->stream), "pass outputs");
  KT_CUDA(ctx, cudaMemcpyAsync(base + off_offs, offsets.data(), (spp + 1) * sizeof(uint64_t),
                               cudaMemcpyHostToDevice, ctx->stream), "pass offsets");
  kt::BatchRays br;
  br.frames = (const kt::Frame*)base;
  br.outs = (const kt::OutSoA*)(base + off_outs);
  br.offsets = (const uint64_t*)(base + off_offs);
  br.n_frames = spp;
  br.refill_min = 1;
  br.list = nullptr;
  br.n_dev = nullptr;
  br.n = nt;
  br.fp32 = std::isfinite(f.r_fp32);
  // the single-frame launch shapes: 64 x 9 for the exact BL kernels, 128 x 1 otherwise
  auto variant = [](kt::Mode md) { return (md == kt::kModeBLRk4 || md == kt::kModeBLDopri5) ? 0 : 1; };
  kt::LaunchShape ls;
  KT_CUDA(ctx, kt::batch_shape(m, variant(m), ctx->device, &ls), "occupancy query");
  KT_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), ctx->stream), "reset queue");
  const kt::Fallback fb = {kt::has_fallback(m) ? ctx->d_fb : nullptr, nullptr, ctx->d_counters + 2};
  KT_CUDA(ctx, kt::launch_batch(m, variant(m), br, ctx->d_counters, fb, ls, ctx->stream),
          "trace kernel launch");
  if (kt::has_fallback(m)) {
    const kt::Mode bm = kt::fallback_mode(f);
    kt::LaunchShape bs;
    KT_CUDA(ctx, kt::batch_shape(bm, variant(bm), ctx->device, &bs), "occupancy query");
    kt::BatchRays fl = br;
    fl.list = ctx->d_fb;
    fl.n_dev = ctx->d_counters + 2;
    fl.n = 0;
    KT_CUDA(ctx, kt::launch_batch(bm, variant(bm), fl, ctx->d_counters + 1, fb, bs, ctx->stream),
            "fallback kernel launch");
  }
  if (f.solver == KT_SOLVER_ELLIPTIC_CLOSED) {
    const kt::RayList all = {nullptr, nullptr, nullptr, (uint32_t)n};
    for (int s = 0; s < spp; ++s)
      KT_CUDA(ctx, kt::launch_elliptic(frames[(size_t)s], outs[(size_t)s], all, ctx->stream),
              "elliptic kernel launch");
  }
  const double gamma_eff = cp->gamma < 1e-6 ? 1e-6 : cp->gamma;
  KT_CUDA(ctx, kt::launch_spp_colorize(cc, (int64_t)n, spp, P, d_bg, bg_w, bg_h, gamma_eff, d_rgb,
                                       ctx->stream), "supersample colour launch");
  KT_CUDA(ctx, cudaMemcpyAsync(rgb_out_host, d_rgb, 3 * n, cudaMemcpyDeviceToHost, ctx->stream),
          "copy image to host");
  KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "render");
  return KT_OK;
}

kt_status kt_elliptic_reasons(kt_context* ctx, const kt_frame_desc* desc, uint8_t* reason,
                              void* stream) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!desc || !reason) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_elliptic_reasons: NULL pointer");
  kt::Frame f;
  kt_status r = kt::prepare_frame(desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const uint32_t n = (uint32_t)((int64_t)desc->width * desc->height);
  const cudaStream_t st = (cudaStream_t)stream;
  if (f.solver != KT_SOLVER_ELLIPTIC_CLOSED || f.bundles) {
    KT_CUDA(ctx, cudaMemsetAsync(reason, 0, n, st), "clear reasons");  // the tag stays 0
    return KT_OK;
  }
  KT_CUDA(ctx, kt::launch_elliptic_reasons(f, n, reason, st), "elliptic reasons launch");
  return KT_OK;
}

kt_status kt_elliptic_reasons_host(kt_context* ctx, const kt_frame_desc* desc, uint8_t* reason_host) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!desc || !reason_host) return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_elliptic_reasons_host: NULL pointer");
  if (desc->width < 1 || desc->height < 1)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_elliptic_reasons_host: bad frame size");
  DeviceGuard g(ctx->device);
  const size_t n = (size_t)desc->width * (size_t)desc->height;
  kt_status r = ensure(ctx, (void**)&ctx->d_stage, &ctx->stage_cap, n + 256, "staging buffer");
  if (r != KT_OK) return r;
  r = kt_elliptic_reasons(ctx, desc, ctx->d_stage, ctx->stream);
  if (r != KT_OK) return r;
  KT_CUDA(ctx, cudaMemcpyAsync(reason_host, ctx->d_stage, n, cudaMemcpyDeviceToHost, ctx->stream),
          "copy reasons to host");
  KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "elliptic reasons");
  return KT_OK;
}

kt_status kt_camera_spp_offsets(int32_t camera_spp, double* xy) {
  if (!xy || camera_spp > KT_MAX_CAMERA_SPP) return KT_ERR_INVALID_ARGUMENT;
  spp_offsets(camera_spp < 1 ? 1 : camera_spp, xy);
  return KT_OK;
}

kt_status kt_colorize_host(kt_context* ctx, const kt_geo_soa* g, int32_t width, int32_t height,
                           double M, double r_isco, double r_disk_in, double r_disk_out,
                           const kt_color_params* cp, const uint8_t* bg_rgb_host, int32_t bg_w,
                           int32_t bg_h, uint8_t* rgb_out_host) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!g || !g->outcome || !g->r || !g->redshift || !g->magnif || !g->theta_esc || !g->phi_esc ||
      !cp || !rgb_out_host)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize_host: NULL pointer");
  if (width < 1 || height < 1 || (int64_t)width * height > 0x7fffffff)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize_host: bad frame size");
  if (bg_rgb_host && (bg_w < 1 || bg_h < 1))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize_host: background size must be >= 1");
  if (cp->palette != 0 && cp->palette != 1)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize_host: palette must be 0 or 1");
  if (cp->palette == 1 && !g->phi_disk)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_colorize_host: the interstellar palette needs phi_disk");
  DeviceGuard guard(ctx->device);
  const size_t n = (size_t)width * (size_t)height;
  const size_t need = n * (6 * 8 + 1 + 3) + 256;
  kt_status r = ensure(ctx, (void**)&ctx->d_stage, &ctx->stage_cap, need, "staging buffer");
  if (r != KT_OK) return r;
  unsigned char* p = ctx->d_stage;
  double* d_r = (double*)p; p += 8 * n;
  double* d_red = (double*)p; p += 8 * n;
  double* d_mag = (double*)p; p += 8 * n;
  double* d_th = (double*)p; p += 8 * n;
  double* d_ph = (double*)p; p += 8 * n;
  double* d_pd = (double*)p; p += 8 * n;
  uint8_t* d_out = p; p += n;
  uint8_t* d_rgb = p;
  const struct { void* dst; const void* src; size_t bytes; } cps[] = {
      {d_r, g->r, 8 * n}, {d_red, g->redshift, 8 * n}, {d_mag, g->magnif, 8 * n},
      {d_th, g->theta_esc, 8 * n}, {d_ph, g->phi_esc, 8 * n}, {d_out, g->outcome, n},
      {d_pd, g->phi_disk, 8 * n}};
  for (const auto& c : cps)
    if (c.src)
      KT_CUDA(ctx, cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyHostToDevice, ctx->stream),
              "copy in");
  const uint8_t* d_bg = nullptr;
  if (bg_rgb_host) {
    const size_t bb = (size_t)bg_w * (size_t)bg_h * 3;
    r = ensure(ctx, (void**)&ctx->d_bg, &ctx->bg_cap, bb, "background buffer");
    if (r != KT_OK) return r;
    KT_CUDA(ctx, cudaMemcpyAsync(ctx->d_bg, bg_rgb_host, bb, cudaMemcpyHostToDevice, ctx->stream),
            "copy background");
    d_bg = ctx->d_bg;
  }
  kt::ColourConst cc;
  cc.M = M;
  cc.r_isco = r_isco;
  cc.exposure = cp->exposure;
  cc.gamma = cp->gamma;
  cc.temp_scale = cp->temp_scale;
  cc.log10_50 = ktm_log10(4e4 / 800.0);
  cc.pt_peak = kt::page_thorne(3.0 * r_isco, r_isco);
  cc.palette = cp->palette;
  cc.rings = cp->disk_rings;
  cc.sectors = cp->disk_sectors;
  cc.pad0 = 0;
  cc.sigma = cp->disk_sigma;
  cc.hue_offset = cp->disk_hue_offset;
  cc.r_in = r_disk_in;
  cc.r_out = r_disk_out;
  KT_CUDA(ctx, kt::launch_colorize(cc, (int64_t)n, d_out, d_r, d_red, d_mag, d_pd, d_th, d_ph, d_bg,
                                   bg_w, bg_h, d_rgb, ctx->stream),
          "colorize kernel launch");
  KT_CUDA(ctx, cudaMemcpyAsync(rgb_out_host, d_rgb, 3 * n, cudaMemcpyDeviceToHost, ctx->stream),
          "copy image to host");
  KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "colorize");
  return KT_OK;
}

kt_status kt_measure_fp64_peak(kt_context* ctx, double* gflops) {
  if (!ctx || !gflops) return KT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(ctx->device);
  int sms = 0;
  KT_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "attr");
  const int block = 256, grid = sms * 8, n_iter = 4096;
  double* d_sink = nullptr;
  KT_CUDA(ctx, cudaMalloc((void**)&d_sink, grid * sizeof(double)), "probe buffer");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best_ms = 1e30f;
  cudaError_t err = cudaSuccess;
  for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    err = kt::launch_fp64_probe(d_sink, n_iter, grid, block, ctx->stream);
    cudaEventRecord(e1, ctx->stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (err == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && rep > 0 && ms < best_ms)
      best_ms = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_sink);
  if (err != cudaSuccess) return cuda_fail(ctx, err, "FP64 probe");
  const double fmas = (double)grid * block * n_iter * 8.0;
  *gflops = 2.0 * fmas / (best_ms * 1e-3) / 1e9;
  return KT_OK;
}

kt_status kt_measure_op_costs(kt_context* ctx, kt_op_costs* out) {
  if (!ctx || !out) return KT_ERR_INVALID_ARGUMENT;
  DeviceGuard g(ctx->device);
  int sms = 0;
  KT_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device), "attr");
  const int block = 256, grid = sms * 8;
  // iterations per op (about a millisecond each) and the FMA-pipe operations
  // each recurrence step adds to the measured one
  const int n_iter[6] = {4096, 512, 512, 512, 64, 32};
  const double extra[6] = {0.0, 0.0, 1.0, 1.0, 2.0, 1.0};
  double* d_sink = nullptr;
  KT_CUDA(ctx, cudaMalloc((void**)&d_sink, grid * sizeof(double)), "probe buffer");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double per_iter_ms[6];
  cudaError_t err = cudaSuccess;
  for (int op = 0; op < 6 && err == cudaSuccess; ++op) {
    float best_ms = 1e30f;
    for (int rep = 0; rep < 4 && err == cudaSuccess; ++rep) {
      cudaEventRecord(e0, ctx->stream);
      err = kt::launch_op_probe(op, d_sink, n_iter[op], grid, block, ctx->stream);
      cudaEventRecord(e1, ctx->stream);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && rep > 0 &&
          ms < best_ms)
        best_ms = ms;
    }
    per_iter_ms[op] = best_ms / n_iter[op];
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_sink);
  if (err != cudaSuccess) return cuda_fail(ctx, err, "operation-cost probe");
  double c[6];
  for (int op = 0; op < 6; ++op) c[op] = 2.0 * (per_iter_ms[op] / per_iter_ms[0] - extra[op]);
  out->fma_gflops = 2.0 * (double)grid * block * 8.0 / (per_iter_ms[0] * 1e-3) / 1e9;
  out->div = c[1];
  out->div3 = c[2];
  out->sqrt = c[3];
  out->sincos = c[4];
  out->pow = c[5];
  return KT_OK;
}

}  // extern "C"
