// kt_compat.cpp -- cuda_render (gpu/cuda/tracer.cuh:23-26) over the C ABI.
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kerrtrace.h"
#include "../../include/kerrtrace_cuda_render.h"

namespace {

// One context per calling thread, created by its first call and kept for the
// following ones (the reference calls cuda_render once per frame or camera
// pass, main.cpp:2437): later calls reuse its stream, device buffers and
// frame-shape caches instead of paying the set-up again.  Destroyed when the
// thread exits (for the main thread, before the CUDA runtime's own exit
// handlers run).
struct ThreadContext {
  kt_context* ctx = nullptr;
  ~ThreadContext() {
    if (ctx) kt_destroy(ctx);
  }
};

kt_context* thread_context() {
  thread_local ThreadContext t;
  if (!t.ctx) {
    kt_context* ctx = nullptr;
    const kt_status st = kt_create(&ctx, 0);
    if (st != KT_OK) throw std::runtime_error(std::string("cuda_render: ") + kt_status_string(st));
    t.ctx = ctx;
  }
  return t.ctx;
}

}  // namespace

std::vector<uint32_t> cuda_render(const KNdSParams_CUDA& kp, const CameraParams_CUDA& cp,
                                  bool require_fp64) {
  (void)require_fp64;  // this backend always traces in FP64 on sm_100a
  kt_context* ctx = thread_context();
  kt_status st;
  kt_frame_desc d;
  kt_frame_desc_defaults(&d);
  d.M = kp.M;
  d.a = kp.a;
  d.Q = kp.Q;
  d.Lambda = kp.Lambda;
  d.disk_out = kp.r_disk_out;
  d.r_obs = cp.r_obs;
  d.theta_deg = cp.theta_obs;  // radians, see flags
  d.phi_deg = cp.phi_obs;
  d.fov_deg = cp.fov_h;
  d.flags = KT_FLAG_ANGLES_RADIANS;
  d.width = cp.width;
  d.height = cp.height;
  d.chart = (cp.chart == 1) ? KT_CHART_KS : KT_CHART_BL;
  kt_color_params c;
  kt_color_params_defaults(&c);
  const size_t n = (size_t)(cp.width > 0 ? cp.width : 0) * (size_t)(cp.height > 0 ? cp.height : 0);
  std::vector<uint8_t> rgb(3 * n);
  st = kt_render_host(ctx, &d, &c, nullptr, 0, 0, rgb.data());
  if (st != KT_OK) throw std::runtime_error(std::string("cuda_render: ") + kt_last_error(ctx));
  std::vector<uint32_t> px(n);
  for (size_t i = 0; i < n; ++i)
    px[i] = (0xFFu << 24) | ((uint32_t)rgb[3 * i + 2] << 16) | ((uint32_t)rgb[3 * i + 1] << 8) |
            (uint32_t)rgb[3 * i];
  return px;
}
