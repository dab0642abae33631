// kt_grad.cpp -- kt_vjp and kt_l2_grad (and their pixel-list and
// magnification forms): the discrete adjoint of the smooth tracer behind the
// C ABI (kernels in kt_adjoint.cu).
#include <cuda_runtime.h>
#include <string.h>

#include <string>

#include "../../include/kerrtrace.h"
#include "kt_adjoint.h"
#include "kt_context.h"
#include "kt_frame.h"
#include "kt_internal.h"

using namespace ktc;

namespace {

constexpr double kDeg = 3.141592653589793 / 180.0;

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// One gradient pass: launch, reduce, copy the kGSlots sums to `sums`.
// force_bl: trace every ray in the BL chart; tangent_dir >= 0: forward-mode
// tangent along that parameter instead of the reverse sweep.
kt_status grad_pass(kt_context* ctx, const kt::Frame& f, const kt::OutSoA& out, uint32_t n,
                    const uint32_t* pix, uint32_t n_pix, bool whole, const kt::SmCot& cot,
                    bool force_bl, int tangent_dir, cudaStream_t st, double* sums, float* ms) {
  kt::SmJob job;
  job.cot = cot;
  job.force_bl = force_bl ? 1 : 0;
  job.tangent_dir = tangent_dir;
  job.contrib = ctx->d_grad;
  job.pix = pix;
  job.n_pix = n_pix;
  EventPair ev;
  KT_CUDA(ctx, cudaEventCreate(&ev.a), "event");
  KT_CUDA(ctx, cudaEventCreate(&ev.b), "event");
  KT_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
  KT_CUDA(ctx, cudaEventRecord(ev.a, st), "event");
  // with a pixel list only the listed pixels' contributions are written
  // (a whole frame in centre-out order writes every pixel's)
  if (pix && !whole)
    KT_CUDA(ctx, cudaMemsetAsync(ctx->d_grad, 0, (size_t)n * kt::kGSlots * sizeof(double), st),
            "clear contributions");
  KT_CUDA(ctx, kt::launch_smooth(f, out, n, &job, ctx->d_counters, ctx->d_fb, ctx->device, st),
          "adjoint kernel launch");
  KT_CUDA(ctx, kt::launch_grad_sum(ctx->d_grad, n, ctx->d_gsum + kt::kGSlots, ctx->d_gsum, st),
          "gradient sum");
  KT_CUDA(ctx, cudaEventRecord(ev.b, st), "event");
  KT_CUDA(ctx, cudaMemcpyAsync(sums, ctx->d_gsum, kt::kGSlots * sizeof(double), cudaMemcpyDeviceToHost, st),
          "copy gradient");
  KT_CUDA(ctx, cudaStreamSynchronize(st), "gradient pass");
  KT_CUDA(ctx, cudaEventElapsedTime(ms, ev.a, ev.b), "event time");
  return KT_OK;
}

kt_status grad_run(kt_context* ctx, const kt_frame_desc* desc_in, const uint32_t* pix, int64_t n_pix,
                   const kt::SmCot& cot, const kt_geo_soa* out_soa, uint32_t flags, double* grad,
                   kt_grad_stats* stats, cudaStream_t st, const char* who) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!desc_in || !grad) return fail(ctx, KT_ERR_INVALID_ARGUMENT, std::string(who) + ": NULL pointer");
  if (n_pix < 0 || (n_pix > 0 && !pix) ||
      n_pix > (int64_t)desc_in->width * (int64_t)desc_in->height)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, std::string(who) + ": bad pixel list");
  if (flags & ~KT_GRAD_SKIP_LAMBDA) return fail(ctx, KT_ERR_INVALID_ARGUMENT, std::string(who) + ": unknown flags");
  if (out_soa && !out_complete(out_soa))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, std::string(who) + ": incomplete output SoA");
  kt_frame_desc desc = *desc_in;
  desc.precision = KT_PREC_SMOOTH;
  kt::Frame f;
  kt_status r = kt::prepare_frame(&desc, &f, nullptr, &ctx->err);
  if (r != KT_OK) return r;
  DeviceGuard g(ctx->device);
  const uint64_t n = (uint64_t)desc.width * (uint64_t)desc.height;
  r = ensure(ctx, (void**)&ctx->d_grad, &ctx->grad_cap, n * kt::kGSlots * sizeof(double), "gradient buffer");
  if (r != KT_OK) return r;
  r = ensure(ctx, (void**)&ctx->d_gsum, &ctx->gsum_cap, kt::grad_sum_scratch_doubles() * sizeof(double),
             "gradient sums");
  if (r != KT_OK) return r;
  r = ensure(ctx, (void**)&ctx->d_fb, &ctx->fb_cap, 2 * n * sizeof(uint32_t), "fallback list");
  if (r != KT_OK) return r;
  kt::OutSoA out;
  memset(&out, 0, sizeof out);
  if (out_soa) out = to_out(out_soa);
  // a whole frame of at least kOrderMinPixels pixels in centre-out order, as
  // kt_trace traces it (the expensive rays by the critical curve first); the
  // contributions are per pixel and summed in pixel order either way.
  // Measured per gradient, row-major against centre-out in 8 x 4 blocks:
  // config 5 48 / 32 ms (the later changes included), the 960x540 bundle
  // frame 559 / 488.
  bool whole = false;
  if (!pix && n >= kt::kOrderMinPixels) {
    const size_t words = (size_t)n + kt::ring_scratch_words((uint32_t)n);
    r = ensure(ctx, (void**)&ctx->d_order, &ctx->order_cap, words * sizeof(uint32_t), "ray order");
    if (r != KT_OK) return r;
    KT_CUDA(ctx, kt::launch_ring_order(desc.width, desc.height, 0, ctx->d_order + n, ctx->d_order, st),
            "ray order");
    pix = ctx->d_order;
    n_pix = (int64_t)n;
    whole = true;
  }
  double s[kt::kGSlots], sl[kt::kGSlots];
  float ms = 0.f, ms_l = 0.f;
  r = grad_pass(ctx, f, out, (uint32_t)n, pix, (uint32_t)n_pix, whole, cot, false, -1, st, s, &ms);
  if (r != KT_OK) return r;
  double lambda = s[kt::kGLambda];
  if (f.chart == KT_CHART_KS) {
    lambda = 0.0;
    if (!(flags & KT_GRAD_SKIP_LAMBDA)) {
      kt::OutSoA none;
      memset(&none, 0, sizeof none);
      // one derivative in the BL chart: forward-mode tangent along Lambda
      r = grad_pass(ctx, f, none, (uint32_t)n, pix, (uint32_t)n_pix, whole, cot, true, kt::kGLambda, st,
                    sl, &ms_l);
      if (r != KT_OK) return r;
      lambda = sl[kt::kGLambda];
    }
  }
  const double th_scale = (desc.flags & KT_FLAG_ANGLES_RADIANS) ? 1.0 : kDeg;
  grad[KT_GRAD_A] = s[kt::kGA];
  grad[KT_GRAD_Q] = s[kt::kGQ];
  grad[KT_GRAD_LAMBDA] = lambda;
  grad[KT_GRAD_THETA] = s[kt::kGTheta] * th_scale;
  grad[KT_GRAD_R_OBS] = s[kt::kGRobs];
  grad[KT_GRAD_DISK_OUT] = 0.0;
  if (stats) {
    memset(stats, 0, sizeof *stats);
    stats->loss = s[kt::kGLoss];
    stats->grad_pixels = (int64_t)s[kt::kGNumGrad];
    stats->bl_pixels = (int64_t)s[kt::kGNumBL];
    stats->unrecorded = (int64_t)s[kt::kGNumUnrecorded];
    stats->ms_main = ms;
    stats->ms_lambda = ms_l;
  }
  return KT_OK;
}

}  // namespace

extern "C" {

kt_status kt_vjp_magnif(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                        int64_t n_pix, const double* cot_redshift, const double* cot_r,
                        const double* cot_magnif, const kt_geo_soa* out, uint32_t flags,
                        double* grad, kt_grad_stats* stats, void* stream) {
  kt::SmCot cot;
  memset(&cot, 0, sizeof cot);
  cot.mode = 1;
  cot.g = cot_redshift;
  cot.r = cot_r;
  cot.m = cot_magnif;
  return grad_run(ctx, desc, pix_dev, n_pix, cot, out, flags, grad, stats, (cudaStream_t)stream,
                  "kt_vjp");
}

kt_status kt_vjp_pixels(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                        int64_t n_pix, const double* cot_redshift, const double* cot_r,
                        const kt_geo_soa* out, uint32_t flags, double* grad, kt_grad_stats* stats,
                        void* stream) {
  return kt_vjp_magnif(ctx, desc, pix_dev, n_pix, cot_redshift, cot_r, nullptr, out, flags, grad,
                       stats, stream);
}

kt_status kt_vjp(kt_context* ctx, const kt_frame_desc* desc, const double* cot_redshift,
                 const double* cot_r, const kt_geo_soa* out, uint32_t flags, double* grad,
                 kt_grad_stats* stats, void* stream) {
  return kt_vjp_pixels(ctx, desc, nullptr, 0, cot_redshift, cot_r, out, flags, grad, stats, stream);
}

kt_status kt_l2_grad(kt_context* ctx, const kt_frame_desc* desc, const kt_geo_soa* target, double w_g,
                     double w_r, const kt_geo_soa* out, uint32_t flags, double* loss, double* grad,
                     kt_grad_stats* stats, void* stream) {
  return kt_l2_grad_pixels(ctx, desc, nullptr, 0, target, w_g, w_r, out, flags, loss, grad, stats,
                           stream);
}

kt_status kt_l2_grad_pixels(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                            int64_t n_pix, const kt_geo_soa* target, double w_g, double w_r,
                            const kt_geo_soa* out, uint32_t flags, double* loss, double* grad,
                            kt_grad_stats* stats, void* stream) {
  return kt_l2_grad_magnif(ctx, desc, pix_dev, n_pix, target, w_g, w_r, 0.0, out, flags, loss, grad,
                           stats, stream);
}

kt_status kt_l2_grad_magnif(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                            int64_t n_pix, const kt_geo_soa* target, double w_g, double w_r,
                            double w_m, const kt_geo_soa* out, uint32_t flags, double* loss,
                            double* grad, kt_grad_stats* stats, void* stream) {
  if (!ctx) return KT_ERR_INVALID_ARGUMENT;
  if (!target || !target->outcome || !target->redshift || !target->r || !loss ||
      (w_m != 0.0 && !target->magnif))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_l2_grad: NULL pointer");
  if (!kt::finite(w_g) || !kt::finite(w_r) || !kt::finite(w_m))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_l2_grad: non-finite weight");
  kt::SmCot cot;
  memset(&cot, 0, sizeof cot);
  cot.mode = 2;
  cot.t_out = target->outcome;
  cot.t_g = target->redshift;
  cot.t_r = target->r;
  cot.w_g = w_g;
  cot.w_r = w_r;
  cot.t_m = w_m != 0.0 ? target->magnif : nullptr;
  cot.w_m = w_m;
  kt_grad_stats st_local;
  kt_grad_stats* sp = stats ? stats : &st_local;
  const kt_status r = grad_run(ctx, desc, pix_dev, n_pix, cot, out, flags, grad, sp, (cudaStream_t)stream,
                               "kt_l2_grad");
  if (r == KT_OK) *loss = sp->loss;
  return r;
}

}  // extern "C"
