// kt_noalloc.cu -- kt_trace_noalloc: trace one frame without allocating.
//
// Who needs this: a caller that is not allowed to call the CUDA allocator at
// all -- a host application that owns every byte of device memory and hands
// the renderer only its input and output buffers (an engine or a render
// service that budgets memory up front), or a frame loop that cannot afford
// cudaMalloc/cudaFree, which may synchronize the whole device.  Such a
// caller cannot create a kt_context either, because kt_create allocates the
// context's scratch.  This entry point needs no context.
//
// The scratch the trace kernels need -- the ray-queue counters, in the KS
// chart the list of rays handed back to the BL chart, and for whole frames
// of at least 2^16 pixels the centre-out ray order that kt_trace uses (the
// list and its counting-sort scratch) -- lives in one file-scope device array
// below, sized for frames of at most KT_NOALLOC_MAX_PIXELS pixels
// (12.5 MiB + 256 bytes).  Every GPU that loads the library holds that array
// until the process exits.  Larger frames are rejected with
// KT_ERR_INVALID_ARGUMENT.
//
// All calls share the one array: each call clears the counters on its
// stream before its kernels run, so calls that are ordered on the device
// (one stream, or synchronized streams) are independent; calls that overlap
// on the device race on the counters and give wrong results.
//
// The first call on a device resolves the array's device address for that
// device (cudaGetSymbolAddress with the device current); make that first
// call before any stream capture on the device.
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "../../include/kerrtrace.h"
#include "kt_frame.h"
#include "kt_internal.h"

namespace {

constexpr size_t kCounterBytes = 256;  // queue counters, padded to the alignment
// centre-out order: the ray list (one word per pixel) and the counting sort's scratch
constexpr size_t kOrderWords =
    KT_NOALLOC_MAX_PIXELS + kt::ring_scratch_words(KT_NOALLOC_MAX_PIXELS);
constexpr size_t kScratchBytes =
    kCounterBytes + (2ull * KT_NOALLOC_MAX_PIXELS + kOrderWords) * sizeof(uint32_t);

// The scratch.  In host code `g_noalloc_scratch` only names the symbol; its
// device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::atomic<unsigned char*> g_scratch_addr[kMaxDevices];
// Launch shapes per (device, mode): state 0 empty, 1 being written by the one
// thread that claimed it, 2 ready to read.
std::atomic<int> g_shape_state[kMaxDevices][kt::kNumModes];
kt::LaunchShape g_shapes[kMaxDevices][kt::kNumModes];

kt_status cuda_status(cudaError_t e) {
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return KT_ERR_NO_DEVICE;
  return KT_ERR_CUDA;
}

// The checks prepare_frame makes, without building a message string (a
// message would allocate on the host), plus the scratch-size limit.
kt_status validate(const kt_frame_desc* d) {
  if (!d) return KT_ERR_INVALID_ARGUMENT;
  if (d->width < 1 || d->height < 1) return KT_ERR_INVALID_ARGUMENT;
  if ((int64_t)d->width * (int64_t)d->height > (int64_t)KT_NOALLOC_MAX_PIXELS)
    return KT_ERR_INVALID_ARGUMENT;
  const double v[] = {d->M, d->a, d->Q, d->Lambda, d->theta_deg, d->phi_deg, d->r_obs,
                      d->disk_out, d->fov_deg, d->pixel_offset_x, d->pixel_offset_y,
                      d->step_init, d->tol};
  for (double x : v)
    if (!kt::finite(x)) return KT_ERR_INVALID_ARGUMENT;
  if ((d->chart != KT_CHART_KS && d->chart != KT_CHART_BL) ||
      (d->integrator != KT_RK4_DOUBLING && d->integrator != KT_DOPRI5) ||
      (d->bundles != 0 && d->bundles != 1) ||
      (d->flags & ~(uint32_t)KT_FLAG_ANGLES_RADIANS) != 0 || !(d->r_obs > 0.0) || !(d->M > 0.0))
    return KT_ERR_INVALID_ARGUMENT;
  if (d->solver_mode != KT_SOLVER_STANDARD || d->precision != KT_PREC_FP64)
    return KT_ERR_UNSUPPORTED;
  return KT_OK;
}

kt::Mode mode_of(const kt::Frame& f) {
  if (f.bundles) return kt::kModeBundle;
  if (f.chart == KT_CHART_KS) return kt::kModeKSRk4;
  return f.intg == KT_DOPRI5 ? kt::kModeBLDopri5 : kt::kModeBLRk4;
}

kt_status shape(int dev, kt::Mode m, kt::LaunchShape* s) {
  if (g_shape_state[dev][m].load(std::memory_order_acquire) == 2) {
    *s = g_shapes[dev][m];
    return KT_OK;
  }
  kt::LaunchShape t;
  const cudaError_t e = kt::launch_shape(m, dev, &t);
  if (e != cudaSuccess) return cuda_status(e);
  // Publish it once: only the thread that moves the state from 0 to 1 writes
  // the cache; a thread that finds another writing uses its own copy.
  int expect = 0;
  if (g_shape_state[dev][m].compare_exchange_strong(expect, 1, std::memory_order_acq_rel)) {
    g_shapes[dev][m] = t;
    g_shape_state[dev][m].store(2, std::memory_order_release);
  }
  *s = t;
  return KT_OK;
}

}  // namespace

extern "C" kt_status kt_trace_noalloc(const kt_frame_desc* desc, const kt_geo_soa* out,
                                      void* stream) {
  kt_status st = validate(desc);
  if (st != KT_OK) return st;
  if (!out || !out->outcome || !out->r || !out->redshift || !out->magnif || !out->phi_disk ||
      !out->theta_esc || !out->phi_esc)
    return KT_ERR_INVALID_ARGUMENT;
  kt::Frame f;
  std::string unused;  // prepare_frame cannot fail after validate(): stays empty
  st = kt::prepare_frame(desc, &f, nullptr, &unused);
  if (st != KT_OK) return st;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kMaxDevices) return KT_ERR_UNSUPPORTED;
  // Set-up, once per device, with that device current.
  unsigned char* base = g_scratch_addr[dev].load(std::memory_order_acquire);
  if (!base) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return e == cudaSuccess ? KT_ERR_INTERNAL : cuda_status(e);
    base = static_cast<unsigned char*>(p);
    g_scratch_addr[dev].store(base, std::memory_order_release);
  }
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t* counters = reinterpret_cast<uint32_t*>(base);  // [0] queue, [1] fallback queue, [2] fallback count
  uint32_t* fb_pix = reinterpret_cast<uint32_t*>(base + kCounterBytes);
  uint32_t* fb_slot = fb_pix + KT_NOALLOC_MAX_PIXELS;
  uint32_t* order = fb_slot + KT_NOALLOC_MAX_PIXELS;  // kOrderWords words
  e = cudaMemsetAsync(counters, 0, 4 * sizeof(uint32_t), s);
  if (e != cudaSuccess) return cuda_status(e);
  kt::OutSoA o;
  o.outcome = out->outcome;
  o.r = out->r;
  o.red = out->redshift;
  o.magnif = out->magnif;
  o.phi_disk = out->phi_disk;
  o.th_esc = out->theta_esc;
  o.ph_esc = out->phi_esc;
  o.status = out->status;
  o.steps = out->steps;
  o.attempts = out->attempts;
  const uint32_t n = (uint32_t)((int64_t)desc->width * desc->height);
  // As kt_trace (run_trace in kt_api.cpp): a whole frame of at least
  // kOrderMinPixels pixels is traced in centre-out order, each ray written at
  // its own pixel; smaller frames in row-major order.
  kt::RayList rl = {nullptr, nullptr, nullptr, n};
  if (n >= kt::kOrderMinPixels) {
    if ((size_t)n + kt::ring_scratch_words(n) > kOrderWords) return KT_ERR_INTERNAL;
    e = kt::launch_ring_order(desc->width, desc->height, 0, order + n, order, s);
    if (e != cudaSuccess) return cuda_status(e);
    rl = {order, order, nullptr, n};
  }
  const kt::Fallback fb = {fb_pix, fb_slot, counters + 2};
  const kt::Mode m = mode_of(f);
  kt::LaunchShape ls;
  st = shape(dev, m, &ls);
  if (st != KT_OK) return st;
  e = kt::launch_trace(m, f, o, rl, counters, fb, ls, s);
  if (e != cudaSuccess) return cuda_status(e);
  if (m == kt::kModeKSRk4) {
    // rays whose KS initialisation failed, traced in the BL chart
    const kt::Mode bm = f.intg == KT_DOPRI5 ? kt::kModeBLDopri5 : kt::kModeBLRk4;
    st = shape(dev, bm, &ls);
    if (st != KT_OK) return st;
    const kt::RayList fl = {fb_pix, fb_slot, counters + 2, 0};
    e = kt::launch_trace(bm, f, o, fl, counters + 1, fb, ls, s);
    if (e != cudaSuccess) return cuda_status(e);
  }
  return KT_OK;
}
