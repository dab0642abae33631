// kt_context.h -- the context behind the C ABI's kt_context handle and the
// helpers every entry point uses (device guard, error recording, growable
// device buffers).  Private to the library.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/kerrtrace.h"
#include "kt_internal.h"

struct kt_context {
  int device = 0;
  std::string err;
  uint32_t* d_counters = nullptr;  // [0] ray queue, [1] fallback queue, [2] fallback count
  uint32_t* d_fb = nullptr;        // fallback list: pix[cap] then slot[cap]
  size_t fb_cap = 0;
  // centre-out ray order of a frame (list, then the rings' counts)
  uint32_t* d_order = nullptr;
  size_t order_cap = 0;
  // device staging for the host-buffer entry points
  unsigned char* d_stage = nullptr;
  size_t stage_cap = 0;
  unsigned char* d_bg = nullptr;
  size_t bg_cap = 0;
  // gradients: per-ray contributions [kGSlots][n], sums, host copy
  double* d_grad = nullptr;
  size_t grad_cap = 0;
  double* d_gsum = nullptr;
  size_t gsum_cap = 0;
  cudaStream_t stream = nullptr;
  kt::LaunchShape shapes[kt::kNumModes];
  bool shape_ok[kt::kNumModes] = {};
};

namespace ktc {

// Makes the context's device current for the duration of a call.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    ok = cudaSetDevice(dev) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

inline kt_status fail(kt_context* ctx, kt_status st, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return st;
}

inline kt_status cuda_fail(kt_context* ctx, cudaError_t e, const char* what) {
  kt_status st = KT_ERR_CUDA;
  if (e == cudaErrorMemoryAllocation) st = KT_ERR_OUT_OF_MEMORY;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) st = KT_ERR_NO_DEVICE;
  return fail(ctx, st, std::string(what) + ": " + cudaGetErrorString(e));
}

#define KT_CUDA(ctx, call, what)                   \
  do {                                             \
    cudaError_t _e = (call);                       \
    if (_e != cudaSuccess) return ktc::cuda_fail(ctx, _e, what); \
  } while (0)

inline kt_status ensure(kt_context* ctx, void** buf, size_t* cap, size_t need, const char* what) {
  if (*cap >= need && *buf) return KT_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(buf, need);
  if (e != cudaSuccess) {
    *buf = nullptr;
    return cuda_fail(ctx, e, what);
  }
  *cap = need;
  return KT_OK;
}

inline kt::OutSoA to_out(const kt_geo_soa* o) {
  kt::OutSoA s;
  s.outcome = o->outcome;
  s.r = o->r;
  s.red = o->redshift;
  s.magnif = o->magnif;
  s.phi_disk = o->phi_disk;
  s.th_esc = o->theta_esc;
  s.ph_esc = o->phi_esc;
  s.status = o->status;
  s.steps = o->steps;
  s.attempts = o->attempts;
  return s;
}

inline bool out_complete(const kt_geo_soa* o) {
  return o && o->outcome && o->r && o->redshift && o->magnif && o->phi_disk && o->theta_esc &&
         o->phi_esc;
}

}  // namespace ktc
