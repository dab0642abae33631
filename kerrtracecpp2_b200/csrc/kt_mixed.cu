// kt_mixed.cu -- mixed-precision trace kernels (KT_PREC_MIXED).
//
// Same persistent loop and the same FP64 integrators as the exact kernels
// (state, stage sums, embedded error estimate, step-size controller, event
// location and the disk-crossing root all stay FP64; in bundle mode the
// Jacobi map W and its determinant too), with a different right-hand side:
// the Hamiltonian gradient is evaluated analytically
// (bl_rhs_analytic / ks_rhs_analytic: one inverse metric with four
// reciprocals instead of five metrics with 26 correctly rounded divisions),
// in FP32 where the tolerance and the geometry allow it, else in FP64.
// FP32 is used for a warp's RHS only when every active lane of the warp is
// beyond r_fp32 and away from a radial or polar turning point, so lanes never
// diverge between the two paths.  This file is compiled with FMA
// contraction on; its results are not bit-identical to the reference and
// are compared with the FP64 oracle statistically.
#include "kt_smooth.cuh"
#include "kt_trace_kernel.cuh"

namespace kt {

__device__ __forceinline__ bool warp_all(bool p) { return __all_sync(__activemask(), p); }

// BL: FP32 beyond r_fp32 unless p_r or p_theta/r is small against |p_t|.
__device__ __forceinline__ void bl_rhs_mixed(const Frame& f, const double y[4], double pt,
                                             double pphi, double k[5]) {
  const double lim = f.turn_frac * fabs(pt);
  const bool far = y[0] > f.r_fp32 && fabs(y[2]) > lim && fabs(y[3]) > lim * y[0];
  if (warp_all(far))
    bl_rhs_analytic<float>(f.g, y[0], y[1], y[2], y[3], pt, pphi, k);
  else
    bl_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], pt, pphi, k);
}

struct ModeBLRk4Mixed {
  using Machine = BLRk4;
  static constexpr int kSlots = BLRk4::kSlots;
  BLRk4* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, uint32_t, const Fallback&) {
    m->init(f, camera_ray(f, pix));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], k[5];
    m->input(s, y);
    bl_rhs_mixed(f, y, m->pt, m->pphi, k);
    const int it0 = m->it;
    if (m->consume(f, s, k, res)) return true;
    mixed_after_slot(f, m, s, it0);
    return false;
  }
};

struct ModeBLDopri5Mixed {
  using Machine = BLDopri5;
  static constexpr int kSlots = BLDopri5::kSlots;
  BLDopri5* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, uint32_t, const Fallback&) {
    m->init(f, camera_ray(f, pix));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], k[5];
    m->input(s, y);
    bl_rhs_mixed(f, y, m->pt, m->pphi, k);
    const int it0 = m->it;
    if (m->consume(f, s, k, res)) return true;
    mixed_after_slot(f, m, s, it0);
    return false;
  }
};

// KS: FP32 beyond r_fp32 unless the radial momentum x.p/|x| is small.
struct ModeKSRk4Mixed {
  using Machine = KSRk4;
  static constexpr int kSlots = KSRk4::kSlots;
  KSRk4* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t out_slot,
                                        uint32_t fb_key, const Fallback& fb) {
    if (m->init(f, camera_ray(f, pix))) return true;
    const uint32_t i = atomicAdd(fb.count, 1u);
    fb.pix[i] = fb_key;
    if (fb.slot) fb.slot[i] = out_slot;
    return false;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[6], k[6];
    m->input(s, y);
    const double rr = sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
    const double prad = (y[0] * y[3] + y[1] * y[4] + y[2] * y[5]) / rr;
    const bool far = rr > f.r_fp32 && fabs(prad) > f.turn_frac * fabs(m->pT);
    if (warp_all(far))
      ks_rhs_analytic<float>(f.g, y[0], y[1], y[2], y[3], y[4], y[5], m->pT, k);
    else
      ks_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], y[4], y[5], m->pT, k);
    const int it0 = m->it;
    if (m->consume(f, s, k, res)) return true;
    mixed_after_slot(f, m, s, it0);
    return false;
  }
};

struct ModeBundleMixed {
  using Machine = Bundle;
  static constexpr int kSlots = Bundle::kSlots;
  Bundle* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, uint32_t, const Fallback&) {
    m->init(f, (int)(pix % (uint32_t)f.cam.W), (int)(pix / (uint32_t)f.cam.W));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], yW[8], k[5], kW[8];
    m->input(s, y, yW);
    bundle_rhs_analytic(f.g, y, m->pt, m->pphi, yW, k, kW);
    return m->consume(f, s, k, kW, res);
  }
};

// Launch shapes, measured on B200 as for the exact kernels: refilling a
// warp only when all 32 lanes are idle matters more here, since the FP32/FP64
// choice is made per warp and a warp of neighbouring rays that started
// together makes it alike (720p config 2 DOPRI5: 24.3 against 31.9 ms; BL
// RK4: 25.2 against 41.1; KS RK4: 22.3 against 52.1; 1080p bundles: 224
// against 243).
template <> struct Shape<ModeBLRk4Mixed> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
template <> struct Shape<ModeBLDopri5Mixed> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
template <> struct Shape<ModeKSRk4Mixed> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
template <> struct Shape<ModeBundleMixed> { static constexpr int kBlock = 128, kMinBlocks = 1, kRefill = 32; };

template <class ModeT>
static cudaError_t launch_one(const Frame& f, const OutSoA& out, const RayList& rl,
                              uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                              cudaStream_t stream) {
  k_trace<ModeT><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb);
  return cudaGetLastError();
}

cudaError_t launch_shape_mixed(Mode mode, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4Mixed: return shape_for<ModeBLRk4Mixed>(device, shape);
    case kModeBLDopri5Mixed: return shape_for<ModeBLDopri5Mixed>(device, shape);
    case kModeKSRk4Mixed: return shape_for<ModeKSRk4Mixed>(device, shape);
    case kModeBundleMixed: return shape_for<ModeBundleMixed>(device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_trace_mixed(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                               uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                               cudaStream_t stream) {
  switch (mode) {
    case kModeBLRk4Mixed: return launch_one<ModeBLRk4Mixed>(f, out, rl, queue, fb, s, stream);
    case kModeBLDopri5Mixed: return launch_one<ModeBLDopri5Mixed>(f, out, rl, queue, fb, s, stream);
    case kModeKSRk4Mixed: return launch_one<ModeKSRk4Mixed>(f, out, rl, queue, fb, s, stream);
    case kModeBundleMixed: return launch_one<ModeBundleMixed>(f, out, rl, queue, fb, s, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t batch_shape_mixed(Mode mode, int variant, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4Mixed: return batch_shape<ModeBLRk4Mixed>(variant, device, shape);
    case kModeBLDopri5Mixed: return batch_shape<ModeBLDopri5Mixed>(variant, device, shape);
    case kModeKSRk4Mixed: return batch_shape<ModeKSRk4Mixed>(variant, device, shape);
    case kModeBundleMixed: return batch_shape<ModeBundleMixed>(variant, device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_batch_mixed(Mode mode, int variant, const BatchRays& br, uint32_t* queue,
                               const Fallback& fb, const LaunchShape& s, cudaStream_t st) {
  switch (mode) {
    case kModeBLRk4Mixed: return batch_launch<ModeBLRk4Mixed>(variant, br, queue, fb, s, st);
    case kModeBLDopri5Mixed: return batch_launch<ModeBLDopri5Mixed>(variant, br, queue, fb, s, st);
    case kModeKSRk4Mixed: return batch_launch<ModeKSRk4Mixed>(variant, br, queue, fb, s, st);
    case kModeBundleMixed: return batch_launch<ModeBundleMixed>(variant, br, queue, fb, s, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kt
