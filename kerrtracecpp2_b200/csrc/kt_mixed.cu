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
#include <cmath>

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

// The single-ray mixed modes come in two instantiations: kFp32 (some frame
// of the launch has a finite r_fp32) carries the FP32 right-hand side and
// the constraint reprojection; the other, for tolerances below 1e-8, runs
// the FP64 analytic RHS alone, without that code in the kernel.
template <bool kFp32>
struct ModeBLRk4MixedT {
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
    if constexpr (kFp32) {
      bl_rhs_mixed(f, y, m->pt, m->pphi, k);
      const int it0 = m->it;
      if (m->consume(f, s, k, res)) return true;
      mixed_after_slot(f, m, s, it0);
      return false;
    } else {
      bl_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, k);
      return m->consume(f, s, k, res);
    }
  }
};

template <bool kFp32>
struct ModeBLDopri5MixedT {
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
    if constexpr (kFp32) {
      bl_rhs_mixed(f, y, m->pt, m->pphi, k);
      const int it0 = m->it;
      if (m->consume(f, s, k, res)) return true;
      mixed_after_slot(f, m, s, it0);
      return false;
    } else {
      bl_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, k);
      return m->consume(f, s, k, res);
    }
  }
};

// KS: FP32 beyond r_fp32 unless the radial momentum x.p/|x| is small.
template <bool kFp32>
struct ModeKSRk4MixedT {
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
    if constexpr (kFp32) {
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
    } else {
      ks_rhs_analytic<double>(f.g, y[0], y[1], y[2], y[3], y[4], y[5], m->pT, k);
      return m->consume(f, s, k, res);
    }
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
template <bool B> struct Shape<ModeBLRk4MixedT<B>> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
// A warp refills once all 32 lanes are idle, so its rays are always the same
// 32 consecutive rays of the queue and the per-warp FP32 choice does not
// depend on the schedule (refilling at 16 idle lanes measured 21.2 ms
// against 22.3 at 720p, tol 1e-8, but mixes the groups).  Block and minimum
// blocks are shared by both instantiations (see launch_shape_mixed).
#ifndef KT_MIXED32_DOPRI5_REFILL
#define KT_MIXED32_DOPRI5_REFILL 32
#endif
#ifndef KT_MIXED_DOPRI5_MINB
#define KT_MIXED_DOPRI5_MINB 9
#endif
template <bool B> struct Shape<ModeBLDopri5MixedT<B>> {
  static constexpr int kBlock = 64, kMinBlocks = KT_MIXED_DOPRI5_MINB,
                       kRefill = B ? KT_MIXED32_DOPRI5_REFILL : 32;
};
template <bool B> struct Shape<ModeKSRk4MixedT<B>> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
// Mixed bundles: 64-thread blocks, at least 6 per SM (168 registers, no
// spill), measured at 1080p: 90.8 ms against 97.2 for 128 x 1 (216
// registers), 98.3 for 128 x 3, 91.7 for 64 x 5; refilling at 16 or 8 idle
// lanes 101.0 / 101.6.
#ifndef KT_MIXED_BUNDLE_BLOCK
#define KT_MIXED_BUNDLE_BLOCK 64
#endif
#ifndef KT_MIXED_BUNDLE_MINB
#define KT_MIXED_BUNDLE_MINB 6
#endif
#ifndef KT_MIXED_BUNDLE_REFILL
#define KT_MIXED_BUNDLE_REFILL 32
#endif
template <> struct Shape<ModeBundleMixed> {
  static constexpr int kBlock = KT_MIXED_BUNDLE_BLOCK, kMinBlocks = KT_MIXED_BUNDLE_MINB,
                       kRefill = KT_MIXED_BUNDLE_REFILL;
};

template <class ModeT>
static cudaError_t launch_one(const Frame& f, const OutSoA& out, const RayList& rl,
                              uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                              cudaStream_t stream) {
  k_trace<ModeT><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb);
  return cudaGetLastError();
}

// Both instantiations of a mode share its launch bounds, block and shared
// memory, so one shape (the kFp32 one's) serves either.
cudaError_t launch_shape_mixed(Mode mode, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4Mixed: return shape_for<ModeBLRk4MixedT<true>>(device, shape);
    case kModeBLDopri5Mixed: return shape_for<ModeBLDopri5MixedT<true>>(device, shape);
    case kModeKSRk4Mixed: return shape_for<ModeKSRk4MixedT<true>>(device, shape);
    case kModeBundleMixed: return shape_for<ModeBundleMixed>(device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_trace_mixed(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                               uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                               cudaStream_t stream) {
  const bool fp32 = std::isfinite(f.r_fp32);
  switch (mode) {
    case kModeBLRk4Mixed:
      return fp32 ? launch_one<ModeBLRk4MixedT<true>>(f, out, rl, queue, fb, s, stream)
                  : launch_one<ModeBLRk4MixedT<false>>(f, out, rl, queue, fb, s, stream);
    case kModeBLDopri5Mixed:
      return fp32 ? launch_one<ModeBLDopri5MixedT<true>>(f, out, rl, queue, fb, s, stream)
                  : launch_one<ModeBLDopri5MixedT<false>>(f, out, rl, queue, fb, s, stream);
    case kModeKSRk4Mixed:
      return fp32 ? launch_one<ModeKSRk4MixedT<true>>(f, out, rl, queue, fb, s, stream)
                  : launch_one<ModeKSRk4MixedT<false>>(f, out, rl, queue, fb, s, stream);
    case kModeBundleMixed: return launch_one<ModeBundleMixed>(f, out, rl, queue, fb, s, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t batch_shape_mixed(Mode mode, int variant, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4Mixed: return batch_shape<ModeBLRk4MixedT<true>>(variant, device, shape);
    case kModeBLDopri5Mixed: return batch_shape<ModeBLDopri5MixedT<true>>(variant, device, shape);
    case kModeKSRk4Mixed: return batch_shape<ModeKSRk4MixedT<true>>(variant, device, shape);
    case kModeBundleMixed: return batch_shape<ModeBundleMixed>(variant, device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_batch_mixed(Mode mode, int variant, const BatchRays& br, uint32_t* queue,
                               const Fallback& fb, const LaunchShape& s, cudaStream_t st) {
  switch (mode) {
    case kModeBLRk4Mixed:
      return br.fp32 ? batch_launch<ModeBLRk4MixedT<true>>(variant, br, queue, fb, s, st)
                     : batch_launch<ModeBLRk4MixedT<false>>(variant, br, queue, fb, s, st);
    case kModeBLDopri5Mixed:
      return br.fp32 ? batch_launch<ModeBLDopri5MixedT<true>>(variant, br, queue, fb, s, st)
                     : batch_launch<ModeBLDopri5MixedT<false>>(variant, br, queue, fb, s, st);
    case kModeKSRk4Mixed:
      return br.fp32 ? batch_launch<ModeKSRk4MixedT<true>>(variant, br, queue, fb, s, st)
                     : batch_launch<ModeKSRk4MixedT<false>>(variant, br, queue, fb, s, st);
    case kModeBundleMixed: return batch_launch<ModeBundleMixed>(variant, br, queue, fb, s, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kt
