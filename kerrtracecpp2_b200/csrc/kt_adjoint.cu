// kt_adjoint.cu -- kernels of the smooth tracer (KT_PREC_SMOOTH) and of its
// discrete adjoint (kt_vjp, kt_l2_grad).
//
// One thread per ray, rays from a device queue (persistent grid) in groups
// of 32 consecutive rays per warp (a warp takes the next group once all its
// lanes are done: neighbouring rays follow alike paths, so the warp's lanes
// stay converged far longer than with rays taken one lane at a time), one
// kernel per chart (a kernel with both charts' code overflowed the instruction
// cache: most issue slots went to instruction-fetch stalls).  The
// gradient kernel traces its ray with checkpoints in local memory
// (SmScratch, ~12 KB per thread), and for a disk hit with a non-zero
// cotangent runs the reverse sweep right away; it writes the ray's loss and
// gradient contributions to a [kGSlots][n] array, which k_sum_* reduce in a
// fixed order (the sum does not depend on the schedule).  The tangent kernel
// gives one parameter's entry by forward mode (no recording).
//
// BL frames integrated with DOPRI5 have their own pair of kernels (the
// smooth DOPRI5 attempt and its reverse, kt_smray.cuh), and so do Jacobi
// bundles (ChartBLB: the geodesic with its 4x2 Jacobi matrix, ~20 KB of
// checkpoints per thread).
//
// Compiled with --fmad=false: the recorded forward and every replay of it
// must round identically, which contraction choices made per inlining site
// would not guarantee.
#include "kt_adjoint.h"
#include "kt_trace_kernel.cuh"

namespace kt {

constexpr int kSmBlock = 64;
constexpr int kSumBlocks = 296;
constexpr int kSumThreads = 256;

// Rays: pixels 0..n-1, or list[0..*n_dev) (a count on the device) or
// list[0..n_list) (on the host).  The KS kernel appends the rays
// whose KS initialisation fails to fb_pix (count *fb_n) for the BL kernel.
// Minimum blocks per SM of the gradient kernels, measured (ms per gradient,
// unconstrained / 6 / 8 blocks of 64 threads): config 5 48 / 58 / 80, the
// 720p DOPRI5 frame 156 / 195 / 233, the 960x540 bundle frame 623 / 596 /
// 657.  Only the bundle kernel takes the bound.
template <class C, bool kGrad>
constexpr int sm_min_blocks() { return (kGrad && C::kBundle) ? 6 : 1; }

template <class C, bool kGrad, class I>
__global__ void __launch_bounds__(kSmBlock, (sm_min_blocks<C, kGrad>())) k_smooth(const Frame f, const OutSoA out, const SmJob job,
                                                     uint32_t n, const uint32_t* __restrict__ list,
                                                     uint32_t n_list,
                                                     const uint32_t* __restrict__ n_dev,
                                                     uint32_t* __restrict__ queue,
                                                     uint32_t* __restrict__ fb_pix,
                                                     uint32_t* __restrict__ fb_n) {
  SmScratch<C::kN> sc;
  const uint32_t count = n_dev ? *n_dev : (list ? n_list : n);
  const unsigned lane = threadIdx.x & 31u;
  KT_ROLLED
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(queue, 32u);
    base = __shfl_sync(kFull, base, 0);
    if (base >= count) break;
    const uint32_t i = base + lane;
    const uint32_t pix = i < count ? (list ? list[i] : i) : n;
    if (pix < n) {  // else past the end, or a caller's list index outside the frame
      RayResult o;
      double g[kGSlots];
      if (!sm_pixel<C, kGrad, I>(f, pix, job.cot, &o, g, kGrad ? &sc : nullptr)) {
        fb_pix[atomicAdd(fb_n, 1u)] = pix;
      } else {
        if (out.outcome) write_result(out, pix, o);
        if (kGrad)
          for (int q = 0; q < kGSlots; ++q) job.contrib[(size_t)q * n + pix] = g[q];
      }
    }
    __syncwarp();
  }
}

// The same over the forward-mode tangent along job.tangent_dir.
template <class C>
__global__ void __launch_bounds__(kSmBlock) k_smooth_tangent(const Frame f, const OutSoA out,
                                                             const SmJob job, uint32_t n,
                                                             const uint32_t* __restrict__ list,
                                                             uint32_t n_list,
                                                             const uint32_t* __restrict__ n_dev,
                                                             uint32_t* __restrict__ queue,
                                                             uint32_t* __restrict__ fb_pix,
                                                             uint32_t* __restrict__ fb_n) {
  const uint32_t count = n_dev ? *n_dev : (list ? n_list : n);
  const unsigned lane = threadIdx.x & 31u;
  KT_ROLLED
  for (;;) {
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(queue, 32u);
    base = __shfl_sync(kFull, base, 0);
    if (base >= count) break;
    const uint32_t i = base + lane;
    const uint32_t pix = i < count ? (list ? list[i] : i) : n;
    if (pix < n) {
      RayResult o;
      double g[kGSlots];
      // without outputs, pixels whose cotangent is zero are not traced
      if (!sm_pixel_tangent<C>(f, pix, job.tangent_dir, job.cot, &o, g, out.outcome != nullptr)) {
        fb_pix[atomicAdd(fb_n, 1u)] = pix;
      } else {
        if (out.outcome) write_result(out, pix, o);
        for (int q = 0; q < kGSlots; ++q) job.contrib[(size_t)q * n + pix] = g[q];
      }
    }
    __syncwarp();
  }
}

// Fixed-order sums of the [kGSlots][n] contributions: block b sums the rays
// [b*n/B, (b+1)*n/B) of every slot (threads strided, then a tree), then one
// block sums the B partials.
__global__ void __launch_bounds__(kSumThreads) k_sum_partial(const double* __restrict__ contrib,
                                                             uint32_t n, double* __restrict__ partial) {
  __shared__ double red[kSumThreads];
  const uint64_t lo = (uint64_t)blockIdx.x * n / gridDim.x;
  const uint64_t hi = (uint64_t)(blockIdx.x + 1) * n / gridDim.x;
  for (int q = 0; q < kGSlots; ++q) {
    double s = 0.0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kSumThreads) s += contrib[(size_t)q * n + i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[q * gridDim.x + blockIdx.x] = red[0];
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kSumThreads) k_sum_final(const double* __restrict__ partial, int nb,
                                                           double* __restrict__ out) {
  __shared__ double red[kSumThreads];
  for (int q = 0; q < kGSlots; ++q) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += kSumThreads) s += partial[q * nb + i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kSumThreads / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = red[0];
    __syncthreads();
  }
}

template <class C>
static cudaError_t tangent_launch(const Frame& f, const OutSoA& out, uint32_t n, const SmJob& job,
                                  const uint32_t* list, uint32_t n_list, const uint32_t* n_dev,
                                  uint32_t* queue,
                                  uint32_t* fb_pix, uint32_t* fb_n, int device, cudaStream_t st) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_smooth_tangent<C>, kSmBlock, 0);
  if (e != cudaSuccess) return e;
  const int grid = sms * (per_sm < 1 ? 1 : per_sm);
  k_smooth_tangent<C><<<grid, kSmBlock, 0, st>>>(f, out, job, n, list, n_list, n_dev, queue, fb_pix,
                                                  fb_n);
  return cudaGetLastError();
}

template <class C, bool kGrad, class I = SmRk4>
static cudaError_t smooth_launch(const Frame& f, const OutSoA& out, uint32_t n, const SmJob& job,
                                 const uint32_t* list, uint32_t n_list, const uint32_t* n_dev,
                                 uint32_t* queue,
                                 uint32_t* fb_pix, uint32_t* fb_n, int device, cudaStream_t st) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_smooth<C, kGrad, I>, kSmBlock, 0);
  if (e != cudaSuccess) return e;
  const int grid = sms * (per_sm < 1 ? 1 : per_sm);
  k_smooth<C, kGrad, I><<<grid, kSmBlock, 0, st>>>(f, out, job, n, list, n_list, n_dev, queue, fb_pix,
                                                    fb_n);
  return cudaGetLastError();
}

cudaError_t launch_smooth(const Frame& f, const OutSoA& out, uint32_t n, const SmJob* job,
                          uint32_t* counters, uint32_t* fb_pix, int device, cudaStream_t st,
                          const uint32_t* order) {
  SmJob none;
  memset(&none, 0, sizeof none);
  none.pix = order;
  none.n_pix = order ? n : 0;
  const SmJob& jb = job ? *job : none;
  const bool grad = job != nullptr;
  // Jacobi bundles (BL chart, RK4 step doubling whatever the integrator, as
  // trace_bundle): no forward-mode tangent (their Lambda comes from the sweep)
  if (f.bundles) {
    if (grad && job->tangent_dir >= 0) return cudaErrorInvalidValue;
    return grad ? smooth_launch<ChartBLB, true>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters,
                                                nullptr, nullptr, device, st)
                : smooth_launch<ChartBLB, false>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters,
                                                 nullptr, nullptr, device, st);
  }
  // BL frames with DOPRI5 (KS frames integrate with RK4, their BL passes too)
  const bool dp5 = f.intg == 1 && f.chart == 1;  // KT_DOPRI5, KT_CHART_BL
  if (dp5) {
    if (grad && job->tangent_dir >= 0) return cudaErrorInvalidValue;  // no DOPRI5 tangent
    return grad ? smooth_launch<ChartBL, true, SmDp5>(f, out, n, jb, jb.pix, jb.n_pix, nullptr,
                                                      counters, nullptr, nullptr, device, st)
                : smooth_launch<ChartBL, false, SmDp5>(f, out, n, jb, jb.pix, jb.n_pix, nullptr,
                                                       counters, nullptr, nullptr, device, st);
  }
  if (grad && job->tangent_dir >= 0) {
    if (f.chart == 0 && !job->force_bl) {
      cudaError_t e = tangent_launch<ChartKS>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters, fb_pix,
                                              counters + 2, device, st);
      if (e != cudaSuccess) return e;
      return tangent_launch<ChartBL>(f, out, n, jb, fb_pix, 0, counters + 2, counters + 1, nullptr,
                                     nullptr, device, st);
    }
    return tangent_launch<ChartBL>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters, nullptr, nullptr,
                                   device, st);
  }
  if (f.chart == 0 && !(job && job->force_bl)) {
    // KS pass over all pixels, then BL over the rays whose KS init failed
    cudaError_t e = grad ? smooth_launch<ChartKS, true>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters,
                                                        fb_pix, counters + 2, device, st)
                         : smooth_launch<ChartKS, false>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters,
                                                         fb_pix, counters + 2, device, st);
    if (e != cudaSuccess) return e;
    return grad ? smooth_launch<ChartBL, true>(f, out, n, jb, fb_pix, 0, counters + 2, counters + 1,
                                               nullptr, nullptr, device, st)
                : smooth_launch<ChartBL, false>(f, out, n, jb, fb_pix, 0, counters + 2, counters + 1,
                                                nullptr, nullptr, device, st);
  }
  return grad ? smooth_launch<ChartBL, true>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters, nullptr,
                                             nullptr, device, st)
              : smooth_launch<ChartBL, false>(f, out, n, jb, jb.pix, jb.n_pix, nullptr, counters, nullptr,
                                              nullptr, device, st);
}

cudaError_t launch_grad_sum(const double* contrib, uint32_t n, double* partial, double* out,
                            cudaStream_t st) {
  k_sum_partial<<<kSumBlocks, kSumThreads, 0, st>>>(contrib, n, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_final<<<1, kSumThreads, 0, st>>>(partial, kSumBlocks, out);
  return cudaGetLastError();
}

size_t grad_sum_scratch_doubles() { return (size_t)kGSlots * kSumBlocks + kGSlots; }

}  // namespace kt
