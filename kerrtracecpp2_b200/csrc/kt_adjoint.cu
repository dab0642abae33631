// kt_adjoint.cu -- kernels of the smooth tracer (KT_PREC_SMOOTH) and of its
// discrete adjoint (kt_vjp, kt_l2_grad).
//
// One thread per ray, rays from a device queue (persistent grid).  The
// gradient kernel traces its ray with checkpoints in local memory
// (SmScratch, ~9 KB per thread), and for a disk hit with a non-zero
// cotangent runs the reverse sweep right away; it writes the ray's loss and
// gradient contributions to a [kGSlots][n] array, which k_sum_* reduce in a
// fixed order (the sum does not depend on the schedule).
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

template <bool kGrad>
__global__ void __launch_bounds__(kSmBlock) k_smooth(const Frame f, const OutSoA out, const SmJob job,
                                                     uint32_t n, uint32_t* __restrict__ queue) {
  SmScratch sc;
  KT_ROLLED
  for (;;) {
    const uint32_t pix = atomicAdd(queue, 1u);
    if (pix >= n) break;
    RayResult o;
    double g[kGSlots];
    sm_pixel<kGrad>(f, pix, job.force_bl != 0, job.cot, &o, g, kGrad ? &sc : nullptr);
    if (out.outcome) write_result(out, pix, o);
    if (kGrad)
      for (int q = 0; q < kGSlots; ++q) job.contrib[(size_t)q * n + pix] = g[q];
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

template <bool kGrad>
static cudaError_t smooth_grid(int device, int* grid) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_smooth<kGrad>, kSmBlock, 0);
  if (e != cudaSuccess) return e;
  *grid = sms * (per_sm < 1 ? 1 : per_sm);
  return cudaSuccess;
}

cudaError_t launch_smooth(const Frame& f, const OutSoA& out, uint32_t n, const SmJob* job,
                          uint32_t* queue, int device, cudaStream_t st) {
  int grid = 0;
  cudaError_t e = job ? smooth_grid<true>(device, &grid) : smooth_grid<false>(device, &grid);
  if (e != cudaSuccess) return e;
  if (job) {
    k_smooth<true><<<grid, kSmBlock, 0, st>>>(f, out, *job, n, queue);
  } else {
    SmJob none;
    memset(&none, 0, sizeof none);
    k_smooth<false><<<grid, kSmBlock, 0, st>>>(f, out, none, n, queue);
  }
  return cudaGetLastError();
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
