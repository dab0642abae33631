// kt_adjoint.h -- launchers of the smooth tracer and of its adjoint
// (kt_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

#include "kt_internal.h"
#include "kt_smray.cuh"

namespace kt {

// Smooth trace of pixels 0..n-1 into `out` (outcome NULL: no outputs); with
// `job`, the reverse sweeps and the per-ray contributions too.  counters[0..3)
// must be zero on entry (queues and the KS fallback count); fb_pix holds n
// rays (the KS chart's fallback list).  Without a job, `order` (n pixel
// indices, or NULL for 0..n-1) is the order the rays are taken in.
cudaError_t launch_smooth(const Frame& f, const OutSoA& out, uint32_t n, const SmJob* job,
                          uint32_t* counters, uint32_t* fb_pix, int device, cudaStream_t st,
                          const uint32_t* order = nullptr);

// out[kGSlots] = fixed-order sums over the rays of contrib[kGSlots][n];
// `partial` holds grad_sum_scratch_doubles() - kGSlots doubles.
cudaError_t launch_grad_sum(const double* contrib, uint32_t n, double* partial, double* out,
                            cudaStream_t st);
size_t grad_sum_scratch_doubles();

}  // namespace kt
