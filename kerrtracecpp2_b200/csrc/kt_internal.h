// kt_internal.h -- declarations shared by the kernels and the C ABI layer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kt_machines.cuh"

namespace kt {

// Device result arrays of one trace (kt_geo_soa minus the optional NULLs).
struct OutSoA {
  uint8_t* outcome;
  double* r;
  double* red;
  double* magnif;
  double* phi_disk;
  double* th_esc;
  double* ph_esc;
  uint8_t* status;
  uint32_t* steps;
  uint32_t* attempts;
};

// Rays to trace: ray i is pixel pix[i] (or i) and writes output slot
// slot[i] (or i); the count is n, or *n_dev when n_dev is set (a count
// produced on the device by an earlier kernel).
struct RayList {
  const uint32_t* pix;
  const uint32_t* slot;
  const uint32_t* n_dev;
  uint32_t n;
};

// Rays the KS kernel hands back to the BL chart (init_ks_state failed).
struct Fallback {
  uint32_t* pix;
  uint32_t* slot;
  uint32_t* count;
};

enum Mode : int {
  kModeBLRk4 = 0,
  kModeBLDopri5 = 1,
  kModeKSRk4 = 2,
  kModeBundle = 3,
  kModeBLRk4Mixed = 4,
  kModeBLDopri5Mixed = 5,
  kModeKSRk4Mixed = 6,
  kNumModes = 7
};

// Kernel mode of a prepared frame (and, for the KS chart, of its BL
// fallback pass).
inline Mode frame_mode(const Frame& f) {
  if (f.bundles) return kModeBundle;
  const bool mixed = f.precision == 1;
  if (f.chart == 0) return mixed ? kModeKSRk4Mixed : kModeKSRk4;
  if (f.intg == 1) return mixed ? kModeBLDopri5Mixed : kModeBLDopri5;
  return mixed ? kModeBLRk4Mixed : kModeBLRk4;
}
inline Mode fallback_mode(const Frame& f) {
  const bool mixed = f.precision == 1;
  if (f.intg == 1) return mixed ? kModeBLDopri5Mixed : kModeBLDopri5;
  return mixed ? kModeBLRk4Mixed : kModeBLRk4;
}
inline bool is_ks_mode(Mode m) { return m == kModeKSRk4 || m == kModeKSRk4Mixed; }

struct LaunchShape {
  int block;    // threads per block
  int grid;     // persistent blocks
  size_t smem;  // dynamic shared memory per block (ray machines)
};

// Occupancy-derived persistent grid for one mode (cached per device).
cudaError_t launch_shape(Mode mode, int device, LaunchShape* shape);

// Launch one persistent trace kernel.  `queue` must be zero on entry.
cudaError_t launch_trace(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                         uint32_t* queue, const Fallback& fb, const LaunchShape& shape,
                         cudaStream_t stream);

// Colour pass: SoA -> RGB8.
cudaError_t launch_colorize(const ColourConst& cc, int64_t n, const uint8_t* outcome,
                            const double* r, const double* red, const double* magnif,
                            const double* th_esc, const double* ph_esc, const uint8_t* bg,
                            int bg_w, int bg_h, uint8_t* rgb, cudaStream_t stream);

// Mixed-precision kernels (kt_mixed.cu).
cudaError_t launch_shape_mixed(Mode mode, int device, LaunchShape* shape);
cudaError_t launch_trace_mixed(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                               uint32_t* queue, const Fallback& fb, const LaunchShape& shape,
                               cudaStream_t stream);

// FP64 throughput probe: n_iter dependent FMA chains per thread.
cudaError_t launch_fp64_probe(double* out, int n_iter, int grid, int block, cudaStream_t stream);

}  // namespace kt
