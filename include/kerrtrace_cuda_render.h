// kerrtrace_cuda_render.h -- link-compatible replacement for the reference
// renderer's CUDA entry point.
//
// The reference's main.cpp, built with -DUSE_CUDA, calls
//   std::vector<uint32_t> cuda_render(const KNdSParams_CUDA&,
//                                     const CameraParams_CUDA&, bool)
// (declared in gpu/cuda/tracer.cuh:11-26, called at main.cpp:2430-2443 for
// the single-ray, standard-solver case).  Linking main.cpp against
// libkerrtrace.so instead of tracer.cu routes that call to this renderer.
// The structs and the signature must stay exactly as the reference declares
// them (C++ mangling and layout); this header restates them.
//
// Behaviour: traces and colours the frame with the reference's CPU
// algorithm (BL or KS chart, RK4 step doubling, tol 1e-7, the reference's
// default controls), with a black background (the call carries none) and
// returns RGBA packed as 0xFF<<24 | B<<16 | G<<8 | R, as the reference's
// CUDA kernel does.  Errors throw std::runtime_error, as the reference's
// CUDA_CHECK does (gpu/cuda/tracer.cu:19-23).  Each calling thread's first
// call creates a renderer context on device 0 that its later calls reuse
// (the reference allocates and frees its device buffers on every call); it
// is destroyed when the thread exits.
#pragma once

#include <cstdint>
#include <vector>

struct KNdSParams_CUDA {
  double M, a, Q, Lambda;
  double r_horizon, r_isco, r_disk_out;
};

struct CameraParams_CUDA {
  double r_obs, theta_obs, phi_obs, fov_h;  // radians
  int width, height;
  int chart;  // 0 = BL, 1 = KS
};

std::vector<uint32_t> cuda_render(const KNdSParams_CUDA& kp, const CameraParams_CUDA& cp,
                                  bool require_fp64);
