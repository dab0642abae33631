// kt_kernels.cu -- persistent geodesic-tracing kernels for sm_100a.
//
// One CUDA thread carries one ray at a time through a per-ray machine
// (kt_machines.cuh); the 32 rays of a warp advance through the slots of an
// adaptive attempt in lockstep, one Hamiltonian right-hand side per slot.
// At every attempt boundary the lanes whose rays finished take new rays from
// a device queue (one atomicAdd per warp for all its idle lanes).  Rays
// differ in length by 3-50x, so refilling keeps the FP64 pipes busy until
// the queue runs dry; the grid is sized to the resident capacity of the GPU
// (persistent kernel).  State lives in registers; results go out as SoA.
//
// The kernels do no waiting on other threads: the only inter-thread
// operation is the warp-synchronous refill and the queue atomic.  Every ray
// stops after at most max_steps accepted steps with at most 65 rejected
// attempts each (the reference's limits), so every loop ends.
#include "kt_internal.h"

namespace kt {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void write_result(const OutSoA& o, uint32_t s, const RayResult& r) {
  o.outcome[s] = (uint8_t)r.outcome;
  o.r[s] = r.r;
  o.red[s] = r.red;
  o.magnif[s] = r.magnif;
  o.phi_disk[s] = r.phi_disk;
  o.th_esc[s] = r.th_esc;
  o.ph_esc[s] = r.ph_esc;
  if (o.status) o.status[s] = (uint8_t)r.status;
  if (o.steps) o.steps[s] = r.steps;
  if (o.attempts) o.attempts[s] = r.attempts;
}

// ---- per-mode start (new ray) and one slot (one RHS) ---------------------

__device__ __forceinline__ Geo camera_ray(const Frame& f, uint32_t pix) {
  const int px = (int)(pix % (uint32_t)f.cam.W);
  const int py = (int)(pix / (uint32_t)f.cam.W);
  double al, be;
  pixel_angles(f.cam, px, py, &al, &be);
  return angle_ray(f.cam, al, be);
}

// Each mode keeps its ray machine in shared memory (one record per thread,
// record size an odd number of 8-byte words so a warp's accesses spread over
// the banks): the machine is touched only between RHS evaluations, so the
// registers are left to the RHS working set and more warps fit per SM.
template <class M>
struct alignas(8) SmemRecord {
  M m;
  double pad[((sizeof(M) + 7) / 8) % 2 == 0 ? 1 : 2];
};

struct ModeBLRk4 {
  using Machine = BLRk4;
  static constexpr int kSlots = BLRk4::kSlots;
  BLRk4* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, const Fallback&) {
    m->init(f, camera_ray(f, pix));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], k[5];
    m->input(s, y);
    bl_rhs(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, k);
    return m->consume(f, s, k, res);
  }
};

struct ModeBLDopri5 {
  using Machine = BLDopri5;
  static constexpr int kSlots = BLDopri5::kSlots;
  BLDopri5* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, const Fallback&) {
    m->init(f, camera_ray(f, pix));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], k[5];
    m->input(s, y);
    bl_rhs(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, k);
    return m->consume(f, s, k, res);
  }
};

struct ModeKSRk4 {
  using Machine = KSRk4;
  static constexpr int kSlots = KSRk4::kSlots;
  KSRk4* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t out_slot,
                                        const Fallback& fb) {
    if (m->init(f, camera_ray(f, pix))) return true;
    // init_ks_state failed: the ray is traced in the BL chart by a second
    // launch over the fallback list.
    const uint32_t i = atomicAdd(fb.count, 1u);
    fb.pix[i] = pix;
    fb.slot[i] = out_slot;
    return false;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[6], k[6];
    m->input(s, y);
    ks_rhs(f.g, y[0], y[1], y[2], y[3], y[4], y[5], m->pT, k);
    return m->consume(f, s, k, res);
  }
};

struct ModeBundle {
  using Machine = Bundle;
  static constexpr int kSlots = Bundle::kSlots;
  Bundle* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, const Fallback&) {
    m->init(f, (int)(pix % (uint32_t)f.cam.W), (int)(pix / (uint32_t)f.cam.W));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[4], yW[8], k[5], kW[8];
    m->input(s, y, yW);
    bundle_rhs(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, yW, k, kW);
    return m->consume(f, s, k, kW, res);
  }
};

template <class ModeT>
constexpr size_t smem_bytes(int block) {
  return sizeof(SmemRecord<typename ModeT::Machine>) * (size_t)block;
}

// Launch shape per mode, measured on B200 (720p KNdS frame, BL chart; 512^2
// Kerr-Newman frame, KS chart; 480x270 bundle frame): the BL single-ray
// kernels run best as 64-thread blocks capped at 113 registers (9 blocks =
// 18 warps per SM, limited by the 46 KB of ray machines per 128 threads);
// the KS and bundle kernels spill under that cap and keep 128 threads.
template <class ModeT> struct Shape { static constexpr int kBlock = 128, kMinBlocks = 1; };
template <> struct Shape<struct ModeBLRk4> { static constexpr int kBlock = 64, kMinBlocks = 9; };
template <> struct Shape<struct ModeBLDopri5> { static constexpr int kBlock = 64, kMinBlocks = 9; };

// ---- the persistent loop ---------------------------------------------------
// One iteration of the outer loop is one adaptive attempt for every ray of
// the warp.  At its start, idle lanes take new rays from the queue (one
// atomicAdd per warp).  Slot -1 runs only if some lane needs it (new rays,
// f at the end of an accepted step); slots 0..kSlots-1 run for every active
// lane.  All lanes of the warp see the same slot index, so the bookkeeping
// after each RHS runs converged; a lane whose ray ends mid-attempt idles to
// the end of the attempt.

template <class ModeT>
__global__ void __launch_bounds__(Shape<ModeT>::kBlock, Shape<ModeT>::kMinBlocks) k_trace(const Frame f, const OutSoA out, const RayList rl,
                                                  uint32_t* __restrict__ queue, const Fallback fb) {
  extern __shared__ __align__(16) unsigned char smem[];
  using Rec = SmemRecord<typename ModeT::Machine>;
  ModeT mode;
  mode.m = &reinterpret_cast<Rec*>(smem)[threadIdx.x].m;
  bool active = false;
  uint32_t out_slot = 0;
  const uint32_t n = rl.n_dev ? *rl.n_dev : rl.n;
  const unsigned lane = threadIdx.x & 31u;
  bool exhausted = false;
  for (;;) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(kFull, !active);
      if (need) {
        const int leader = __ffs(need) - 1;
        const unsigned cnt = (unsigned)__popc(need);
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(queue, cnt);
        base = __shfl_sync(kFull, base, leader);
        if (base + cnt >= n) exhausted = true;
        if (!active) {
          const unsigned idx = base + (unsigned)__popc(need & ((1u << lane) - 1u));
          if (idx < n) {
            const uint32_t pix = rl.pix ? rl.pix[idx] : idx;
            out_slot = rl.slot ? rl.slot[idx] : idx;
            active = mode.start(f, pix, out_slot, fb);
          }
        }
      }
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    KT_ROLLED
    for (int s = -1; s < ModeT::kSlots; ++s) {
      const bool part = active && (s >= 0 || mode.needs_k1());
      if (s < 0 && !__any_sync(kFull, part)) continue;
      if (part) {
        RayResult res;
        if (mode.slot(f, s, &res)) {
          write_result(out, out_slot, res);
          active = false;
        }
      }
    }
  }
}

template <class ModeT>
static cudaError_t shape_for(int device, LaunchShape* shape) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  const int block = Shape<ModeT>::kBlock;
  const size_t smem = smem_bytes<ModeT>(block);
  e = cudaFuncSetAttribute(k_trace<ModeT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace<ModeT>, block, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  shape->block = block;
  shape->grid = sms * per_sm;
  shape->smem = smem;
  return cudaSuccess;
}

cudaError_t launch_shape(Mode mode, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4: return shape_for<ModeBLRk4>(device, shape);
    case kModeBLDopri5: return shape_for<ModeBLDopri5>(device, shape);
    case kModeKSRk4: return shape_for<ModeKSRk4>(device, shape);
    case kModeBundle: return shape_for<ModeBundle>(device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_trace(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                         uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                         cudaStream_t stream) {
  switch (mode) {
    case kModeBLRk4: k_trace<ModeBLRk4><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeBLDopri5: k_trace<ModeBLDopri5><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeKSRk4: k_trace<ModeKSRk4><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeBundle: k_trace<ModeBundle><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ---- colour ------------------------------------------------------------------

// colorize_buffer (main.cpp:1817-1866), blackbody palette.  The reference
// colours from float32 GeoPixel fields; the same rounding is applied here.
__global__ void k_colorize(const ColourConst cc, int64_t n, const uint8_t* __restrict__ outcome,
                           const double* __restrict__ r, const double* __restrict__ red,
                           const double* __restrict__ magnif, const double* __restrict__ th_esc,
                           const double* __restrict__ ph_esc, const uint8_t* __restrict__ bg,
                           int bg_w, int bg_h, uint8_t* __restrict__ rgb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint8_t c[3] = {0, 0, 0};
    const int oc = outcome[i];
    if (oc == kOutDisk) {
      disk_colour(cc, (double)(float)r[i], (double)(float)red[i], (double)(float)magnif[i], c);
    } else if (oc == kOutEscaped && bg != nullptr) {
      bg_sample(bg, bg_w, bg_h, (double)(float)th_esc[i], (double)(float)ph_esc[i], c);
    }
    rgb[3 * i + 0] = c[0];
    rgb[3 * i + 1] = c[1];
    rgb[3 * i + 2] = c[2];
  }
}

cudaError_t launch_colorize(const ColourConst& cc, int64_t n, const uint8_t* outcome,
                            const double* r, const double* red, const double* magnif,
                            const double* th_esc, const double* ph_esc, const uint8_t* bg,
                            int bg_w, int bg_h, uint8_t* rgb, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int block = 256;
  int64_t grid = (n + block - 1) / block;
  if (grid > 148 * 32) grid = 148 * 32;
  k_colorize<<<(int)grid, block, 0, stream>>>(cc, n, outcome, r, red, magnif, th_esc, ph_esc, bg,
                                              bg_w, bg_h, rgb);
  return cudaGetLastError();
}

// ---- FP64 pipe probe -----------------------------------------------------------

// Eight independent dependent-FMA chains per thread: measures the FP64 FMA
// issue rate the trace kernels are bounded by (2 flops per FMA).
__global__ void k_fp64_probe(double* out, int n_iter) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-9, a2 = a0 + 2e-9, a3 = a0 + 3e-9;
  double a4 = a0 + 4e-9, a5 = a0 + 5e-9, a6 = a0 + 6e-9, a7 = a0 + 7e-9;
  const double m = 0.999999999, c = 1e-12;
  for (int i = 0; i < n_iter; ++i) {
    a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
    a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
  }
  const double s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}

cudaError_t launch_fp64_probe(double* out, int n_iter, int grid, int block, cudaStream_t stream) {
  k_fp64_probe<<<grid, block, 0, stream>>>(out, n_iter);
  return cudaGetLastError();
}

}  // namespace kt
