// kt_trace_kernel.cuh -- the persistent trace loop, shared by the exact
// (kt_kernels.cu) and the mixed-precision (kt_mixed.cu) kernels.
//
// One CUDA thread carries one ray at a time through a per-ray machine
// (kt_machines.cuh); the 32 rays of a warp advance through the slots of an
// adaptive attempt in lockstep, one Hamiltonian right-hand side per slot.
// At every attempt boundary the lanes whose rays finished take new rays from
// a device queue (one atomicAdd per warp for all its idle lanes).  Rays
// differ in length by 3-50x, so refilling keeps the FP64 pipes busy until
// the queue runs dry; the grid is sized to the resident capacity of the GPU
// (persistent kernel).  Ray machines live in shared memory; results go out
// as SoA.
//
// The kernels do no waiting on other threads: the only inter-thread
// operation is the warp-synchronous refill and the queue atomic.  Every ray
// stops after at most max_steps accepted steps with at most 65 rejected
// attempts each (the reference's limits), so every loop ends.
#pragma once

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

template <class ModeT>
constexpr size_t smem_bytes(int block) {
  return sizeof(SmemRecord<typename ModeT::Machine>) * (size_t)block;
}

// Modes whose slot() may finish a ray without a result (handed to the
// fallback list: RayResult::outcome < 0); specialised where that happens.
template <class ModeT> struct Defers { static constexpr bool value = false; };

// Launch shape per mode: threads per block, minimum resident blocks (the
// register cap) and the refill threshold -- idle lanes of a warp take new
// rays only when at least kRefill lanes are idle (or the warp is empty).
// 128-thread blocks and refill at every idle lane by default; a mode may
// specialise this (see kt_kernels.cu, kt_mixed.cu).
template <class ModeT> struct Shape { static constexpr int kBlock = 128, kMinBlocks = 1, kRefill = 1; };
// ---- the persistent loop ---------------------------------------------------
// One iteration of the outer loop is one adaptive attempt for every ray of
// the warp.  At its start, idle lanes take new rays from the queue (one
// atomicAdd per warp).  Slot -1 runs only if some lane needs it (new rays,
// f at the end of an accepted step); slots 0..kSlots-1 run for every active
// lane.  All lanes of the warp see the same slot index, so the bookkeeping
// after each RHS runs converged; a lane whose ray ends mid-attempt idles to
// the end of the attempt.

template <class ModeT>
__global__ void __launch_bounds__(Shape<ModeT>::kBlock, Shape<ModeT>::kMinBlocks) k_trace(const __grid_constant__ Frame f, const OutSoA out, const RayList rl,
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
      if (need && (Shape<ModeT>::kRefill <= 1 || need == kFull ||
                   __popc(need) >= Shape<ModeT>::kRefill)) {
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
            active = mode.start(f, pix, out_slot, pix, fb);
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
          if (!Defers<ModeT>::value || res.outcome >= 0) write_result(out, out_slot, res);
          active = false;
        }
      }
    }
  }
}

// ---- two lanes per ray ------------------------------------------------------
// Pair modes: lanes 2i and 2i+1 of a warp carry one ray, 16 rays per warp.
// The mode's slot() splits the right-hand side between the two lanes with
// the same instructions on lane-dependent inputs (no divergence) and one
// shuffle exchange; the ray machine (one shared-memory record per pair) is
// written by the even lane only, with __syncwarp over the slot's lanes
// between the reads of a slot and the writes of its bookkeeping, and after
// them.  Both lanes of a pair always share `active`, so idle lanes come in
// pairs and a pair's two lanes take the same queue index.  As in k_trace,
// there is no waiting on other warps: the barriers are warp-local.
template <class ModeT>
constexpr size_t smem_bytes_pair(int block) {
  return sizeof(SmemRecord<typename ModeT::Machine>) * (size_t)(block / 2);
}

template <class ModeT>
__global__ void __launch_bounds__(Shape<ModeT>::kBlock, Shape<ModeT>::kMinBlocks)
    k_trace_pair(const __grid_constant__ Frame f, const OutSoA out, const RayList rl,
                 uint32_t* __restrict__ queue, const Fallback fb) {
  extern __shared__ __align__(16) unsigned char smem[];
  using Rec = SmemRecord<typename ModeT::Machine>;
  ModeT mode;
  mode.m = &reinterpret_cast<Rec*>(smem)[threadIdx.x >> 1].m;
  bool active = false;
  uint32_t out_slot = 0;
  const uint32_t n = rl.n_dev ? *rl.n_dev : rl.n;
  const unsigned lane = threadIdx.x & 31u;
  const bool odd = (lane & 1u) != 0;
  bool exhausted = false;
  for (;;) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(kFull, !active);
      if (need && (need == kFull || __popc(need) >= Shape<ModeT>::kRefill)) {
        const int leader = __ffs(need) - 1;
        const unsigned cnt = (unsigned)__popc(need) >> 1;  // rays
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(queue, cnt);
        base = __shfl_sync(kFull, base, leader);
        if (base + cnt >= n) exhausted = true;
        if (!active) {
          const unsigned idx = base + ((unsigned)__popc(need & ((1u << lane) - 1u)) >> 1);
          if (idx < n) {
            const uint32_t pix = rl.pix ? rl.pix[idx] : idx;
            out_slot = rl.slot ? rl.slot[idx] : idx;
            if (!odd) mode.start(f, pix, out_slot, pix, fb);
            active = true;
          }
        }
      }
      __syncwarp();  // new records written by the even lanes are visible to their partners
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    KT_ROLLED
    for (int s = -1; s < ModeT::kSlots; ++s) {
      const bool part = active && (s >= 0 || mode.needs_k1());
      const unsigned pmask = __ballot_sync(kFull, part);
      if (s < 0 && !pmask) continue;
      if (part) {
        RayResult res;
        if (mode.slot(f, s, &res, odd, pmask)) {
          if (!odd) write_result(out, out_slot, res);
          active = false;
        }
      }
    }
  }
}

template <class ModeT>
static cudaError_t shape_for_pair(int device, LaunchShape* shape) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  const int block = Shape<ModeT>::kBlock;
  const size_t smem = smem_bytes_pair<ModeT>(block);
  e = cudaFuncSetAttribute(k_trace_pair<ModeT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_pair<ModeT>, block, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  shape->block = block;
  shape->grid = sms * per_sm;
  shape->smem = smem;
  return cudaSuccess;
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

// ---- batches of frames -----------------------------------------------------
// Many frames (parameter sets, resolutions) in one persistent launch
// (BatchRays, kt_internal.h).  Each lane carries its own frame index; the
// frame constants are read from global memory through L1.  The loop is
// k_trace's, with a refill threshold and a binary search for a new ray's
// frame.

// Frame of batch ray g: the last k with offsets[k] <= g.
__device__ __forceinline__ int batch_frame_of(const BatchRays& br, uint64_t g) {
  int lo = 0, hi = br.n_frames - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (br.offsets[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <class ModeT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_trace_batch(const BatchRays br, uint32_t* __restrict__ queue, const Fallback fb) {
  extern __shared__ __align__(16) unsigned char smem[];
  using Rec = SmemRecord<typename ModeT::Machine>;
  ModeT mode;
  mode.m = &reinterpret_cast<Rec*>(smem)[threadIdx.x].m;
  bool active = false;
  int fi = 0;
  uint32_t pix = 0;
  const uint64_t n = br.n_dev ? (uint64_t)*br.n_dev : br.n;
  const unsigned lane = threadIdx.x & 31u;
  bool exhausted = false;
  for (;;) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(kFull, !active);
      const int idle = __popc(need);
      if (need && (idle >= br.refill_min || need == kFull)) {
        const int leader = __ffs(need) - 1;
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(queue, (unsigned)idle);
        base = __shfl_sync(kFull, base, leader);
        if ((uint64_t)base + (uint64_t)idle >= n) exhausted = true;
        if (!active) {
          const uint64_t idx = (uint64_t)base + (unsigned)__popc(need & ((1u << lane) - 1u));
          if (idx < n) {
            const uint32_t g = br.list ? br.list[idx] : (uint32_t)idx;
            fi = batch_frame_of(br, g);
            pix = (uint32_t)(g - br.offsets[fi]);
            active = mode.start(br.frames[fi], pix, pix, g, fb);
          }
        }
      }
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    const Frame& f = br.frames[fi];
    KT_ROLLED
    for (int s = -1; s < ModeT::kSlots; ++s) {
      const bool part = active && (s >= 0 || mode.needs_k1());
      if (s < 0 && !__any_sync(kFull, part)) continue;
      if (part) {
        RayResult res;
        if (mode.slot(f, s, &res)) {
          if (!Defers<ModeT>::value || res.outcome >= 0) write_result(br.outs[fi], pix, res);
          active = false;
        }
      }
    }
  }
}

// k_trace_batch with two lanes per ray (pair modes, as k_trace_pair): 16
// rays per warp; both lanes of a pair take the same batch ray.
template <class ModeT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
    k_trace_batch_pair(const BatchRays br, uint32_t* __restrict__ queue, const Fallback fb) {
  extern __shared__ __align__(16) unsigned char smem[];
  using Rec = SmemRecord<typename ModeT::Machine>;
  ModeT mode;
  mode.m = &reinterpret_cast<Rec*>(smem)[threadIdx.x >> 1].m;
  bool active = false;
  int fi = 0;
  uint32_t pix = 0;
  const uint64_t n = br.n_dev ? (uint64_t)*br.n_dev : br.n;
  const unsigned lane = threadIdx.x & 31u;
  const bool odd = (lane & 1u) != 0;
  bool exhausted = false;
  for (;;) {
    if (!exhausted) {
      const unsigned need = __ballot_sync(kFull, !active);
      const int idle = __popc(need);
      if (need && (idle >= br.refill_min || need == kFull)) {
        const int leader = __ffs(need) - 1;
        const unsigned cnt = (unsigned)idle >> 1;  // rays
        unsigned base = 0;
        if ((int)lane == leader) base = atomicAdd(queue, cnt);
        base = __shfl_sync(kFull, base, leader);
        if ((uint64_t)base + (uint64_t)cnt >= n) exhausted = true;
        if (!active) {
          const uint64_t idx =
              (uint64_t)base + ((unsigned)__popc(need & ((1u << lane) - 1u)) >> 1);
          if (idx < n) {
            const uint32_t g = br.list ? br.list[idx] : (uint32_t)idx;
            fi = batch_frame_of(br, g);
            pix = (uint32_t)(g - br.offsets[fi]);
            if (!odd) mode.start(br.frames[fi], pix, pix, g, fb);
            active = true;
          }
        }
      }
      __syncwarp();  // new records written by the even lanes are visible to their partners
    }
    if (!__any_sync(kFull, active)) {
      if (exhausted) break;
      continue;
    }
    const Frame& f = br.frames[fi];
    KT_ROLLED
    for (int s = -1; s < ModeT::kSlots; ++s) {
      const bool part = active && (s >= 0 || mode.needs_k1());
      const unsigned pmask = __ballot_sync(kFull, part);
      if (s < 0 && !pmask) continue;
      if (part) {
        RayResult res;
        if (mode.slot(f, s, &res, odd, pmask)) {
          if (!odd) write_result(br.outs[fi], pix, res);
          active = false;
        }
      }
    }
  }
}

template <class ModeT, int BLOCK, int MINB>
static cudaError_t batch_shape_pair_for(int device, LaunchShape* shape) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  const size_t smem = smem_bytes_pair<ModeT>(BLOCK);
  e = cudaFuncSetAttribute(k_trace_batch_pair<ModeT, BLOCK, MINB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_batch_pair<ModeT, BLOCK, MINB>,
                                                    BLOCK, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  shape->block = BLOCK;
  shape->grid = sms * per_sm;
  shape->smem = smem;
  return cudaSuccess;
}

template <class ModeT, int BLOCK, int MINB>
static cudaError_t batch_shape_for(int device, LaunchShape* shape) {
  int sms = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return e;
  const size_t smem = smem_bytes<ModeT>(BLOCK);
  e = cudaFuncSetAttribute(k_trace_batch<ModeT, BLOCK, MINB>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_batch<ModeT, BLOCK, MINB>,
                                                    BLOCK, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  shape->block = BLOCK;
  shape->grid = sms * per_sm;
  shape->smem = smem;
  return cudaSuccess;
}

// One case per entry of kBatchBlock / kBatchMinBlocks (kt_internal.h).
template <class ModeT>
static cudaError_t batch_shape(int variant, int device, LaunchShape* s) {
  switch (variant) {
    case 0: return batch_shape_for<ModeT, 64, 9>(device, s);
    case 1: return batch_shape_for<ModeT, 128, 1>(device, s);
    case 2: return batch_shape_for<ModeT, 64, 12>(device, s);
  }
  return cudaErrorInvalidValue;
}

template <class ModeT>
static cudaError_t batch_launch(int variant, const BatchRays& br, uint32_t* queue,
                                const Fallback& fb, const LaunchShape& s, cudaStream_t st) {
  switch (variant) {
    case 0: k_trace_batch<ModeT, 64, 9><<<s.grid, s.block, s.smem, st>>>(br, queue, fb); break;
    case 1: k_trace_batch<ModeT, 128, 1><<<s.grid, s.block, s.smem, st>>>(br, queue, fb); break;
    case 2: k_trace_batch<ModeT, 64, 12><<<s.grid, s.block, s.smem, st>>>(br, queue, fb); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace kt
