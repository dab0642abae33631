// kt_kernels.cu -- the exact (bit-faithful FP64) trace kernels for sm_100a.
//
// Compiled with --fmad=false: every multiply and add of the reference's
// arithmetic is rounded separately, as in the reference's CPU build.
#include "kt_elliptic.cuh"
#include "kt_trace_kernel.cuh"

namespace kt {

struct ModeBLRk4 {
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
    bl_rhs(f.g, y[0], y[1], y[2], y[3], m->pt, m->pphi, k);
    return m->consume(f, s, k, res);
  }
};

struct ModeBLDopri5 {
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
                                        uint32_t fb_key, const Fallback& fb) {
    if (m->init(f, camera_ray(f, pix))) return true;
    // init_ks_state failed: the ray is traced in the BL chart by a second
    // launch over the fallback list.
    const uint32_t i = atomicAdd(fb.count, 1u);
    fb.pix[i] = fb_key;
    if (fb.slot) fb.slot[i] = out_slot;
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
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, uint32_t, const Fallback&) {
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

// Bundles with two lanes per ray (k_trace_pair): the right-hand side is
// split by bundle_rhs_half, the halves swapped with one shuffle each, and
// bundle_rhs_combine assembles it in bundle_rhs's order (bit-identical); the
// even lane runs the machine's bookkeeping.
__device__ __forceinline__ void bundle_rhs_paired(const Metric& g, const double y[4], double pt,
                                                  double pphi, const double W[8], double k[5],
                                                  double kW[8], bool odd, unsigned pmask) {
  BundleHalf me, other;
  bundle_rhs_half(g, y[0], y[1], y[2], y[3], pt, pphi, odd, &me);
#pragma unroll
  for (int t = 0; t < 3; ++t)
#pragma unroll
    for (int j = 0; j < 5; ++j) other.h5[t][j] = __shfl_xor_sync(pmask, me.h5[t][j], 1);
#pragma unroll
  for (int i = 0; i < 4; ++i) other.h1[i] = __shfl_xor_sync(pmask, me.h1[i], 1);
  // the even lane's view (the odd lane's result is not used)
  bundle_rhs_combine(me, other, y[0], y[2], y[3], W, k, kW);
}

struct ModeBundlePair {
  using Machine = Bundle;
  static constexpr int kSlots = Bundle::kSlots;
  Bundle* m;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t, uint32_t, const Fallback&) {
    m->init(f, (int)(pix % (uint32_t)f.cam.W), (int)(pix / (uint32_t)f.cam.W));
    return true;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res, bool odd,
                                       unsigned pmask) {
    double y[4], yW[8], k[5], kW[8];
    m->input(s, y, yW);
    bundle_rhs_paired(f.g, y, m->pt, m->pphi, yW, k, kW, odd, pmask);
    __syncwarp(pmask);  // both lanes have read the record
    int done = 0;
    if (!odd) done = m->consume(f, s, k, kW, res) ? 1 : 0;
    __syncwarp(pmask);  // the even lane's updates are visible to the odd lane
    return __shfl_sync(pmask, done, (int)((threadIdx.x & 31u) & ~1u)) != 0;
  }
};

// Separable Kerr (semi-analytic solver): rays that give up are appended to
// the fallback list for the BL RK4 launch and write no result here.
struct ModeSepRk4 {
  using Machine = SepRk4;
  static constexpr int kSlots = SepRk4::kSlots;
  SepRk4* m;
  Fallback fb;
  __device__ __forceinline__ bool needs_k1() const { return m->needs_k1(); }
  __device__ __forceinline__ void hand_back(uint32_t key, uint32_t out_slot) const {
    const uint32_t i = atomicAdd(fb.count, 1u);
    fb.pix[i] = key;
    if (fb.slot) fb.slot[i] = out_slot;
  }
  __device__ __forceinline__ bool start(const Frame& f, uint32_t pix, uint32_t out_slot,
                                        uint32_t fb_key, const Fallback& fbl) {
    fb = fbl;
    if (m->init(f, camera_ray(f, pix), fb_key, out_slot)) return true;
    hand_back(fb_key, out_slot);
    return false;
  }
  __device__ __forceinline__ bool slot(const Frame& f, int s, RayResult* res) {
    double y[2], k[3];
    m->input(s, y);
    const bool ok = m->rhs(s, y, k);
    if (!m->consume(f, s, k, ok, res)) return false;
    if (m->fallback) {
      hand_back(m->fb_key, m->out_slot);
      res->outcome = -1;
    }
    return true;
  }
};

template <> struct Defers<ModeSepRk4> { static constexpr bool value = true; };

// Launch shape per mode, measured on B200 (720p config-2 frame, BL chart
// DOPRI5 and RK4; 720p Kerr KS frame; 1080p config-3 bundles): the BL and KS
// single-ray kernels run best as 64-thread blocks capped at 113 registers
// (9 blocks per SM), the bundle kernel as 128-thread blocks.  Refilling a
// warp only once all its lanes are idle (kRefill 32) keeps the 32 rays of a
// warp neighbouring pixels that start together: the camera set-up and the
// first slots run converged and the rays' step sequences stay alike, which
// outweighs the lanes idling at the end of each group of 32 (KS: 62 against
// 73 ms, BL RK4: 66 against 68, DOPRI5: equal; bundles best at 16).
template <> struct Shape<struct ModeBLRk4> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
#ifndef KT_BL_DOPRI5_MINB
#define KT_BL_DOPRI5_MINB 9
#endif
#ifndef KT_BL_DOPRI5_REFILL
#define KT_BL_DOPRI5_REFILL 32
#endif
#ifndef KT_BL_DOPRI5_BLOCK
#define KT_BL_DOPRI5_BLOCK 64
#endif
template <> struct Shape<struct ModeBLDopri5> {
  static constexpr int kBlock = KT_BL_DOPRI5_BLOCK, kMinBlocks = KT_BL_DOPRI5_MINB,
                       kRefill = KT_BL_DOPRI5_REFILL;
};
template <> struct Shape<struct ModeKSRk4> { static constexpr int kBlock = 64, kMinBlocks = 9, kRefill = 32; };
template <> struct Shape<struct ModeBundle> { static constexpr int kBlock = 128, kMinBlocks = 1, kRefill = 16; };
// Paired bundles: 64 rays per 128-thread block; kRefill counts lanes.
#ifndef KT_BUNDLE_PAIR_BLOCK
#define KT_BUNDLE_PAIR_BLOCK 128
#endif
#ifndef KT_BUNDLE_PAIR_MINB
#define KT_BUNDLE_PAIR_MINB 3
#endif
#ifndef KT_BUNDLE_PAIR_REFILL
#define KT_BUNDLE_PAIR_REFILL 8
#endif
template <> struct Shape<ModeBundlePair> {
  static constexpr int kBlock = KT_BUNDLE_PAIR_BLOCK, kMinBlocks = KT_BUNDLE_PAIR_MINB,
                       kRefill = KT_BUNDLE_PAIR_REFILL;
};

cudaError_t launch_shape(Mode mode, int device, LaunchShape* shape) {
  if (is_mixed_mode(mode)) return launch_shape_mixed(mode, device, shape);
  switch (mode) {
    case kModeBLRk4: return shape_for<ModeBLRk4>(device, shape);
    case kModeBLDopri5: return shape_for<ModeBLDopri5>(device, shape);
    case kModeKSRk4: return shape_for<ModeKSRk4>(device, shape);
    case kModeBundle: return shape_for_pair<ModeBundlePair>(device, shape);
    case kModeSepRk4: return shape_for<ModeSepRk4>(device, shape);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_trace(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                         uint32_t* queue, const Fallback& fb, const LaunchShape& s,
                         cudaStream_t stream) {
  if (is_mixed_mode(mode)) return launch_trace_mixed(mode, f, out, rl, queue, fb, s, stream);
  switch (mode) {
    case kModeBLRk4: k_trace<ModeBLRk4><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeBLDopri5: k_trace<ModeBLDopri5><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeKSRk4: k_trace<ModeKSRk4><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeBundle: k_trace_pair<ModeBundlePair><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    case kModeSepRk4: k_trace<ModeSepRk4><<<s.grid, s.block, s.smem, stream>>>(f, out, rl, queue, fb); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t batch_shape(Mode mode, int variant, int device, LaunchShape* shape) {
  switch (mode) {
    case kModeBLRk4: return batch_shape<ModeBLRk4>(variant, device, shape);
    case kModeBLDopri5: return batch_shape<ModeBLDopri5>(variant, device, shape);
    case kModeKSRk4: return batch_shape<ModeKSRk4>(variant, device, shape);
    case kModeBundle:
      if (variant == kBatchPairVariant)
        return batch_shape_pair_for<ModeBundlePair, kBatchBlock[kBatchPairVariant],
                                    kBatchMinBlocks[kBatchPairVariant]>(device, shape);
      return batch_shape<ModeBundle>(variant, device, shape);
    case kModeSepRk4: return batch_shape<ModeSepRk4>(variant, device, shape);
    default: return batch_shape_mixed(mode, variant, device, shape);
  }
}

cudaError_t launch_batch(Mode mode, int variant, const BatchRays& br, uint32_t* queue,
                         const Fallback& fb, const LaunchShape& s, cudaStream_t st) {
  switch (mode) {
    case kModeBLRk4: return batch_launch<ModeBLRk4>(variant, br, queue, fb, s, st);
    case kModeBLDopri5: return batch_launch<ModeBLDopri5>(variant, br, queue, fb, s, st);
    case kModeKSRk4: return batch_launch<ModeKSRk4>(variant, br, queue, fb, s, st);
    case kModeBundle:
      if (variant == kBatchPairVariant) {
        k_trace_batch_pair<ModeBundlePair, kBatchBlock[kBatchPairVariant],
                           kBatchMinBlocks[kBatchPairVariant]><<<s.grid, s.block, s.smem, st>>>(
            br, queue, fb);
        return cudaGetLastError();
      }
      return batch_launch<ModeBundle>(variant, br, queue, fb, s, st);
    case kModeSepRk4: return batch_launch<ModeSepRk4>(variant, br, queue, fb, s, st);
    default: return launch_batch_mixed(mode, variant, br, queue, fb, s, st);
  }
}

// ---- elliptic-closed solver -------------------------------------------------

// After the standard trace of the same rays (the reference's fallback and its
// horizon-precedence check, main.cpp:1227-1295): a ray whose closed-form
// equator crossing lies in the disk, and which the standard tracer did not
// end at the horizon, becomes that disk hit.  One thread per ray.
__global__ void __launch_bounds__(128) k_elliptic(const __grid_constant__ Frame f, const OutSoA out,
                                                  const RayList rl) {
  const uint32_t n = rl.n_dev ? *rl.n_dev : rl.n;
  for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
    const uint32_t pix = rl.pix ? rl.pix[idx] : idx;
    const uint32_t slot = rl.slot ? rl.slot[idx] : idx;
    if (out.outcome[slot] == kOutHorizon) continue;
    double r, g;
    int why;
    if (!elliptic_closed_form(f, camera_ray(f, pix), &r, &g, &why)) continue;
    // TraceResult{DISK_HIT, r, g}: phi_disk and the escape angles stay 0
    out.outcome[slot] = (uint8_t)kOutDisk;
    out.r[slot] = r;
    out.red[slot] = g;
    out.magnif[slot] = 1.0;
    out.phi_disk[slot] = 0.0;
    out.th_esc[slot] = 0.0;
    out.ph_esc[slot] = 0.0;
  }
}

// The closed form's fallback reason per pixel (the reference's
// --debug-elliptic tag, main.cpp:2111-2121): 0 where it places the crossing
// in the disk, else the EllipticFallbackReason.
__global__ void __launch_bounds__(128) k_elliptic_reasons(const __grid_constant__ Frame f, uint32_t n,
                                                          uint8_t* __restrict__ reason) {
  for (uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x; pix < n; pix += gridDim.x * blockDim.x) {
    double r, g;
    int why = kEfNone;
    elliptic_closed_form(f, camera_ray(f, pix), &r, &g, &why);
    reason[pix] = (uint8_t)why;
  }
}

cudaError_t launch_elliptic_reasons(const Frame& f, uint32_t n, uint8_t* reason, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  uint64_t grid = ((uint64_t)n + 127) / 128;
  if (grid > 148 * 8) grid = 148 * 8;
  k_elliptic_reasons<<<(int)grid, 128, 0, stream>>>(f, n, reason);
  return cudaGetLastError();
}

cudaError_t launch_elliptic(const Frame& f, const OutSoA& out, const RayList& rl, cudaStream_t stream) {
  const uint64_t n = rl.n_dev ? (uint64_t)0xffffffffu : rl.n;
  if (n == 0) return cudaSuccess;
  uint64_t grid = (n + 127) / 128;
  if (grid > 148 * 8) grid = 148 * 8;
  k_elliptic<<<(int)grid, 128, 0, stream>>>(f, out, rl);
  return cudaGetLastError();
}

// ---- centre-out ray order ----------------------------------------------------
// The camera looks at the black hole, so the image centre holds the shadow
// and the critical curve, whose rays are the longest, and the edges hold
// short escaping rays.  A whole frame is traced in rings about the image
// centre, innermost first, in blocks of 8 x 4 pixels (ring_item): the long
// rays start early and the persistent kernel's tail is short, while a
// warp's 32 rays are one compact block of neighbours.  Each ray's
// arithmetic does not depend on when or beside which rays it runs, so the
// results are bit for bit those of the row-major trace.  Rings are 4
// pixels wide, wider where the frame needs more than kOrderClasses of them.
// The list is a stable counting sort of ring_item's order: per-tile ring
// counts, one exclusive scan in (ring, tile) order, then each tile scattered
// in item order (a "tile" here is the sort's chunk of items).

// counts[c * tiles + t]: pixels of ring c in tile t (tile = `tile` pixels)
__global__ void k_ring_count(int W, int H, uint32_t tile, uint32_t tiles, uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[kOrderClasses];
  for (int i = threadIdx.x; i < kOrderClasses; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const RingGeom g = ring_geom(W, H);
  const uint32_t n = (uint32_t)W * (uint32_t)H;
  const uint32_t t = blockIdx.x;
  const uint32_t end = min(n, (t + 1) * tile);
  for (uint32_t e = t * tile + threadIdx.x; e < end; e += blockDim.x) {
    uint32_t p;
    int c;
    ring_item(g, e, &p, &c);
    atomicAdd(&h[c], 1u);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < kOrderClasses; c += blockDim.x) counts[(uint32_t)c * tiles + t] = h[c];
}

// Exclusive scan of counts[0..m) in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_ring_scan(uint32_t* __restrict__ a, uint32_t m) {
  __shared__ uint32_t warp_sum[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  for (uint32_t base = 0; base < m; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = (i < m) ? a[i] : 0u;
    uint32_t x = v;  // inclusive warp scan
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, d);
      if ((int)lane >= d) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = warp_sum[lane];
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, s, d);
        if ((int)lane >= d) s += y;
      }
      warp_sum[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = carry + (warp ? warp_sum[warp - 1] : 0u) + (x - v);
    if (i < m) a[i] = before;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_sum[31];
    __syncthreads();
  }
}

// One warp per tile: the tile's pixels in order, each ring's in consecutive
// places from that ring's offset for the tile.
__global__ void k_ring_place(int W, int H, uint32_t tile, uint32_t tiles,
                             const uint32_t* __restrict__ offsets, uint32_t base,
                             uint32_t* __restrict__ list) {
  __shared__ uint32_t next[kOrderClasses];
  const uint32_t t = blockIdx.x;
  for (int c = threadIdx.x; c < kOrderClasses; c += 32) next[c] = offsets[(uint32_t)c * tiles + t];
  __syncwarp();
  const RingGeom g = ring_geom(W, H);
  const uint32_t n = (uint32_t)W * (uint32_t)H;
  const uint32_t end = min(n, (t + 1) * tile);
  const unsigned lane = threadIdx.x;
  for (uint32_t e0 = t * tile; e0 < end; e0 += 32) {
    const uint32_t e = e0 + lane;
    uint32_t p = 0;
    int c = -1;
    if (e < end) ring_item(g, e, &p, &c);
    const unsigned same = __match_any_sync(kFull, c);
    uint32_t at = 0;
    if (c >= 0) at = next[c] + (uint32_t)__popc(same & ((1u << lane) - 1u));
    __syncwarp();
    if (c >= 0) {
      list[at] = base + p;
      if ((int)lane == __ffs(same) - 1) next[c] += (uint32_t)__popc(same);
    }
    __syncwarp();
  }
}

cudaError_t launch_ring_order(int W, int H, uint32_t base, uint32_t* scratch, uint32_t* list,
                              cudaStream_t stream) {
  const uint64_t n = (uint64_t)W * (uint64_t)H;
  const uint32_t tile = ring_tile(n), tiles = (uint32_t)((n + tile - 1) / tile);
  k_ring_count<<<tiles, 256, 0, stream>>>(W, H, tile, tiles, scratch);
  k_ring_scan<<<1, 1024, 0, stream>>>(scratch, (uint32_t)kOrderClasses * tiles);
  k_ring_place<<<tiles, 32, 0, stream>>>(W, H, tile, tiles, scratch, base, list);
  return cudaGetLastError();
}

// ---- colour ------------------------------------------------------------------

// One pixel of colorize_buffer (main.cpp:1817-1866), both palettes.  The
// reference colours from float32 GeoPixel fields; the same rounding is
// applied here.
__device__ __forceinline__ void pixel_colour(const ColourConst& cc, int oc, double r, double red,
                                             double magnif, double phi_disk, double th_esc,
                                             double ph_esc, const uint8_t* __restrict__ bg, int bg_w,
                                             int bg_h, uint8_t c[3]) {
  c[0] = c[1] = c[2] = 0;
  if (oc == kOutDisk && cc.palette == 1) {
    disk_colour_interstellar(cc, (double)(float)r, (double)(float)phi_disk, (double)(float)red,
                             (double)(float)magnif, c);
  } else if (oc == kOutDisk) {
    disk_colour(cc, (double)(float)r, (double)(float)red, (double)(float)magnif, c);
  } else if (oc == kOutEscaped && bg != nullptr) {
    bg_sample(bg, bg_w, bg_h, (double)(float)th_esc, (double)(float)ph_esc, c);
  }
}

__global__ void k_colorize(const ColourConst cc, int64_t n, const uint8_t* __restrict__ outcome,
                           const double* __restrict__ r, const double* __restrict__ red,
                           const double* __restrict__ magnif, const double* __restrict__ phi_disk,
                           const double* __restrict__ th_esc,
                           const double* __restrict__ ph_esc, const uint8_t* __restrict__ bg,
                           int bg_w, int bg_h, uint8_t* __restrict__ rgb) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint8_t c[3];
    pixel_colour(cc, outcome[i], r[i], red[i], magnif[i], phi_disk[i], th_esc[i], ph_esc[i], bg,
                 bg_w, bg_h, c);
    rgb[3 * i + 0] = c[0];
    rgb[3 * i + 1] = c[1];
    rgb[3 * i + 2] = c[2];
  }
}

cudaError_t launch_colorize(const ColourConst& cc, int64_t n, const uint8_t* outcome,
                            const double* r, const double* red, const double* magnif,
                            const double* phi_disk, const double* th_esc, const double* ph_esc,
                            const uint8_t* bg,
                            int bg_w, int bg_h, uint8_t* rgb, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  const int block = 256;
  int64_t grid = (n + block - 1) / block;
  if (grid > 148 * 32) grid = 148 * 32;
  k_colorize<<<(int)grid, block, 0, stream>>>(cc, n, outcome, r, red, magnif, phi_disk, th_esc,
                                              ph_esc, bg, bg_w, bg_h, rgb);
  return cudaGetLastError();
}

// ---- camera supersampling ------------------------------------------------------

// render_image's camera_spp > 1 branch (main.cpp:2280-2321) after all passes
// are traced: per pixel, the colour of every pass, taken to linear light
// pow(clamp(c/255, 0, 1), gamma) and summed in pass order (the sum of the
// first pass is the value itself), then lround(255 pow(clamp(sum/n, 0, 1),
// 1/gamma)), lround's half-away-from-zero rounding written out for a
// non-negative value.  The 256 linear values of the 8-bit levels are
// computed once per block.
__global__ void k_spp_colorize(const ColourConst cc, int64_t n, int spp, const SppPasses P,
                               const uint8_t* __restrict__ bg, int bg_w, int bg_h, double gamma,
                               uint8_t* __restrict__ rgb) {
  __shared__ double lin[256];
  for (int c = threadIdx.x; c < 256; c += blockDim.x)
    lin[c] = ktm_pow(dclamp((double)c / 255.0, 0.0, 1.0), gamma);
  __syncthreads();
  const double inv_n = 1.0 / (double)spp;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < spp; ++s) {
      const int64_t j = (int64_t)s * n + i;
      uint8_t c[3];
      pixel_colour(cc, P.outcome[j], P.r[j], P.red[j], P.magnif[j], P.phi_disk[j], P.th_esc[j],
                   P.ph_esc[j], bg, bg_w, bg_h, c);
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) acc[ch] = (s == 0) ? lin[c[ch]] : acc[ch] + lin[c[ch]];
    }
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const double x = 255.0 * ktm_pow(dclamp(acc[ch] * inv_n, 0.0, 1.0), 1.0 / gamma);
      const double t = trunc(x);
      rgb[3 * i + ch] = (uint8_t)(int)((x - t >= 0.5) ? t + 1.0 : t);
    }
  }
}

cudaError_t launch_spp_colorize(const ColourConst& cc, int64_t n, int spp, const SppPasses& P,
                                const uint8_t* bg, int bg_w, int bg_h, double gamma, uint8_t* rgb,
                                cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  int64_t grid = (n + 255) / 256;
  if (grid > 148 * 16) grid = 148 * 16;
  k_spp_colorize<<<(int)grid, 256, 0, stream>>>(cc, n, spp, P, bg, bg_w, bg_h, gamma, rgb);
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

// Throughput of the operations the algorithmic flop count weights (division,
// x/3, square root, sincos, pow): eight independent recurrences per thread,
// each step one operation plus `kOpProbeExtra[op]` FMA-pipe operations that
// keep its argument in range (2.5/x; sqrt(3x); x/3 + 1; 1.2 + 0.3 sin x +
// 0.001 cos x; 0.3 + 0.5 x^-0.2).  Op 0 is the FMA chain of k_fp64_probe.
template <int OP>
__global__ void k_op_probe(double* out, int n_iter) {
  double v[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) v[j] = 1.0 + (threadIdx.x * 8 + j) * 1e-7;
  for (int i = 0; i < n_iter; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      double x = v[j];
      if (OP == 0) x = fma(x, 0.999999999, 1e-12);
      if (OP == 1) x = 2.5 / x;
      if (OP == 2) x = ktm_div3(x) + 1.0;
      if (OP == 3) x = sqrt(x * 3.0);
      if (OP == 4) {
        double sn, cs;
        ktm_sincos(x, &sn, &cs);
        x = fma(0.3, sn, fma(1e-3, cs, 1.2));
      }
      if (OP == 5) x = fma(0.5, ktm_pow(x, -0.2), 0.3);
      v[j] = x;
    }
  }
  const double s = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the recurrences alive
}

cudaError_t launch_op_probe(int op, double* out, int n_iter, int grid, int block, cudaStream_t stream) {
  switch (op) {
    case 0: k_op_probe<0><<<grid, block, 0, stream>>>(out, n_iter); break;
    case 1: k_op_probe<1><<<grid, block, 0, stream>>>(out, n_iter); break;
    case 2: k_op_probe<2><<<grid, block, 0, stream>>>(out, n_iter); break;
    case 3: k_op_probe<3><<<grid, block, 0, stream>>>(out, n_iter); break;
    case 4: k_op_probe<4><<<grid, block, 0, stream>>>(out, n_iter); break;
    case 5: k_op_probe<5><<<grid, block, 0, stream>>>(out, n_iter); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace kt
