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
  kModeBundleMixed = 7,
  kModeSepRk4 = 8,
  kNumModes = 9
};

// Kernel mode of a prepared frame (and of the BL pass over the rays its
// kernel hands back: KS rays whose initialisation failed, separable-Kerr
// rays that gave up).
inline Mode frame_mode(const Frame& f) {
  const bool mixed = f.precision == 1;
  if (f.solver == 1) return kModeSepRk4;
  if (f.bundles) return mixed ? kModeBundleMixed : kModeBundle;
  if (f.chart == 0) return mixed ? kModeKSRk4Mixed : kModeKSRk4;
  if (f.intg == 1) return mixed ? kModeBLDopri5Mixed : kModeBLDopri5;
  return mixed ? kModeBLRk4Mixed : kModeBLRk4;
}
inline Mode fallback_mode(const Frame& f) {
  const bool mixed = f.precision == 1;
  // trace_single_separable_kerr falls back to RK4 step doubling whatever the
  // integrator (main.cpp:582-583, 612, 646)
  if (f.solver == 1) return kModeBLRk4;
  if (f.intg == 1) return mixed ? kModeBLDopri5Mixed : kModeBLDopri5;
  return mixed ? kModeBLRk4Mixed : kModeBLRk4;
}
inline bool is_ks_mode(Mode m) { return m == kModeKSRk4 || m == kModeKSRk4Mixed; }
inline bool is_mixed_mode(Mode m) { return m >= kModeBLRk4Mixed && m <= kModeBundleMixed; }
// Modes whose kernel may hand rays to a second, BL launch (fallback list).
inline bool has_fallback(Mode m) { return is_ks_mode(m) || m == kModeSepRk4; }

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

// Elliptic-closed solver: after the standard trace of rl into out, the
// closed-form disk hits replace the rays the standard tracer did not end at
// the horizon.
cudaError_t launch_elliptic(const Frame& f, const OutSoA& out, const RayList& rl, cudaStream_t stream);
// Its fallback reason per pixel of the frame (n = width x height).
cudaError_t launch_elliptic_reasons(const Frame& f, uint32_t n, uint8_t* reason, cudaStream_t stream);

// Colour pass: SoA -> RGB8.
cudaError_t launch_colorize(const ColourConst& cc, int64_t n, const uint8_t* outcome,
                            const double* r, const double* red, const double* magnif,
                            const double* phi_disk, const double* th_esc, const double* ph_esc,
                            const uint8_t* bg,
                            int bg_w, int bg_h, uint8_t* rgb, cudaStream_t stream);

// Camera supersampling: the traced passes as [spp][n] arrays, coloured and
// averaged in linear light into rgb (3 n bytes) by one kernel.
struct SppPasses {
  const uint8_t* outcome;
  const double *r, *red, *magnif, *phi_disk, *th_esc, *ph_esc;
};
cudaError_t launch_spp_colorize(const ColourConst& cc, int64_t n, int spp, const SppPasses& P,
                                const uint8_t* bg, int bg_w, int bg_h, double gamma, uint8_t* rgb,
                                cudaStream_t stream);

// Mixed-precision kernels (kt_mixed.cu).
cudaError_t launch_shape_mixed(Mode mode, int device, LaunchShape* shape);
cudaError_t launch_trace_mixed(Mode mode, const Frame& f, const OutSoA& out, const RayList& rl,
                               uint32_t* queue, const Fallback& fb, const LaunchShape& shape,
                               cudaStream_t stream);

// ---- batches of frames (k_trace_batch, kt_trace_kernel.cuh) ---------------
// Ray g of a batch is pixel g - offsets[k] of frame k, where offsets[k] <= g
// < offsets[k+1]; frames[k] and outs[k] are that frame's constants and
// result arrays.  Rays traced: list[0..n) (batch ray indices) or 0..n-1 when
// list is NULL; the count is *n_dev when n_dev is set.  Idle lanes of a warp
// take new rays only when at least `refill_min` lanes are idle (or the warp
// is empty), so more lanes share the new rays' first RHS evaluations.
struct BatchRays {
  const Frame* frames;
  const OutSoA* outs;
  const uint64_t* offsets;
  int n_frames;
  int refill_min;
  const uint32_t* list;
  const uint32_t* n_dev;
  uint64_t n;
  // some frame may run the mixed tracer's FP32 right-hand side (a finite
  // r_fp32): selects the mixed kernels that carry the FP32 branch
  bool fp32 = true;
};

// Launch-shape variants the batch autotuner chooses from: (threads per
// block, minimum resident blocks per SM).  The second number sets the
// register cap: 65536 / (threads x blocks) per thread, rounded down to the
// allocation granule (112 for 64 x 9, 80 for 64 x 12, none for 128 x 1).
constexpr int kBatchVariants = 4;
constexpr int kBatchBlock[kBatchVariants] = {64, 128, 64, 128};
constexpr int kBatchMinBlocks[kBatchVariants] = {9, 1, 12, 3};
// Variant 3 runs two lanes per ray (16 rays per warp); only the FP64 bundle
// kernel has that form.
constexpr int kBatchPairVariant = 3;
constexpr int kBatchRaysPerWarp[kBatchVariants] = {32, 32, 32, 16};
inline bool batch_variant_ok(Mode m, int v) {
  return v >= 0 && v < kBatchVariants && (v != kBatchPairVariant || m == kModeBundle);
}

// Shape (grid at full occupancy) and launch of variant `variant` of `mode`.
// The KS fallback list receives batch ray indices.
cudaError_t batch_shape(Mode mode, int variant, int device, LaunchShape* shape);
cudaError_t launch_batch(Mode mode, int variant, const BatchRays& br, uint32_t* queue,
                         const Fallback& fb, const LaunchShape& s, cudaStream_t st);
cudaError_t batch_shape_mixed(Mode mode, int variant, int device, LaunchShape* shape);
cudaError_t launch_batch_mixed(Mode mode, int variant, const BatchRays& br, uint32_t* queue,
                               const Fallback& fb, const LaunchShape& s, cudaStream_t st);

// Centre-out ray order (kt_kernels.cu): base + the W x H frame's pixels in
// rings about the image centre, innermost first, in blocks of 8 x 4 pixels
// within a ring, into `list` (W*H words); `scratch` holds
// ring_scratch_words(W*H) words.
// Whole frames of at least kOrderMinPixels pixels are traced in this order,
// and every frame of a batch (base = the frame's first ray of its group).
constexpr int kOrderClasses = 512;
constexpr uint32_t kOrderMinPixels = 1u << 16;
// pixels per tile of the counting sort: at least 4096, at most 1024 tiles
constexpr uint32_t ring_tile(uint64_t n) {
  uint64_t t = (n + 1023) / 1024;
  t = (t + 31) / 32 * 32;
  return (uint32_t)(t < 4096 ? 4096 : t);
}
constexpr size_t ring_scratch_words(uint64_t n) {
  const uint32_t tile = ring_tile(n);
  return (size_t)kOrderClasses * (size_t)((n + tile - 1) / tile);
}
cudaError_t launch_ring_order(int W, int H, uint32_t base, uint32_t* scratch, uint32_t* list,
                              cudaStream_t stream);

// The order's geometry and its input order (ring_item), shared by the sort
// kernels and their host check.
struct RingGeom {
  float cx, cy, inv_w;
  int W, H, Wt, Ht;   // frame; the top-left region covered by whole 8 x 4 blocks
  uint32_t n_int;     // its pixels, Wt * Ht
};

KT_HD RingGeom ring_geom(int W, int H) {
  RingGeom g;
  g.cx = 0.5f * (float)(W - 1);
  g.cy = 0.5f * (float)(H - 1);
  const float rmax = sqrtf(g.cx * g.cx + g.cy * g.cy) + 1.0f;
  const float w = fmaxf(4.0f, rmax / (float)kOrderClasses);
  g.inv_w = 1.0f / w;
  g.W = W;
  g.H = H;
  g.Wt = W / 8 * 8;
  g.Ht = H / 4 * 4;
  g.n_int = (uint32_t)g.Wt * (uint32_t)g.Ht;
  return g;
}

KT_HD int ring_of(const RingGeom& g, float x, float y) {
  const float dx = x - g.cx, dy = y - g.cy;
  const int c = (int)(sqrtf(dx * dx + dy * dy) * g.inv_w);
  return c < kOrderClasses - 1 ? c : kOrderClasses - 1;
}

// Item e (0 <= e < W*H) of the sort's input order, a one-to-one map onto
// the pixels: the 8 x 4 blocks of the top-left Wt x Ht region block by block
// (row-major over blocks, each block's 32 pixels row-major), a block in the
// ring of its centre, so that a warp's 32 rays are one compact block; then
// the right strip (x >= Wt, every row) and the bottom strip (y >= Ht,
// x < Wt) pixel by pixel, each pixel in its own ring.  Measured on the 720p
// headline frame: 54.4 ms against 58.2 with single pixels placed in the
// rings in row-major order (8 x 8 blocks 54.3, 4 x 8 54.7, 16 x 2 55.1;
// pixels sorted by angle within each ring 54.6; row-major order 64.5).
KT_HD void ring_item(const RingGeom& g, uint32_t e, uint32_t* p, int* c) {
  if (e < g.n_int) {
    const uint32_t bw = (uint32_t)g.Wt / 8u;
    const uint32_t blk = e >> 5, j = e & 31u;
    const uint32_t bx = blk % bw, by = blk / bw;
    const uint32_t x = bx * 8u + (j & 7u), y = by * 4u + (j >> 3);
    *p = y * (uint32_t)g.W + x;
    *c = ring_of(g, (float)(bx * 8u) + 3.5f, (float)(by * 4u) + 1.5f);
    return;
  }
  const uint32_t r = e - g.n_int;
  const uint32_t wr = (uint32_t)(g.W - g.Wt);
  const uint32_t n_right = wr * (uint32_t)g.H;
  uint32_t x, y;
  if (r < n_right) {
    y = r / wr;
    x = (uint32_t)g.Wt + r % wr;
  } else {
    const uint32_t r2 = r - n_right;
    y = (uint32_t)g.Ht + r2 / (uint32_t)g.Wt;
    x = r2 % (uint32_t)g.Wt;
  }
  *p = y * (uint32_t)g.W + x;
  *c = ring_of(g, (float)x, (float)y);
}


// FP64 throughput probe: n_iter dependent FMA chains per thread.
cudaError_t launch_fp64_probe(double* out, int n_iter, int grid, int block, cudaStream_t stream);
// Operation-cost probe (op 0 FMA, 1 division, 2 ktm_div3, 3 sqrt, 4 ktm_sincos,
// 5 ktm_pow), eight recurrences per thread.
cudaError_t launch_op_probe(int op, double* out, int n_iter, int grid, int block, cudaStream_t stream);

}  // namespace kt
