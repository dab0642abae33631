/*
 * kerrtrace.h -- C ABI of the B200-native geodesic renderer.
 *
 * This is the drop-in boundary for the reference renderer's backend dispatch
 * (render_image, main.cpp:2209-2478).  The reference routes one frame either
 * to its CPU two-phase path (trace_geodesics main.cpp:2014-2206, then
 * colorize_buffer main.cpp:1817-1866) or to `cuda_render`
 * (gpu/cuda/tracer.cuh:23-26).  The entry points below replace both with
 * plain C: pointers, sizes and status codes, no C++ types, no exceptions.
 *
 *   kt_frame_desc   <- FrameParams (main.cpp:1885-1893) + IntegratorControls
 *                      (main.cpp:193-197) + trace_geodesics' arguments
 *                      (main.cpp:2014-2027): chart, integrator, bundles,
 *                      solver mode, pixel offsets, M, Q, Lambda.
 *   kt_frame_derive <- the per-frame host work of trace_geodesics
 *                      (main.cpp:2033-2082): chart fallback rules, r_horizon,
 *                      r_isco, disk bounds, escape radius, camera angles.
 *   kt_trace        <- trace_geodesics' per-pixel loop (main.cpp:2098-2183):
 *                      fills a per-pixel SoA (GeoPixel main.cpp:84-94, in
 *                      float64 instead of float32).
 *   kt_colorize     <- colorize_buffer (main.cpp:1817-1866) with the
 *                      blackbody palette (disk_colour main.cpp:1799-1814) and
 *                      the equirectangular background (main.cpp:153-170).
 *   kt_render_host  <- render_image's CPU branch (main.cpp:2468-2476):
 *                      trace + colorize, host buffers in and out.
 *   kt_kgeo_write / kt_kgeo_read <- save_kgeo / load_kgeo (main.cpp:96-137).
 *
 * Threading: a kt_context belongs to one host thread at a time.  Device
 * pointers passed to the asynchronous calls belong to the caller; the
 * context owns its scratch (queue counters) only.  Every call returns a
 * kt_status; kt_last_error() gives the message of the last failure.
 */
#ifndef KERRTRACE_H
#define KERRTRACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KT_ABI_VERSION 1

typedef enum kt_status {
  KT_OK = 0,
  KT_ERR_INVALID_ARGUMENT = 1, /* bad sizes, NaN parameters, NULL pointers */
  KT_ERR_UNSUPPORTED = 2,      /* a mode this backend does not run */
  KT_ERR_CUDA = 3,             /* a CUDA runtime call failed */
  KT_ERR_OUT_OF_MEMORY = 4,
  KT_ERR_NO_DEVICE = 5,
  KT_ERR_IO = 6,               /* .kgeo read/write failure */
  KT_ERR_INTERNAL = 7
} kt_status;

/* Coordinate chart (CoordinateChart, main.cpp:175). */
enum { KT_CHART_KS = 0, KT_CHART_BL = 1 };
/* Integrator (Integrator, geodesic.hpp:417). */
enum { KT_RK4_DOUBLING = 0, KT_DOPRI5 = 1 };
/* Ray solver (RaySolverMode, main.cpp:176): STANDARD, SEMI_ANALYTIC (the
 * separable Kerr tracer, main.cpp:436-703) and ELLIPTIC_CLOSED (the closed-
 * form disk crossing over the standard trace, main.cpp:705-1295), the last
 * two in FP64 precision only.  A solver
 * the frame cannot use falls back to STANDARD as in the reference: bundles;
 * SEMI_ANALYTIC in the KS chart; either with Q or Lambda != 0. */
enum { KT_SOLVER_STANDARD = 0, KT_SOLVER_SEMI_ANALYTIC = 1, KT_SOLVER_ELLIPTIC_CLOSED = 2 };
/* Arithmetic of the trace.  FP64: the reference's arithmetic bit for bit.
 * MIXED: analytic Hamiltonian gradient, FP32 right-hand side in the far
 * field when tol >= 1e-8, FP64 state, error control and events; agrees with
 * FP64 to about the reference's own finite-difference noise.  With
 * bundles: Hess(H) W by one dual-number evaluation of the analytic gradient
 * (FP64; the Jacobi map and its determinant FP64).
 * SMOOTH: the differentiable tracer (kt_vjp, kt_l2_grad): FP64, analytic
 * Hamiltonian gradient, analytic BL->KS Jacobian, disk crossing solved to
 * convergence, error estimate formed from the stages; RK4 step doubling, or
 * DOPRI5 for frames traced in the BL chart (a KS-chart frame integrates
 * with RK4, as the reference's KS tracer does); bundles with the analytic
 * Hessian, RK4 step doubling as the reference's bundle tracer.  Its outputs
 * are smooth functions of the frame parameters between changes of the
 * accept/reject pattern. */
enum { KT_PREC_FP64 = 0, KT_PREC_MIXED = 1, KT_PREC_SMOOTH = 2 };
/* kt_frame_desc.flags: theta_deg, phi_deg and fov_deg hold radians (the
 * reference's CameraParams_CUDA carries radians, gpu/cuda/tracer.cuh:16-20). */
#define KT_FLAG_ANGLES_RADIANS 1u
/* kt_frame_desc.flags: bundle rays that creep onto the horizon (ingoing
 * within 1e-4 r_+ of r_+ with the horizon test skipped near the equator,
 * ray_bundle.hpp:352-356) are traced on until the reference's reject or
 * step cap, so that their steps and attempts equal the reference's.
 * Without the flag they stop there with status KT_RAY_CREEP and the same
 * record (every way such a ray can end gives BundleResult{}). */
#define KT_FLAG_BUNDLE_FULL_CREEP 2u

/* Per-pixel outcome codes (GeoPixel::outcome, main.cpp:85). */
enum { KT_OUT_ESCAPED = 0, KT_OUT_DISK = 1, KT_OUT_HORIZON = 2 };
/* Per-pixel status (extension: why a ray stopped). */
enum {
  KT_RAY_EVENT = 0,      /* stopped at a disk / horizon / escape event */
  KT_RAY_STEP_CAP = 1,   /* max_steps accepted steps without an event */
  KT_RAY_REJECT_CAP = 2, /* more than 64 consecutive rejected attempts */
  KT_RAY_NONFINITE = 3,  /* step size became non-finite */
  KT_RAY_CREEP = 4       /* bundle ray creeping onto a horizon: the record of
                          * its eventual end (KT_FLAG_BUNDLE_FULL_CREEP) */
};

typedef struct kt_frame_desc {
  /* metric (M_bh, fp.a, Q_bh, Lam) */
  double M, a, Q, Lambda;
  /* camera and disk (FrameParams; angles in degrees as on the CLI) */
  double theta_deg, phi_deg, r_obs, disk_out, fov_deg;
  int32_t width, height;
  double pixel_offset_x, pixel_offset_y;
  /* integrator (requested; kt_frame_derive applies the fallback rules) */
  int32_t chart, integrator, bundles, solver_mode;
  int32_t max_steps, precision;
  double step_init, tol;
  uint32_t flags; /* KT_FLAG_* bits, 0 by default */
  int32_t reserved0;
} kt_frame_desc;

typedef struct kt_frame_derived {
  int32_t chart;      /* effective chart: KS+Lambda!=0 -> BL, bundles -> BL */
  int32_t integrator; /* effective integrator: the KS chart always uses RK4 */
  double r_horizon, rh_cut, r_isco, r_disk_in, r_disk_out, r_escape;
  double r_obs, theta_obs, phi_obs, fov_h; /* radians */
  double dlam0;       /* max(step_init, 1e-10) */
  int32_t max_steps;  /* max(1, max_steps) */
  int32_t solver;     /* effective solver (select_solver_mode, main.cpp:235-276) */
  double tol;
  double bundle_eps;  /* fov_h / width * 0.5 (ray_bundle.hpp:282) */
  double r_fp32;      /* KT_PREC_MIXED: FP32 right-hand side beyond this
                         radius (infinity: FP32 not used at this tolerance) */
} kt_frame_derived;

/* Per-pixel results, struct of arrays, width*height entries, row-major
 * (index = py*width + px).  Slot meaning is the reference's GeoPixel. */
typedef struct kt_geo_soa {
  uint8_t* outcome;
  double* r;
  double* redshift;
  double* magnif;
  double* phi_disk;
  double* theta_esc;
  double* phi_esc;
  uint8_t* status;    /* optional (NULL): KT_RAY_* */
  uint32_t* steps;    /* optional (NULL): accepted steps */
  uint32_t* attempts; /* optional (NULL): adaptive attempts (accepted+rejected) */
} kt_geo_soa;

/* ColorParams (main.cpp:72-81). */
typedef struct kt_color_params {
  double exposure, gamma, temp_scale;
  int32_t palette; /* 0 = blackbody (disk_colour); 1 = interstellar
                      (disk_colour_interstellar, main.cpp:1719-1797) */
  int32_t reserved0;
  /* interstellar palette: rings x sectors of hashed warm colours,
   * Gaussian-blended with width disk_sigma (cell units), hue offset */
  int32_t disk_rings, disk_sectors;
  double disk_sigma, disk_hue_offset;
} kt_color_params;

typedef struct kt_context kt_context;

int kt_abi_version(void);
const char* kt_status_string(kt_status s);
/* sizeof of kt_frame_desc, kt_frame_derived, kt_geo_soa, kt_color_params,
 * kt_batch_options, kt_batch_group_info, kt_grad_stats (lets bindings check
 * their struct layout); writes min(n, 7) sizes and returns the count written. */
int kt_abi_struct_sizes(size_t* sizes, int n);

kt_status kt_create(kt_context** ctx, int device);
void kt_destroy(kt_context* ctx);
const char* kt_last_error(const kt_context* ctx);

/* Host-side frame preparation; needs no GPU. */
kt_status kt_frame_derive(const kt_frame_desc* desc, kt_frame_derived* out);
void kt_frame_desc_defaults(kt_frame_desc* desc);
void kt_color_params_defaults(kt_color_params* cp);

/* Trace one frame into caller-owned device buffers, asynchronously on
 * `stream` (a cudaStream_t, NULL = legacy default stream).  Frames of at
 * least 65536 pixels are traced in rings about the image centre, innermost
 * first (three small kernels build that order on the same stream, in
 * context scratch); the results are those of any other order, bit for bit. */
kt_status kt_trace(kt_context* ctx, const kt_frame_desc* desc,
                   const kt_geo_soa* out, void* stream);

/* Trace only the pixels listed in pix[0..n) (index py*width+px) into
 * compact device outputs out[i] (used for sampling and tile sharding). */
kt_status kt_trace_pixels(kt_context* ctx, const kt_frame_desc* desc,
                          const uint32_t* pix_dev, int64_t n,
                          const kt_geo_soa* out, void* stream);

/* kt_trace for callers that may not allocate device memory (no counterpart
 * in the reference renderer).  A host that owns all device memory, or a
 * frame loop that cannot afford cudaMalloc/cudaFree (they can synchronize
 * the device), passes only its own output buffers: no context, nothing
 * allocated.  The trace kernels' scratch (ray-queue counters, KS fallback
 * list, the centre-out ray order of whole frames of at least 2^16 pixels, as
 * kt_trace uses) is a fixed device array inside the library, sized for frames
 * of at most KT_NOALLOC_MAX_PIXELS pixels (12.5 MiB per GPU, held until the
 * process exits); larger frames return KT_ERR_INVALID_ARGUMENT.  Runs on the
 * current device, asynchronously on `stream`.  All calls share that array:
 * calls ordered on the device are independent, calls that overlap on the
 * device race.  The first call on a device resolves the array's address for
 * it; make that call before any stream capture on the device. */
#define KT_NOALLOC_MAX_PIXELS (1u << 20)
kt_status kt_trace_noalloc(const kt_frame_desc* desc, const kt_geo_soa* out, void* stream);

/* Same as kt_trace but with host buffers: returns after the results are on
 * the host.  When every given buffer is page-locked and mapped for the
 * context's device (cudaHostAlloc, cudaHostRegister), the kernels write the
 * records into them directly (so they must be writable: not registered
 * with cudaHostRegisterReadOnly, and each must hold width*height entries
 * inside its page-locked range, as every output buffer must: the kernels
 * write through the mapping without a bounds check); otherwise they go
 * through a device staging area and are copied after the trace. */
kt_status kt_trace_host(kt_context* ctx, const kt_frame_desc* desc,
                        const kt_geo_soa* out_host);

/* Phase 2 on the device: SoA -> RGB8 (width*height*3 bytes).  bg_rgb is a
 * device RGB8 equirectangular image (bg_w*bg_h*3) or NULL for black. */
kt_status kt_colorize(kt_context* ctx, const kt_frame_desc* desc,
                      const kt_geo_soa* geo, const kt_color_params* cp,
                      const uint8_t* bg_rgb, int32_t bg_w, int32_t bg_h,
                      uint8_t* rgb_out, void* stream);

/* colorize_buffer (main.cpp:1817) on host buffers: the per-pixel records of
 * a width x height frame (e.g. read from a .kgeo file), black-hole mass M,
 * the ISCO radius and the disk's inner and outer radii recorded with them
 * (KGeoMeta, main.cpp:101-106); RGB8 out (width*height*3 bytes). */
kt_status kt_colorize_host(kt_context* ctx, const kt_geo_soa* geo_host, int32_t width,
                           int32_t height, double M, double r_isco, double r_disk_in,
                           double r_disk_out, const kt_color_params* cp,
                           const uint8_t* bg_rgb_host, int32_t bg_w, int32_t bg_h,
                           uint8_t* rgb_out_host);

/* render_image equivalent: trace + colorize, host buffers in and out. */
kt_status kt_render_host(kt_context* ctx, const kt_frame_desc* desc,
                         const kt_color_params* cp, const uint8_t* bg_rgb_host,
                         int32_t bg_w, int32_t bg_h, uint8_t* rgb_out_host);

/* render_image with its camera_spp argument (main.cpp:2232-2322, the CLI's
 * --camera-spp / --spp, main.cpp:2557): camera_spp passes, each a full
 * trace + colorize at the frame's pixel offset plus the pass's jitter
 * (kt_camera_spp_offsets), averaged in linear light
 * (pow(c / 255, gamma), mean, pow(., 1 / gamma), lround) on the device.
 * camera_spp <= 1 is kt_render_host.  KT_ERR_INVALID_ARGUMENT above
 * KT_MAX_CAMERA_SPP. */
#define KT_MAX_CAMERA_SPP 256
kt_status kt_render_spp_host(kt_context* ctx, const kt_frame_desc* desc,
                             const kt_color_params* cp, int32_t camera_spp,
                             const uint8_t* bg_rgb_host, int32_t bg_w, int32_t bg_h,
                             uint8_t* rgb_out_host);

/* The elliptic-closed solver's fallback reason per pixel, the reference's
 * --debug-elliptic tag (EllipticFallbackReason, main.cpp:178-186, stored in
 * GeoPixel padding at main.cpp:2111-2121 and coloured by colorize_buffer,
 * main.cpp:1828-1843): 0 the closed form placed the crossing in the disk,
 * 1 constants of motion, 2 polar crossing, 3 radial map, 4 radial value
 * invalid, 5 outside the disk.  All 0 where the frame's effective solver is
 * not ELLIPTIC_CLOSED.  reason: width*height bytes (device / host). */
#define KT_ELLIPTIC_REASONS 6
kt_status kt_elliptic_reasons(kt_context* ctx, const kt_frame_desc* desc, uint8_t* reason,
                              void* stream);
kt_status kt_elliptic_reasons_host(kt_context* ctx, const kt_frame_desc* desc,
                                   uint8_t* reason_host);

/* The camera_spp jitter offsets in pixels (main.cpp:2238-2279):
 * xy[2 s], xy[2 s + 1] for pass s < max(camera_spp, 1). */
kt_status kt_camera_spp_offsets(int32_t camera_spp, double* xy);

/* ---- batches: many frames in one CUDA graph launch ----------------------
 * No counterpart in the reference renderer, which traces one frame per
 * render_image call (main.cpp:2209-2478) and loops over frames in its
 * animation driver.  A batch holds n_frames frames of any sizes, charts,
 * integrators and precisions, each with its own caller-owned device result
 * arrays.  kt_batch_create groups the frames by kernel (KS RK4, BL RK4, BL
 * DOPRI5, bundles; FP64 or mixed), prepares one persistent launch per group
 * over the group's rays (all its frames in one device ray queue), and
 * captures the launches into one CUDA graph; kt_batch_launch replays that
 * graph with a single cudaGraphLaunch.  Results are bit-identical to
 * kt_trace of each frame.
 *
 * Tuning: each group's launch has a block size and register cap (one of
 * KT_BATCH_VARIANTS compiled variants), a persistent grid, and a regroup
 * threshold (idle lanes of a warp take new rays only when at least that many
 * are idle).  Variants 0-2 run one ray per lane (32 rays per warp); variant
 * 3 runs two lanes per ray (16 rays per warp), which only the FP64 bundle
 * kernel has -- other groups given variant 3 take their default variant, and
 * the tuner times it for bundle groups only.  With KT_BATCH_AUTOTUNE,
 * kt_batch_create times every variant x threshold on a sample of the group's
 * rays (tune_fraction of them, in runs of 256 neighbouring pixels) and keeps
 * the fastest; the sample's results are written to the outputs.  Otherwise
 * the variant and threshold are the options' (or the single-frame defaults).
 *
 * The graph reads the frames' parameters and output pointers from device
 * memory owned by the batch: the outputs stay bound to the batch.  Launches
 * of one batch must not overlap on the device (they share its queues);
 * different batches are independent. */
typedef struct kt_batch kt_batch;

#define KT_BATCH_VARIANTS 4
#define KT_BATCH_AUTOTUNE 1u

typedef struct kt_batch_options {
  uint32_t flags;          /* KT_BATCH_AUTOTUNE */
  int32_t variant;         /* -1: per-mode default; else 0..KT_BATCH_VARIANTS-1 */
  int32_t refill_min;      /* 0: per-mode default (the single-frame kernels' threshold:
                              8 for FP64 bundles, 1 for the separable tracer, 32 otherwise);
                              1..32: idle lanes of a warp take new rays once this many are idle */
  int32_t tune_reps;       /* timed repetitions per candidate (>= 1) */
  double tune_fraction;    /* share of a group's rays in the tuning sample, (0, 1] */
} kt_batch_options;

typedef struct kt_batch_group_info {
  int32_t kernel;          /* 0 BL RK4, 1 BL DOPRI5, 2 KS RK4, 3 bundles, 4-7 mixed BL RK4 / BL DOPRI5 / KS RK4 / bundles, 8 separable Kerr */
  int32_t n_frames;
  uint64_t n_rays;
  int32_t variant;
  int32_t block;           /* threads per block */
  int32_t min_blocks;      /* blocks per SM the register cap is set for */
  int32_t grid;            /* persistent blocks */
  int32_t refill_min;
  int32_t rays_per_warp;
  int32_t tuned;           /* 1: chosen by measurement */
  int32_t candidates;      /* candidates timed */
  double sample_rays;      /* rays in the tuning sample */
  double best_ms;          /* tuning sample time of the chosen candidate */
  double default_ms;       /* tuning sample time of the default candidate */
} kt_batch_group_info;

void kt_batch_options_defaults(kt_batch_options* opt);
/* Creates the batch on the context's device.  descs[i] and outs[i] (device
 * pointers, as for kt_trace) describe frame i.  opt may be NULL (defaults).
 * Tuning, when asked for, runs synchronously on the context's stream. */
kt_status kt_batch_create(kt_context* ctx, const kt_frame_desc* descs,
                          const kt_geo_soa* outs, int32_t n_frames,
                          const kt_batch_options* opt, kt_batch** batch);
/* Traces every frame of the batch: one cudaGraphLaunch on `stream`. */
kt_status kt_batch_launch(kt_batch* batch, void* stream);
int32_t kt_batch_group_count(const kt_batch* batch);
kt_status kt_batch_group(const kt_batch* batch, int32_t i, kt_batch_group_info* info);
/* Total rays of the batch (sum of width*height). */
uint64_t kt_batch_rays(const kt_batch* batch);
void kt_batch_destroy(kt_batch* batch);

/* ---- gradients: the discrete adjoint of the smooth tracer ---------------
 * No counterpart in the reference renderer.  The gradient is that of the
 * KT_PREC_SMOOTH tracer (whatever desc->precision says) with respect to the
 * frame parameters, in this order (units of kt_frame_desc): */
enum {
  KT_GRAD_A = 0, KT_GRAD_Q = 1, KT_GRAD_LAMBDA = 2, KT_GRAD_THETA = 3, KT_GRAD_R_OBS = 4,
  KT_GRAD_DISK_OUT = 5, KT_GRAD_COUNT = 6
};
/* Point-sampled pixels: g and r_hit of a disk pixel do not depend on the
 * disk's outer radius (it only decides which rays hit), so the
 * KT_GRAD_DISK_OUT entry is 0 by construction.  In the KS chart (Lambda = 0 only; any other
 * Lambda sends the frame to the BL chart, main.cpp:2033-2040) the Lambda
 * entry is the derivative of the BL-chart trace of the same frame, which
 * is what the tracer computes for Lambda != 0; it takes a second pass
 * unless KT_GRAD_SKIP_LAMBDA is given (the entry is then 0). */
#define KT_GRAD_SKIP_LAMBDA 1u

typedef struct kt_grad_stats {
  double loss;           /* kt_l2_grad: the loss; kt_vjp: 0 */
  int64_t grad_pixels;   /* disk pixels whose reverse sweep ran */
  int64_t bl_pixels;     /* pixels traced in the BL chart (first pass) */
  int64_t unrecorded;    /* disk pixels with a cotangent but > 131072 steps: no gradient */
  float ms_main;         /* device time of the gradient pass */
  float ms_lambda;       /* device time of the BL pass for Lambda (0 if none) */
} kt_grad_stats;

/* Vector-Jacobian product: grad[k] = sum over pixels p of
 * cot_redshift[p] dg_p/dtheta_k + cot_r[p] d r_hit,p/dtheta_k over the disk
 * pixels (device arrays of width*height doubles; either may be NULL).
 * `out` (device SoA, optional) receives the smooth forward results.  grad
 * and stats are host memory; the call returns when they are written. */
kt_status kt_vjp(kt_context* ctx, const kt_frame_desc* desc, const double* cot_redshift,
                 const double* cot_r, const kt_geo_soa* out, uint32_t flags,
                 double grad[KT_GRAD_COUNT], kt_grad_stats* stats, void* stream);

/* L2 image loss against a target frame (device SoA of a smooth trace with
 * other parameters): L = sum over pixels that are disk hits in both frames
 * of w_g (g - g_t)^2 + w_r (r_hit - r_t)^2, and its gradient, in one fused
 * forward + reverse pass per pixel. */
kt_status kt_l2_grad(kt_context* ctx, const kt_frame_desc* desc, const kt_geo_soa* target,
                     double w_g, double w_r, const kt_geo_soa* out, uint32_t flags,
                     double* loss, double grad[KT_GRAD_COUNT], kt_grad_stats* stats,
                     void* stream);

/* The same over the pixels pix_dev[0..n_pix) only (device indices
 * py*width+px; outputs and cotangents still indexed over the whole frame):
 * the per-GPU share of a frame split across GPUs, whose partial gradients
 * add up (one all-reduce of KT_GRAD_COUNT doubles).  Indices outside the
 * frame are skipped. */
kt_status kt_vjp_pixels(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                        int64_t n_pix, const double* cot_redshift, const double* cot_r,
                        const kt_geo_soa* out, uint32_t flags, double grad[KT_GRAD_COUNT],
                        kt_grad_stats* stats, void* stream);
kt_status kt_l2_grad_pixels(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                            int64_t n_pix, const kt_geo_soa* target, double w_g, double w_r,
                            const kt_geo_soa* out, uint32_t flags, double* loss,
                            double grad[KT_GRAD_COUNT], kt_grad_stats* stats, void* stream);

/* The same with the Jacobi bundle's magnification (GeoPixel::magnif of a
 * bundle frame, ray_bundle.hpp:386-392; the renderer scales a disk pixel's
 * intensity by clamp(1/magnif, 0.05, 5), main.cpp:1789): kt_vjp_magnif adds
 * cot_magnif[p] d magnif_p / d theta_k (device array over the frame, or
 * NULL), kt_l2_grad_magnif adds w_m (magnif - magnif_t)^2 to the loss
 * (target->magnif must then be set).  pix_dev / n_pix as kt_vjp_pixels
 * (NULL, 0: every pixel).  On a frame without bundles the magnification is
 * the constant 1 and these equal kt_vjp_pixels / kt_l2_grad_pixels.  Not in
 * the reference (which has no gradients). */
kt_status kt_vjp_magnif(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                        int64_t n_pix, const double* cot_redshift, const double* cot_r,
                        const double* cot_magnif, const kt_geo_soa* out, uint32_t flags,
                        double grad[KT_GRAD_COUNT], kt_grad_stats* stats, void* stream);
kt_status kt_l2_grad_magnif(kt_context* ctx, const kt_frame_desc* desc, const uint32_t* pix_dev,
                            int64_t n_pix, const kt_geo_soa* target, double w_g, double w_r,
                            double w_m, const kt_geo_soa* out, uint32_t flags, double* loss,
                            double grad[KT_GRAD_COUNT], kt_grad_stats* stats, void* stream);

/* Measured FP64 FMA throughput of the context's device (GFLOP/s, 2 flops
 * per FMA): the non-tensor FP64 peak the trace kernels are bounded by. */
kt_status kt_measure_fp64_peak(kt_context* ctx, double* gflops);

/* Measured cost of the operations that the algorithmic flop count weights,
 * in flops (2 per FMA, so an operation that takes the time of n FMAs at full
 * throughput costs 2n): eight independent recurrences per thread on all SMs,
 * each operation's throughput against the FMA throughput of the same probe. */
typedef struct kt_op_costs {
  double fma_gflops; /* FP64 FMA throughput of the probe, GFLOP/s */
  double div;        /* correctly rounded division */
  double div3;       /* x / 3, the correctly rounded quotient (three operations) */
  double sqrt;       /* correctly rounded square root */
  double sincos;     /* sin and cos of one argument (the renderer's libm) */
  double pow;        /* pow (the renderer's libm) */
} kt_op_costs;
kt_status kt_measure_op_costs(kt_context* ctx, kt_op_costs* out);

/* Deterministic procedural equirectangular star field (RGB8, w*h*3 bytes),
 * the stand-in for the reference's background photographs, which are not in
 * its tree.  Same seed, same image, on any host. */
kt_status kt_starfield(uint64_t seed, int32_t w, int32_t h, uint8_t* rgb);

/* .kgeo two-phase cache (main.cpp:96-137): 4-byte magic, u32 version, the
 * 88-byte KGeoMeta, then width*height 28-byte float32 GeoPixel records. */
kt_status kt_kgeo_write(const char* path, const kt_frame_desc* desc,
                        const kt_geo_soa* geo_host);
kt_status kt_kgeo_read_header(const char* path, int32_t* width, int32_t* height,
                              double meta[10]);
kt_status kt_kgeo_read(const char* path, const kt_geo_soa* geo_host,
                       int64_t capacity);

#ifdef __cplusplus
}
#endif

#endif /* KERRTRACE_H */
