// kt_batch.cpp -- batches of frames: one persistent launch per kernel mode
// over all rays of the mode's frames, captured into one CUDA graph, with an
// autotuner for the launch variant and the regroup threshold.
//
// Device memory of a batch (one allocation, 256-byte aligned sections):
//   per group: Frame[n_g], OutSoA[n_g], uint64 offsets[n_g + 1], and for the
//   KS and separable-Kerr groups the fallback list uint32[n_rays_g]; then 4 uint32 counters per
//   group ([0] ray queue, [1] fallback queue, [2] fallback count).
// The graph: memset(counters) -> one branch per group, each branch the
// group's persistent launch (KS groups: then the BL launch over the rays
// whose KS initialisation failed, main.cpp:1537-1538; separable-Kerr
// groups: the BL RK4 launch over the rays that gave up) -> join.
#include <cmath>
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "../../include/kerrtrace.h"
#include "kt_context.h"
#include "kt_frame.h"
#include "kt_internal.h"

using namespace ktc;

namespace {

constexpr uint32_t kSampleRun = 256;     // neighbouring rays per tuning run
constexpr int kRefillCandidates[] = {1, 16, 24, 32};
constexpr uint64_t kMaxGroupRays = 1ull << 31;
static_assert(KT_BATCH_VARIANTS == kt::kBatchVariants, "variant count of the ABI");

struct Group {
  kt::Mode mode;
  kt::Mode fb_mode = kt::kModeBLRk4;  // BL launch over the fallback list
  std::vector<int> frames;  // batch frame indices
  bool fp32 = false;        // some frame may run the mixed FP32 right-hand side
  uint64_t n_rays = 0;
  kt::Frame* d_frames = nullptr;
  kt::OutSoA* d_outs = nullptr;
  uint64_t* d_offsets = nullptr;
  uint32_t* d_fb = nullptr;      // groups with a fallback pass only
  uint32_t* d_order = nullptr;   // the group's rays, each frame in centre-out order
  uint32_t* d_counters = nullptr;
  int variant = 0;
  int refill_min = 1;
  kt::LaunchShape shape{};
  int fb_variant = 0;
  kt::LaunchShape fb_shape{};
  // frames of the elliptic-closed solver: after the group's trace, the
  // closed-form disk hits (k_elliptic) over each such frame
  std::vector<kt::Frame> ell_frames;
  std::vector<kt::OutSoA> ell_outs;
  kt_batch_group_info info{};
};

int default_variant(kt::Mode m) {
  // The single-frame launch shapes (kt_kernels.cu, kt_mixed.cu): two lanes
  // per ray, 128 x 3, for the FP64 bundle kernel; 128 x 1 for the mixed
  // bundle and separable-Kerr kernels; 64 x 9 for the others.
  if (m == kt::kModeBundle) return kt::kBatchPairVariant;
  return (m == kt::kModeBundleMixed || m == kt::kModeSepRk4) ? 1 : 0;
}

int default_refill(kt::Mode m) {
  // ... and their refill thresholds (in lanes)
  return m == kt::kModeBundle ? 8 : m == kt::kModeSepRk4 ? 1 : 32;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct kt_batch {
  kt_context* ctx = nullptr;
  std::vector<Group> groups;
  uint64_t n_rays = 0;
  unsigned char* d_mem = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

kt::BatchRays group_rays(const Group& g, const uint32_t* list, const uint32_t* n_dev,
                         uint64_t n, int refill_min) {
  kt::BatchRays br;
  br.frames = g.d_frames;
  br.outs = g.d_outs;
  br.offsets = g.d_offsets;
  br.n_frames = (int)g.frames.size();
  br.refill_min = refill_min;
  br.list = list;
  br.n_dev = n_dev;
  br.n = n;
  br.fp32 = g.fp32;
  return br;
}

// Enqueue one group's trace: the persistent launch over `list` (or all its
// rays) and, for groups with a fallback pass, the BL launch over the fallback list.  The
// group's counters must be zero.
cudaError_t enqueue_group(const Group& g, int variant, const kt::LaunchShape& s, int refill_min,
                          const uint32_t* list, uint64_t n, cudaStream_t st) {
  kt::Fallback fb = {g.d_fb, nullptr, g.d_counters + 2};
  cudaError_t e = kt::launch_batch(g.mode, variant,
                                   group_rays(g, list ? list : g.d_order, nullptr, n, refill_min),
                                   g.d_counters, fb, s, st);
  if (e != cudaSuccess) return e;
  if (kt::has_fallback(g.mode))
    e = kt::launch_batch(g.fb_mode, g.fb_variant, group_rays(g, g.d_fb, g.d_counters + 2, 0, 1),
                          g.d_counters + 1, fb, g.fb_shape, st);
  if (e != cudaSuccess || list != nullptr) return e;  // a tuning sample: no closed form
  for (size_t k = 0; k < g.ell_frames.size() && e == cudaSuccess; ++k) {
    const kt::Frame& f = g.ell_frames[k];
    const kt::RayList all = {nullptr, nullptr, nullptr, (uint32_t)((uint64_t)f.cam.W * f.cam.H)};
    e = kt::launch_elliptic(f, g.ell_outs[k], all, st);
  }
  return e;
}

// Time the candidates (variant x regroup threshold) on a sample of the
// group's rays and keep the fastest.
kt_status tune_group(kt_context* ctx, Group& g, const kt_batch_options& opt) {
  const uint64_t n = g.n_rays;
  uint64_t stride_runs = (uint64_t)(1.0 / opt.tune_fraction + 0.5);
  if (stride_runs < 1) stride_runs = 1;
  std::vector<uint32_t> sample;
  for (uint64_t run = 0; run * kSampleRun < n; run += stride_runs)
    for (uint64_t k = run * kSampleRun; k < std::min(n, (run + 1) * kSampleRun); ++k)
      sample.push_back((uint32_t)k);
  uint32_t* d_sample = nullptr;
  KT_CUDA(ctx, cudaMalloc((void**)&d_sample, sample.size() * sizeof(uint32_t)), "tuning sample");
  struct Guard {
    uint32_t* p;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Guard() {
      cudaFree(p);
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    }
  } guard{d_sample};
  cudaStream_t st = ctx->stream;
  KT_CUDA(ctx, cudaMemcpyAsync(d_sample, sample.data(), sample.size() * sizeof(uint32_t),
                               cudaMemcpyHostToDevice, st), "tuning sample");
  KT_CUDA(ctx, cudaEventCreate(&guard.e0), "event");
  KT_CUDA(ctx, cudaEventCreate(&guard.e1), "event");
  kt::LaunchShape shapes[kt::kBatchVariants];
  for (int v = 0; v < kt::kBatchVariants; ++v) {
    if (!kt::batch_variant_ok(g.mode, v)) continue;
    KT_CUDA(ctx, kt::batch_shape(g.mode, v, ctx->device, &shapes[v]), "occupancy query");
    // Untimed first launch of each variant (module load, caches).
    KT_CUDA(ctx, cudaMemsetAsync(g.d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
    KT_CUDA(ctx, enqueue_group(g, v, shapes[v], 1, d_sample, std::min<uint64_t>(sample.size(), 4096),
                               st), "tuning launch");
  }
  const int reps = std::max(1, opt.tune_reps);
  float best = 1e30f, dflt = -1.f;
  int candidates = 0;
  for (int v = 0; v < kt::kBatchVariants; ++v) {
    if (!kt::batch_variant_ok(g.mode, v)) continue;
    for (int rm : kRefillCandidates) {
      float t = 1e30f;
      for (int r = 0; r < reps; ++r) {
        KT_CUDA(ctx, cudaMemsetAsync(g.d_counters, 0, 4 * sizeof(uint32_t), st), "reset queue");
        KT_CUDA(ctx, cudaEventRecord(guard.e0, st), "event");
        KT_CUDA(ctx, enqueue_group(g, v, shapes[v], rm, d_sample, sample.size(), st),
                "tuning launch");
        KT_CUDA(ctx, cudaEventRecord(guard.e1, st), "event");
        KT_CUDA(ctx, cudaEventSynchronize(guard.e1), "tuning run");
        float ms = 0.f;
        KT_CUDA(ctx, cudaEventElapsedTime(&ms, guard.e0, guard.e1), "event time");
        t = std::min(t, ms);
      }
      ++candidates;
      if (v == default_variant(g.mode) && rm == 1) dflt = t;
      if (t < best) {
        best = t;
        g.variant = v;
        g.refill_min = rm;
      }
    }
  }
  g.shape = shapes[g.variant];
  g.info.tuned = 1;
  g.info.candidates = candidates;
  g.info.sample_rays = (double)sample.size();
  g.info.best_ms = best;
  g.info.default_ms = dflt;
  return KT_OK;
}

kt_status capture(kt_context* ctx, kt_batch* b, size_t counters_bytes, uint32_t* d_counters) {
  const size_t ng = b->groups.size();
  std::vector<cudaStream_t> side(ng, nullptr);
  std::vector<cudaEvent_t> join(ng, nullptr);
  cudaEvent_t fork = nullptr;
  cudaStream_t origin = nullptr;
  struct Cleanup {
    std::vector<cudaStream_t>& s;
    std::vector<cudaEvent_t>& j;
    cudaEvent_t& f;
    cudaStream_t& o;
    ~Cleanup() {
      for (auto x : s)
        if (x) cudaStreamDestroy(x);
      for (auto x : j)
        if (x) cudaEventDestroy(x);
      if (f) cudaEventDestroy(f);
      if (o) cudaStreamDestroy(o);
    }
  } cleanup{side, join, fork, origin};
  KT_CUDA(ctx, cudaStreamCreateWithFlags(&origin, cudaStreamNonBlocking), "stream");
  KT_CUDA(ctx, cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), "event");
  for (size_t i = 0; i < ng; ++i) {
    KT_CUDA(ctx, cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking), "stream");
    KT_CUDA(ctx, cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming), "event");
  }
  KT_CUDA(ctx, cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal), "begin capture");
  cudaError_t e = cudaMemsetAsync(d_counters, 0, counters_bytes, origin);
  if (e == cudaSuccess) e = cudaEventRecord(fork, origin);
  for (size_t i = 0; i < ng && e == cudaSuccess; ++i) {
    const Group& g = b->groups[i];
    e = cudaStreamWaitEvent(side[i], fork, 0);
    if (e == cudaSuccess)
      e = enqueue_group(g, g.variant, g.shape, g.refill_min, nullptr, g.n_rays, side[i]);
    if (e == cudaSuccess) e = cudaEventRecord(join[i], side[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(origin, join[i], 0);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(origin, &graph);
  if (e == cudaSuccess) e = ee;
  if (e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_fail(ctx, e, "batch graph capture");
  }
  b->graph = graph;
  KT_CUDA(ctx, cudaGraphInstantiate(&b->exec, graph, 0), "batch graph instantiate");
  return KT_OK;
}

}  // namespace

extern "C" {

void kt_batch_options_defaults(kt_batch_options* opt) {
  if (!opt) return;
  memset(opt, 0, sizeof *opt);
  opt->variant = -1;
  opt->refill_min = 0;
  opt->tune_reps = 2;
  opt->tune_fraction = 1.0 / 16.0;
}

void kt_batch_destroy(kt_batch* b) {
  if (!b) return;
  DeviceGuard dg(b->ctx->device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_mem);
  delete b;
}

kt_status kt_batch_create(kt_context* ctx, const kt_frame_desc* descs, const kt_geo_soa* outs,
                          int32_t n_frames, const kt_batch_options* opt_in, kt_batch** out) {
  if (!ctx || !out) return KT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!descs || !outs || n_frames < 1)
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_batch_create: no frames");
  kt_batch_options opt;
  kt_batch_options_defaults(&opt);
  if (opt_in) opt = *opt_in;
  if (opt.variant < -1 || opt.variant >= kt::kBatchVariants || opt.refill_min < 0 ||
      opt.refill_min > 32 || opt.tune_reps < 0 || !(opt.tune_fraction > 0.0) ||
      !(opt.tune_fraction <= 1.0) || (opt.flags & ~KT_BATCH_AUTOTUNE))
    return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_batch_create: bad options");
  // Frames -> groups by kernel mode.
  std::vector<kt::Frame> frames((size_t)n_frames);
  // key: kernel mode x mode of its fallback pass (a KS frame's BL pass
  // integrates with the frame's integrator, main.cpp:1537-1538)
  std::vector<int> group_of_key(kt::kNumModes * kt::kNumModes, -1);
  kt_batch* b = new (std::nothrow) kt_batch();
  if (!b) return fail(ctx, KT_ERR_OUT_OF_MEMORY, "kt_batch_create: host allocation");
  b->ctx = ctx;
  struct Owner {
    kt_batch*& b;
    ~Owner() {
      if (b) kt_batch_destroy(b);
    }
  } owner{b};
  for (int i = 0; i < n_frames; ++i) {
    kt_status r = kt::prepare_frame(&descs[i], &frames[i], nullptr, &ctx->err);
    if (r != KT_OK) {
      ctx->err = "frame " + std::to_string(i) + ": " + ctx->err;
      return r;
    }
    if (frames[i].precision == KT_PREC_SMOOTH)
      return fail(ctx, KT_ERR_UNSUPPORTED,
                  "frame " + std::to_string(i) + ": the smooth tracer does not run in batches");
    if (!out_complete(&outs[i]))
      return fail(ctx, KT_ERR_INVALID_ARGUMENT,
                  "frame " + std::to_string(i) + ": output pointer is NULL");
    const kt::Mode m = kt::frame_mode(frames[i]);
    const kt::Mode fm = kt::has_fallback(m) ? kt::fallback_mode(frames[i]) : kt::kModeBLRk4;
    const int key = m * kt::kNumModes + fm;
    if (group_of_key[key] < 0) {
      group_of_key[key] = (int)b->groups.size();
      b->groups.emplace_back();
      b->groups.back().mode = m;
      b->groups.back().fb_mode = fm;
    }
    Group& g = b->groups[group_of_key[key]];
    g.frames.push_back(i);
    g.fp32 = g.fp32 || std::isfinite(frames[i].r_fp32);
    if (frames[i].solver == KT_SOLVER_ELLIPTIC_CLOSED) {
      g.ell_frames.push_back(frames[i]);
      g.ell_outs.push_back(to_out(&outs[i]));
    }
    g.n_rays += (uint64_t)descs[i].width * (uint64_t)descs[i].height;
    b->n_rays += (uint64_t)descs[i].width * (uint64_t)descs[i].height;
  }
  for (const Group& g : b->groups)
    if (g.n_rays > kMaxGroupRays)
      return fail(ctx, KT_ERR_INVALID_ARGUMENT, "kt_batch_create: more than 2^31 rays of one kernel");
  DeviceGuard dg(ctx->device);
  // Device layout.
  size_t bytes = 0;
  std::vector<size_t> off_frames, off_outs, off_offsets, off_fb, off_order;
  size_t ring_scratch = 0;
  for (int i = 0; i < n_frames; ++i)
    ring_scratch = std::max(ring_scratch,
                            kt::ring_scratch_words((uint64_t)descs[i].width * (uint64_t)descs[i].height));
  for (const Group& g : b->groups) {
    const size_t nf = g.frames.size();
    off_order.push_back(bytes);
    bytes = align256(bytes + g.n_rays * sizeof(uint32_t));
    off_frames.push_back(bytes);
    bytes = align256(bytes + nf * sizeof(kt::Frame));
    off_outs.push_back(bytes);
    bytes = align256(bytes + nf * sizeof(kt::OutSoA));
    off_offsets.push_back(bytes);
    bytes = align256(bytes + (nf + 1) * sizeof(uint64_t));
    off_fb.push_back(bytes);
    if (kt::has_fallback(g.mode)) bytes = align256(bytes + g.n_rays * sizeof(uint32_t));
  }
  const size_t off_counters = bytes;
  const size_t counters_bytes = b->groups.size() * 4 * sizeof(uint32_t);
  bytes = align256(bytes + counters_bytes);
  const size_t off_scratch = bytes;
  bytes = align256(bytes + ring_scratch * sizeof(uint32_t));
  KT_CUDA(ctx, cudaMalloc((void**)&b->d_mem, bytes), "batch buffers");
  uint32_t* d_counters = (uint32_t*)(b->d_mem + off_counters);
  for (size_t gi = 0; gi < b->groups.size(); ++gi) {
    Group& g = b->groups[gi];
    const size_t nf = g.frames.size();
    g.d_frames = (kt::Frame*)(b->d_mem + off_frames[gi]);
    g.d_outs = (kt::OutSoA*)(b->d_mem + off_outs[gi]);
    g.d_offsets = (uint64_t*)(b->d_mem + off_offsets[gi]);
    g.d_fb = kt::has_fallback(g.mode) ? (uint32_t*)(b->d_mem + off_fb[gi]) : nullptr;
    g.d_counters = d_counters + 4 * gi;
    g.d_order = (uint32_t*)(b->d_mem + off_order[gi]);
    std::vector<kt::Frame> hf(nf);
    std::vector<kt::OutSoA> ho(nf);
    std::vector<uint64_t> hoff(nf + 1, 0);
    for (size_t k = 0; k < nf; ++k) {
      const int i = g.frames[k];
      hf[k] = frames[i];
      ho[k] = to_out(&outs[i]);
      hoff[k + 1] = hoff[k] + (uint64_t)descs[i].width * (uint64_t)descs[i].height;
    }
    KT_CUDA(ctx, cudaMemcpy(g.d_frames, hf.data(), nf * sizeof(kt::Frame), cudaMemcpyHostToDevice),
            "batch frames");
    KT_CUDA(ctx, cudaMemcpy(g.d_outs, ho.data(), nf * sizeof(kt::OutSoA), cudaMemcpyHostToDevice),
            "batch outputs");
    KT_CUDA(ctx, cudaMemcpy(g.d_offsets, hoff.data(), (nf + 1) * sizeof(uint64_t),
                            cudaMemcpyHostToDevice), "batch offsets");
    for (size_t k = 0; k < nf; ++k) {
      const kt_frame_desc& dk = descs[g.frames[k]];
      KT_CUDA(ctx, kt::launch_ring_order(dk.width, dk.height, (uint32_t)hoff[k],
                                         (uint32_t*)(b->d_mem + off_scratch), g.d_order + hoff[k],
                                         ctx->stream), "ray order");
    }
    KT_CUDA(ctx, cudaStreamSynchronize(ctx->stream), "ray order");
    if (kt::has_fallback(g.mode)) {
      g.fb_variant = default_variant(g.fb_mode);
      KT_CUDA(ctx, kt::batch_shape(g.fb_mode, g.fb_variant, ctx->device, &g.fb_shape), "occupancy query");
    }
    // a variant the group's kernel lacks (the paired one, outside bundles)
    // gives the group its default variant
    g.variant = kt::batch_variant_ok(g.mode, opt.variant) ? opt.variant : default_variant(g.mode);
    g.refill_min = opt.refill_min > 0 ? opt.refill_min : default_refill(g.mode);
    if (opt.flags & KT_BATCH_AUTOTUNE) {
      kt_status r = tune_group(ctx, g, opt);
      if (r != KT_OK) return r;
    } else {
      KT_CUDA(ctx, kt::batch_shape(g.mode, g.variant, ctx->device, &g.shape), "occupancy query");
    }
    kt_batch_group_info& in = g.info;
    in.kernel = (int32_t)g.mode;
    in.n_frames = (int32_t)nf;
    in.n_rays = g.n_rays;
    in.variant = g.variant;
    in.block = kt::kBatchBlock[g.variant];
    in.min_blocks = kt::kBatchMinBlocks[g.variant];
    in.grid = g.shape.grid;
    in.refill_min = g.refill_min;
    in.rays_per_warp = kt::kBatchRaysPerWarp[g.variant];
  }
  kt_status r = capture(ctx, b, counters_bytes, d_counters);
  if (r != KT_OK) return r;
  *out = b;
  b = nullptr;  // owned by the caller now
  return KT_OK;
}

kt_status kt_batch_launch(kt_batch* b, void* stream) {
  if (!b) return KT_ERR_INVALID_ARGUMENT;
  kt_context* ctx = b->ctx;
  DeviceGuard dg(ctx->device);
  KT_CUDA(ctx, cudaGraphLaunch(b->exec, (cudaStream_t)stream), "batch graph launch");
  return KT_OK;
}

int32_t kt_batch_group_count(const kt_batch* b) { return b ? (int32_t)b->groups.size() : 0; }

kt_status kt_batch_group(const kt_batch* b, int32_t i, kt_batch_group_info* info) {
  if (!b || !info || i < 0 || i >= (int32_t)b->groups.size()) return KT_ERR_INVALID_ARGUMENT;
  *info = b->groups[i].info;
  return KT_OK;
}

uint64_t kt_batch_rays(const kt_batch* b) { return b ? b->n_rays : 0; }

}  // extern "C"
