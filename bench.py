#!/usr/bin/env python
"""Headline benchmark: primary rays traced per second (Mrays/s) at 1280x720.

Workload (default): Kerr-Newman-de Sitter, BL chart, a=0.9, Q=0.3,
Lambda=1e-4, r_obs=60, theta=85 deg, fov=30 deg, disk ISCO..20, DOPRI5 at
tol 1e-10, plain FP64 (bit-identical to the reference CPU path).  A step is
one full 1280x720 frame traced by kt_trace into device-resident SoA
buffers.  Inputs are frame parameters only; between steps a 256 MB buffer
is written to flush L2 (the 55 MB of outputs would otherwise stay cached).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs under torchrun, one process per GPU: every rank traces its own
720p frame (an orbit of the camera, phi = 360*rank/N deg), no data-path
collective, scaling "weak"; time = max over ranks.  `--impl reference`
times the reference renderer's own CPU path (compiled from its sources,
oracle/_ref) on the host cores for the same metric.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s 720p: plain FP64 vs mixed-precision at stated error; adjoint ms/frame"

WORKLOADS = {
    "knds_bl_dopri5_720p": dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4,
                                r_obs=60.0, theta_deg=85.0, phi_deg=0.0, fov_deg=30.0,
                                disk_out=20.0, width=1280, height=720),
    "kerr_ks_rk4_320x180": dict(chart=0, a=0.5, r_obs=40.0, theta_deg=80.0, phi_deg=0.0,
                                fov_deg=45.0, disk_out=12.0, width=320, height=180),
    "bundles_bl_1080p": dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=1920, height=1080),
    # config 3's geometry at a quarter and at half the resolution (profiling sizes)
    "bundles_bl_480x270": dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=480, height=270),
    "bundles_bl_960x540": dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=960, height=540),
    # configuration 2's geometry in mixed precision at tol 1e-8, where the FP32
    # right-hand side runs (profiling size)
    "knds_bl_dopri5_mixed_tol1e-8_640x360": dict(chart=1, integrator=1, tol=1e-8, a=0.9, Q=0.3,
                                                 Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
                                                 fov_deg=30.0, disk_out=20.0, width=640,
                                                 height=360, precision=1),
    "kn_ks_rk4_512": dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
                          width=512, height=512),
    # 64 seeded parameter sets (kerrtracecpp2_b200.random_parameter_sets, seed
    # 1) at 256^2..1024^2, KS chart requested, RK4 step doubling; one batch.
    "batch64_ks_rk4_seed1": dict(batch=64, seed=1, width=0, height=0, chart=0),
    # Config 5 gradient alone (adjoint_leg): value = adjoint ms per frame.
    "adjoint_ks_512": dict(adjoint=True, width=512, height=512, chart=0),
    # The semi-analytic solver (--bl --semi-analytic) at the CLI's default
    # Kerr frame, 720p, default step cap 500000: every ray with a radial
    # turning point parks there and runs to the cap, ~1 s of CPU per ray.
    # The elliptic-closed solver (--elliptic-closed) on config 1's Kerr frame
    # at 720p: the standard KS trace plus the closed-form disk crossings.
    "elliptic_ks_kerr_720p": dict(chart=0, solver_mode=2, a=0.5, r_obs=40.0, theta_deg=80.0,
                                  fov_deg=45.0, disk_out=12.0, width=1280, height=720),
    "semi_bl_kerr_720p": dict(chart=1, solver_mode=1, a=0.998, r_obs=40.0, theta_deg=80.0,
                              fov_deg=30.0, disk_out=12.0, width=1280, height=720,
                              cpu_calib_pixels=64),
}
# Frames of the batched 720p leg: the headline frame seen from this many
# camera azimuths, traced as one batch.
BATCH_720P_FRAMES = 8

# Algorithmic FP64 work, counted from the reference's arithmetic as
# kt_physics.cuh evaluates it (+, -, * = 1 flop, fma = 2), each division,
# square root, sincos and pow weighted by its cost measured on the device in
# the same run (kt_measure_op_costs: the FMA-pipe time of one operation at
# full throughput, in flops):
#   BL RHS (geodesic_rhs + dphi_vel): 211 flops of arithmetic (5 g^{mu nu}
#   evaluations: 28 flops full, 21 at the centre, 19 when only theta changes;
#   4 Hamiltonians of 16; 18 in the three angle factors; 14 for the offsets,
#   k and the differences), 26 divisions, 6 divisions by 3 (the Lambda/3
#   terms), 3 sincos.
#   DOPRI5 attempt: 6 RHS + 328 flops (stage sums 189, y5/y4 117, error norm
#   21, controller 1) + 5 divisions + 1 sqrt + 1 pow.
#   RK4 doubling attempt: 10 RHS + 219 flops (stage inputs/sums 207, error
#   11, controller 1) + 2 divisions + 1 sqrt + 1 pow; one more RHS per
#   accepted step.
# With unit weights (division, x/3 and sqrt 1 flop; sincos 70 and pow 113,
# the flops of their own arithmetic) the counts give 453, 447 and 335.
RHS_COUNTS = {"flops": 211.0, "div": 26.0, "div3": 6.0, "sincos": 3.0}
DOPRI5_ATTEMPT_COUNTS = {"flops": 328.0, "div": 5.0, "sqrt": 1.0, "pow": 1.0}
RK4_ATTEMPT_COUNTS = {"flops": 219.0, "div": 2.0, "sqrt": 1.0, "pow": 1.0}
UNIT_WEIGHTS = {"div": 1.0, "div3": 1.0, "sqrt": 1.0, "sincos": 70.0, "pow": 113.0}
# DRAM bytes read + written by one k_trace<ModeBLDopri5> launch on the
# default 720p frame, from one ncu capture of that launch
# (dram__bytes_read.sum 0.471 MB + dram__bytes_write.sum 3.600 MB): the
# frame's 52.5 MB of outputs stay in L2 during the launch.
TRAFFIC_DOPRI5_720P = 4.070144e6


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def start_clock_sampler(path):
    cmd = ["nvidia-smi",
           "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
           "--format=csv,noheader,nounits", "-lms", "200"]
    try:
        f = open(path, "w")
        return subprocess.Popen(cmd, stdout=f, stderr=subprocess.DEVNULL), f
    except (OSError, FileNotFoundError):
        return None, None


def stop_clock_sampler(proc, f, path, gpu_index):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
        proc.kill()
    f.close()
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in open(path):
        parts = [p.strip() for p in line.split(",")]
        if len(parts) < 9 or parts[0] != str(gpu_index):
            continue
        try:
            sm.append(float(parts[1]))
            mx.append(float(parts[2]))
        except ValueError:
            continue
        for n, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "samples": len(sm),
            "reasons": sorted(reasons)}


def weighted(counts, w):
    return counts["flops"] + sum(n * w[k] for k, n in counts.items() if k != "flops")


def ray_flops(desc, steps, attempts, w=UNIT_WEIGHTS):
    """Algorithmic FP64 flops of one traced frame from the kernel's counters,
    with operation weights w (flops per division, x/3, sqrt, sincos, pow)."""
    if (desc.bundles or desc.chart == 0 and abs(desc.Lambda) <= 1e-15 or desc.solver_mode != 0
            or desc.precision != 0):
        return None  # counted only for the standard BL single-ray integrators in FP64
    n = desc.width * desc.height
    f_rhs = weighted(RHS_COUNTS, w)
    if desc.integrator == 1:
        rhs = n + 6.0 * attempts
        return rhs * f_rhs + attempts * weighted(DOPRI5_ATTEMPT_COUNTS, w)
    rhs = n + 10.0 * attempts + steps
    return rhs * f_rhs + attempts * weighted(RK4_ATTEMPT_COUNTS, w)


ORDER_MIN_PIXELS = 1 << 16  # kt_internal.h kOrderMinPixels


def trace_launches(dv, desc):
    """Kernel launches of one kt_trace: the centre-out ray order of a whole
    frame of at least ORDER_MIN_PIXELS pixels (three kernels), the
    persistent trace kernel, the BL launch over the fallback list (KS chart,
    semi-analytic solver) and the elliptic-closed kernel."""
    from kerrtracecpp2_b200 import abi

    n = 1
    if desc.width * desc.height >= ORDER_MIN_PIXELS and desc.precision != abi.KT_PREC_SMOOTH:
        n += 3
    if not desc.bundles and (dv.chart == 0 or dv.solver == 1):
        n += 1
    if dv.solver == 2:
        n += 1
    return n


def cpu_reference_sample(desc, seconds, flavour="ieee", calib_pixels=None):
    """Time the reference's CPU path on a strided sample of the frame
    (calibrated on calib_pixels pixels, by default 512 or 16 per thread).

    Returns (rays_per_s, pixels, threads, kind, sample, results, seconds),
    seconds the time of the timed sample alone."""
    import oracle_lib as O  # noqa: E402  (tests/oracle_lib.py)

    n = desc.width * desc.height
    threads = os.cpu_count() or 1
    use_ref = O.ref_available(flavour)
    kind = "reference" if use_ref else "port"

    def trace(pix):
        if use_ref:
            return O.trace_ref(desc, flavour, pix=pix, nthreads=threads)
        return O.trace_port(desc, pix=pix, nthreads=threads)

    # calibrate on ~0.2% of the frame, then size the sample to `seconds`
    stride = max(1, n // (calib_pixels or max(512, threads * 16)))
    pix = np.arange(0, n, stride, dtype=np.uint32)
    t0 = time.perf_counter()
    trace(pix)
    rate = len(pix) / max(time.perf_counter() - t0, 1e-6)
    want = int(min(n, max(len(pix), rate * seconds)))
    stride = max(1, n // want)
    pix = np.arange(0, n, stride, dtype=np.uint32)
    t0 = time.perf_counter()
    res = trace(pix)
    dt = time.perf_counter() - t0
    sample = f"{len(pix)} of {n} pixels (every {stride}th, row-major) of the same frame"
    return len(pix) / dt, pix, threads, kind, sample, res, dt


ADJOINT_FRAME = dict(chart=0, a=0.7, Q=0.1, Lambda=0.0, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
                     width=512, height=512)

# Secondary legs of the default line run a few steps each (their frames take
# up to seconds per step).
LEG_STEPS = 3


def _timed_steps(fn, steps, warmup, stream, flush):
    """Device time (ms) of `steps` calls of fn, L2 flushed before each, after
    `warmup` untimed calls; one event pair around the whole loop."""
    import torch

    for _ in range(max(warmup, 1)):
        flush.fill_(1)
        fn()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    for _ in range(steps):
        flush.fill_(1)
        fn()
    ev[1].record(stream)
    torch.cuda.synchronize()
    return ev[0].elapsed_time(ev[1])


def bundles_leg(R, stream, flush):
    """Config 3: 1920x1080 Jacobi-bundle frame (BL, a=0.998, theta=60, r_obs
    40, fov 30, disk ISCO-12, RK4 doubling, tol 1e-7), plain FP64
    (bit-identical to the reference's records; rays creeping onto the
    horizon stop with the record their end gives) and, for the reference's
    counters as well, with KT_FLAG_BUNDLE_FULL_CREEP; mixed (analytic
    Hessian-vector products), with the mixed frame's error against the
    FP64 one."""
    import torch
    from kerrtracecpp2_b200 import abi

    kw = WORKLOADS["bundles_bl_1080p"]
    n = kw["width"] * kw["height"]
    d = abi.frame_desc(**kw)
    df = abi.frame_desc(**dict(kw, flags=abi.KT_FLAG_BUNDLE_FULL_CREEP))
    dm = abi.frame_desc(**dict(kw, precision=abi.KT_PREC_MIXED))
    o, of, om = R.alloc(n), R.alloc(n), R.alloc(n)
    t = _timed_steps(lambda: R.trace(d, o, stream), LEG_STEPS, 1, stream, flush)
    tf = _timed_steps(lambda: R.trace(df, of, stream), LEG_STEPS, 1, stream, flush)
    tm = _timed_steps(lambda: R.trace(dm, om, stream), LEG_STEPS, 1, stream, flush)
    torch.cuda.synchronize()
    rec_same = all(torch.equal(o[k], of[k]) for k in ("outcome", "r", "redshift", "magnif", "phi_disk",
                                                     "theta_esc", "phi_esc"))
    creep = int((o["status"] == abi.KT_RAY_CREEP).sum())
    same = o["outcome"] == om["outcome"]
    disk = same & (o["outcome"] == 1)
    eg = ((om["redshift"] - o["redshift"]).abs() / o["redshift"].abs())[disk]
    em = ((om["magnif"] - o["magnif"]).abs() / o["magnif"].abs())[disk]
    q = lambda x, p: float(torch.quantile(x.float(), p)) if x.numel() else None  # noqa: E731
    return {"frame": "1920x1080 Jacobi bundles, BL, a=0.998, theta=60, r_obs=40, fov=30, disk ISCO-12",
            "steps": LEG_STEPS, "fp64_value": LEG_STEPS * n / (t * 1e-3) / 1e6,
            "fp64_ms_per_step": t / LEG_STEPS, "fp64_creeping_rays_stopped": creep,
            "fp64_full_creep_value": LEG_STEPS * n / (tf * 1e-3) / 1e6,
            "fp64_full_creep_ms_per_step": tf / LEG_STEPS,
            "fp64_records_equal_full_creep": rec_same,
            "mixed_value": LEG_STEPS * n / (tm * 1e-3) / 1e6, "mixed_ms_per_step": tm / LEG_STEPS,
            "unit": "Mrays/s", "mixed_speedup": t / tm,
            "mixed_error_vs_fp64": {"class_mismatch_frac": float(1.0 - same.double().mean()),
                                    "g_rel_p50": q(eg, 0.5), "g_rel_p99": q(eg, 0.99),
                                    "magnif_rel_p50": q(em, 0.5), "magnif_rel_p99": q(em, 0.99)}}


def batch_leg(R, stream, flush, seed=1, frames=64):
    """Config 4: the 64 seeded parameter sets in one autotuned batch (one
    CUDA graph launch per step), against one kt_trace per frame."""
    import time as _t

    import kerrtracecpp2_b200 as kt
    from kerrtracecpp2_b200 import abi

    descs = kt.random_parameter_sets(frames, seed=seed)
    n_rays = sum(d.width * d.height for d in descs)
    t0 = _t.perf_counter()
    b = R.batch(descs, options=abi.batch_options(autotune=True))
    tune_s = _t.perf_counter() - t0
    steps = max(1, LEG_STEPS - 1)
    tb = _timed_steps(lambda: b.launch(stream), steps, 1, stream, flush)

    def per_frame():
        for d, o in zip(descs, b.outs):
            R.trace(d, o, stream)

    tl = _timed_steps(per_frame, steps, 0, stream, flush)
    groups = [{k: g[k] for k in ("kernel_name", "n_frames", "n_rays", "variant", "block",
                                 "min_blocks", "refill_min", "best_ms", "default_ms")}
              for g in b.groups()]
    b.close()
    return {"frames": frames, "seed": seed, "rays": n_rays, "steps": steps,
            "value": steps * n_rays / (tb * 1e-3) / 1e6, "unit": "Mrays/s",
            "ms_per_step": tb / steps, "autotune_s": tune_s,
            "per_frame_kt_trace_value": steps * n_rays / (tl * 1e-3) / 1e6,
            "speedup_vs_per_frame": tl / tb, "groups": groups,
            "mode": "plain FP64, bit-identical to the reference CPU path"}


def adjoint_leg(R, steps, warmup, stream, flush, frame=None, target=None, fd_check=True, w_m=0.0):
    """Config 5 (default): 512x512 KS frame, L2 loss of (g, r_hit) against
    the smooth tracer at a=0.72, theta=71; kt_l2_grad (fused forward +
    reverse per ray) timed on the device against kt_trace of the same frame
    (plain FP64, the reference's arithmetic) and the smooth forward alone.
    `frame` / `target` give another frame and the target's parameters; w_m
    adds a bundle frame's magnification to the loss."""
    import torch
    from kerrtracecpp2_b200 import abi

    frame = frame or ADJOINT_FRAME
    target = target or dict(a=0.72, theta_deg=71.0)
    n = frame["width"] * frame["height"]
    d = abi.frame_desc(**frame)
    ds = abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **frame)
    tgt = R.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **dict(frame, **target)))
    out = R.alloc(n)

    def timed(fn):
        for _ in range(max(warmup, 1)):
            flush.fill_(1)
            fn()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps)]
        for i in range(steps):
            flush.fill_(1)
            ev[2 * i].record(stream)
            fn()
            ev[2 * i + 1].record(stream)
        torch.cuda.synchronize()
        return float(np.mean([ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(steps)]))

    fwd_ms = timed(lambda: R.trace(d, out, stream))
    smooth_ms = timed(lambda: R.trace(ds, out, stream))
    res = {}

    def grad():
        res["r"] = R.l2_grad(d, tgt, 1.0, 0.01, out=out, stream=stream, w_m=w_m)

    grad_ms = timed(grad)
    loss, g, st = res["r"]
    desc_txt = {k: frame[k] for k in ("width", "height", "chart", "bundles", "a", "Q", "Lambda",
                                      "theta_deg", "r_obs", "disk_out") if k in frame}
    desc_txt["integrator"] = ("DOPRI5" if frame.get("integrator", 0) == 1 and not frame.get("bundles")
                              else "RK4-doubling")
    desc_txt["tol"] = frame.get("tol", 1e-7)
    mterm = f" + {w_m:g} (magnif-magnif_t)^2" if w_m else ""
    leg = {"frame": desc_txt,
           "loss": f"sum over pixels that are disk hits in both frames of (g-g_t)^2 + 0.01 (r-r_t)^2{mterm}, "
                   f"target: the same tracer at {target}",
           "ms_per_frame": grad_ms, "ms_main_pass": st["ms_main"], "ms_lambda_pass": st["ms_lambda"],
           "forward_fp64_ms": fwd_ms, "forward_smooth_ms": smooth_ms,
           "ratio_vs_forward_fp64": grad_ms / fwd_ms,
           "grad": dict(zip(abi.GRAD_NAMES, [float(x) for x in g])), "loss_value": loss,
           "grad_pixels": st["grad_pixels"], "unrecorded": st["unrecorded"],
           "checkpoint_interval_steps": 32}
    if not fd_check:
        return leg
    # Central differences of the same loss (tests/grad_lib.py): five-point
    # at h = 1e-4 and two-point at h = 1e-6, on the pixels whose stencil
    # renders keep their class and step sequence.
    import grad_lib  # noqa: E402  (tests/grad_lib.py)

    fd = grad_lib.fd_check(R)
    return {"frame": "512x512 KS, a=0.7, Q=0.1, theta=70, r_obs=50, disk ISCO-15, tol 1e-7",
            "loss": "sum over pixels that are disk hits in both frames of (g-g_t)^2 + 0.01 (r-r_t)^2, "
                    "target: the same tracer at a=0.72, theta=71",
            "ms_per_frame": grad_ms, "ms_main_pass": st["ms_main"], "ms_lambda_pass": st["ms_lambda"],
            "forward_fp64_ms": fwd_ms, "forward_smooth_ms": smooth_ms,
            "ratio_vs_forward_fp64": grad_ms / fwd_ms,
            "ratio_vs_forward_fp64_without_lambda_pass": st["ms_main"] / fwd_ms,
            "grad": dict(zip(abi.GRAD_NAMES, [float(x) for x in g])), "loss_value": loss,
            "grad_pixels": st["grad_pixels"], "unrecorded": st["unrecorded"],
            "checkpoint_interval_steps": 32,
            "fd_rel_h1e-4_5pt": fd["five_point"]["worst_rel"],
            "fd_rel_h1e-6": fd["two_point"]["worst_rel"],
            "fd_rel_h1e-6_loose_mask": fd["two_point_loose"]["worst_rel"],
            "smooth_pixels": fd["five_point"]["pixels"],
            "smooth_pixels_h1e-6": fd["two_point"]["pixels"],
            "pixels_h1e-6_loose_mask": fd["two_point_loose"]["pixels"],
            "disk_pixels": fd["five_point"]["disk_pixels"],
            "fd_per_param": {k: {"h1e-4_5pt": fd["five_point"]["per_param"][k]["rel"],
                                 "h1e-6": fd["two_point"]["per_param"][k]["rel"],
                                 "h1e-6_loose_mask": fd["two_point_loose"]["per_param"][k]["rel"]}
                             for k in grad_lib.PARAMS},
            "fd_check": ("worst relative disagreement over (a, Q, Lambda, theta, r_obs) of the "
                         "adjoint with central differences of the same loss over the pixels whose "
                         "stencil renders keep class, step and attempt counts: five-point with "
                         "h = 1e-4 (Lambda 1e-6) on pixels also without second-difference spikes "
                         "or kinks; two-point with h = 1e-6 (Lambda 1e-8) on those pixels, and "
                         "on every pixel whose class and step sequence survive +-1e-6 (loose)")}


def bench_adjoint(args, rank, world, local_rank):
    """The config-5 gradient as its own line: value = adjoint ms per frame
    (kt_l2_grad, both passes), one frame per GPU; the reference has no
    gradient, so its arm is unavailable for this workload."""
    cfg = {"workload": args.workload, "width": 512, "height": 512, "chart": "KS", "a": 0.7, "Q": 0.1,
           "theta": 70.0, "r_obs": 50.0, "tol": 1e-7, "parallelism": f"frames{args.gpus}",
           "l2": "256 MB flush between steps"}
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference renderer has no "
                              "gradient (no adjoint or VJP entry)"}), flush=True)
        return 0
    import torch

    import kerrtracecpp2_b200 as kt

    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    R = kt.Renderer(local_rank)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)
    adj = adjoint_leg(R, args.steps, args.warmup, stream, flush)
    line = {"metric": METRIC, "value": adj["ms_per_frame"], "unit": "ms/frame (adjoint)",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": adj["ms_per_frame"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (procedural camera frame; no dataset)",
            "config": cfg, "adjoint": adj, "gpu_launches": args.steps * 9}
    if rank == 0:
        print(json.dumps(line), flush=True)
    R.close()
    return 0


def cpu_reference_batch(descs, seconds, flavour="ieee"):
    """The reference's CPU path on the same strided fraction of every frame
    of a batch.  Returns (rays_per_s, threads, kind, sample, seconds), seconds
    the time of the timed sample alone."""
    import oracle_lib as O  # noqa: E402  (tests/oracle_lib.py)

    threads = os.cpu_count() or 1
    use_ref = O.ref_available(flavour)
    kind = "reference" if use_ref else "port"

    def run(stride):
        t0 = time.perf_counter()
        rays = 0
        for d in descs:
            pix = np.arange(0, d.width * d.height, stride, dtype=np.uint32)
            if use_ref:
                O.trace_ref(d, flavour, pix=pix, nthreads=threads)
            else:
                O.trace_port(d, pix=pix, nthreads=threads)
            rays += len(pix)
        return rays, time.perf_counter() - t0

    total = sum(d.width * d.height for d in descs)
    stride = max(1, total // (len(descs) * max(64, threads * 4)))
    rays, dt = run(stride)
    rate = rays / max(dt, 1e-6)
    stride = max(1, int(total / max(rays, rate * seconds)))
    rays, dt = run(stride)
    sample = (f"{rays} of {total} rays: every {stride}th pixel (row-major) of each of the "
              f"{len(descs)} frames")
    return rays / dt, threads, kind, sample, dt


def bench_batch(args, wl, base_cfg, rank, world, local_rank):
    """Config 4: 64 seeded parameter sets at uneven resolutions, one CUDA
    graph launch per step (kt_batch_launch), launch variants and regroup
    thresholds chosen by the autotuner.  The per-frame kt_trace loop over
    the same frames is timed beside it."""
    import kerrtracecpp2_b200 as kt
    from kerrtracecpp2_b200 import abi

    from kerrtracecpp2_b200 import shard

    all_descs = kt.random_parameter_sets(wl["batch"], seed=wl["seed"])
    # N > 1: the 64 frames are dealt to the ranks longest-first by estimated
    # cost (shard.assign_frames); each rank traces its share as one batch, and
    # the value is all 64 frames' rays over the slowest rank's time.
    parts = shard.assign_frames([shard.frame_cost(d) for d in all_descs], world)
    descs = [all_descs[i] for i in parts[rank]] if world > 1 else all_descs
    n_rays_all = sum(d.width * d.height for d in all_descs)
    n_rays = sum(d.width * d.height for d in descs)
    common = {"metric": METRIC, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
              "warmup": args.warmup, "higher_is_better": True,
              "scaling": "strong" if world > 1 else "weak",
              "vs_baseline": None, "dtype": "f64",
              "data": "synthetic (seeded random parameter sets; no dataset)", "config": base_cfg}
    if args.impl == "reference":
        if rank != 0:
            return 0
        per_step = max(2.0, 120.0 / max(1, args.steps + args.warmup))
        for _ in range(args.warmup):
            cpu_reference_batch(all_descs, per_step)
        rates, secs, info = [], [], None
        for _ in range(args.steps):
            rate, threads, kind, sample, dt = cpu_reference_batch(all_descs, per_step)
            rates.append(rate)
            secs.append(dt)
            info = (threads, kind, sample)
        v = float(np.mean(rates)) / 1e6
        # ms_per_step: the time each step took (a bounded sample of the
        # batch); value: rays per second of those samples.
        line = dict(common, impl="reference", value=v, ms_per_step=1e3 * float(np.mean(secs)),
                    cpu_baseline={"value": v, "unit": "Mrays/s", "cores": info[0], "kind": info[1],
                                  "sample": info[2]},
                    e2e={"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                         "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return 0

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    R = kt.Renderer(local_rank)
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    t0 = time.perf_counter()
    b = R.batch(descs, options=abi.batch_options(autotune=True))
    tune_s = time.perf_counter() - t0
    groups = b.groups()
    for _ in range(max(args.warmup, 1)):
        flush.fill_(1)
        b.launch(stream)
    torch.cuda.synchronize(device)

    def timed(fn):
        if dist:
            dist.barrier()
        torch.cuda.synchronize(device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(args.steps):
            flush.fill_(1)
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize(device)
        t = torch.tensor([ev[0].elapsed_time(ev[1])], dtype=torch.float64, device=device)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0])

    clk_path = os.path.join(tempfile.gettempdir(), f"kt_clocks_{os.getpid()}.csv")
    proc, fh = start_clock_sampler(clk_path)
    time.sleep(0.3)
    total_ms = timed(lambda: b.launch(stream))
    clocks = stop_clock_sampler(proc, fh, clk_path, local_rank)
    value = args.steps * n_rays_all / (total_ms * 1e-3) / 1e6

    # The same frames, one kt_trace per frame (the reference's one frame per
    # render call), into the same outputs.
    def per_frame():
        for d, o in zip(descs, b.outs):
            R.trace(d, o, stream)

    seq_ms = timed(per_frame)
    seq_value = args.steps * n_rays_all / (seq_ms * 1e-3) / 1e6

    # Algorithmic flops of the BL frames (the FP64 roofline counts cover the
    # BL integrators); the KS frames' share of the time is not attributed.
    flops_bl, rays_bl = 0.0, 0
    for d, o in zip(descs, b.outs):
        f = ray_flops(d, float(o["steps"].to(torch.int64).sum()),
                      float(o["attempts"].to(torch.int64).sum()))
        if f is not None:
            flops_bl += f
            rays_bl += d.width * d.height

    # End to end: launch + copy every frame's results to pinned host memory.
    host = [{k: torch.empty(d.width * d.height, dtype=o[k].dtype, pin_memory=True)
             for k in ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")}
            for d, o in zip(descs, b.outs)]
    d2h = sum(t.numel() * t.element_size() for h in host for t in h.values())
    e2e_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        b.launch(stream)
        for h, o in zip(host, b.outs):
            for k, t in h.items():
                t.copy_(o[k], non_blocking=True)
        torch.cuda.synchronize(device)
        e2e_ms.append(1e3 * (time.perf_counter() - t1))
    et = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = args.steps * n_rays_all / (float(et[0]) * 1e-3) / 1e6

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        rate, threads, kind, sample, _ = cpu_reference_batch(descs, args.cpu_seconds)
        cpu = {"value": rate / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
               "sample": sample + ("; reference built -O3 without -ffast-math, glibc libm"
                                   if kind == "reference" else "")}

    launches = sum(1 + (1 if g["kernel_name"].startswith("ks_rk4") else 0) for g in groups)
    line = dict(common, value=value, ms_per_step=total_ms / args.steps,
                mode="plain FP64, bit-identical to the reference CPU path",
                batch={"frames": len(all_descs), "rays": n_rays_all,
                       "frames_rank0": len(descs), "rays_rank0": n_rays,
                       "assignment": "longest-first by estimated cost (shard.assign_frames)"
                       if world > 1 else "all frames on one GPU",
                       "graph_launches_per_step": 1,
                       "autotune_s": tune_s, "groups": groups,
                       "per_frame_kt_trace": {"value": seq_value, "unit": "Mrays/s",
                                              "ms_per_step": seq_ms / args.steps},
                       "speedup_vs_per_frame": value / seq_value},
                roofline=None, roofline_note=(
                    f"BL frames: {rays_bl} rays, {flops_bl:.4g} algorithmic FP64 flops per step (unit weights); "
                    "KS RHS flops are not counted, so no whole-batch roofline"),
                cpu_baseline=cpu,
                e2e={"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                     "d2h_bytes_per_step": d2h,
                     "call": "kt_batch_launch + copies of every frame's results to pinned host"},
                clocks=clocks, gpu_launches=args.steps * launches)
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    R.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def bench_tiles(args, wl, base_cfg, rank, world, local_rank):
    """One frame split over the ranks by interleaved 16x16 tiles
    (shard.frame_tiles): every rank traces its tiles (kt_trace_pixels) and
    the parts are gathered on rank 0 (shard.trace_frame_sharded: one NCCL
    gather of a byte buffer per rank), every step.  Total work is fixed as N
    grows (strong scaling); value = the frame's pixels per step over the
    slowest rank's device time."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    import kerrtracecpp2_b200 as kt
    from kerrtracecpp2_b200 import abi, shard

    torch.cuda.set_device(local_rank)
    dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = torch.device("cuda", local_rank)
    R = kt.Renderer(local_rank)
    desc = abi.frame_desc(**wl)
    n = desc.width * desc.height
    stream = torch.cuda.current_stream(device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    fields = [k for k, dt in abi.GEO_FIELDS if k not in ("status", "steps", "attempts")]

    def step():
        return shard.trace_frame_sharded(R, desc, fields=fields)

    for _ in range(max(args.warmup, 1)):
        flush.fill_(1)
        step()
    torch.cuda.synchronize(device)
    clk_path = os.path.join(tempfile.gettempdir(), f"kt_clocks_{os.getpid()}.csv")
    proc, fh = start_clock_sampler(clk_path)
    time.sleep(0.3)
    dist.barrier()
    torch.cuda.synchronize(device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    frame = None
    for _ in range(args.steps):
        flush.fill_(1)
        frame = step()
    ev[1].record(stream)
    torch.cuda.synchronize(device)
    dist.barrier()
    clocks = stop_clock_sampler(proc, fh, clk_path, local_rank)
    t = torch.tensor([ev[0].elapsed_time(ev[1])], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms = float(t[0])
    value = args.steps * n / (total_ms * 1e-3) / 1e6
    # end to end: the sharded step plus rank 0's copy of the frame to pinned
    # host memory, host wall clock, max over ranks
    host = {k: torch.empty(n, dtype=v.dtype, pin_memory=True) for k, v in frame.items()} \
        if frame is not None else {}
    e2e = []
    for _ in range(args.steps):
        dist.barrier()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        f = step()
        if f is not None:
            for k, v in f.items():
                host[k].copy_(v, non_blocking=True)
        torch.cuda.synchronize(device)
        e2e.append(1e3 * (time.perf_counter() - t0))
    et = torch.tensor([sum(e2e)], dtype=torch.float64, device=device)
    dist.all_reduce(et, op=dist.ReduceOp.MAX)
    d2h = sum(v.numel() * v.element_size() for v in host.values())
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (procedural camera frame; no dataset)",
            "config": dict(base_cfg, parallelism=f"tiles{world}", split="16x16 tiles round-robin"),
            "mode": "plain FP64, bit-identical to the reference CPU path",
            "e2e": {"value": args.steps * n / (float(et[0]) * 1e-3) / 1e6, "unit": "Mrays/s",
                    "h2d_bytes_per_step": ctypes.sizeof(desc), "d2h_bytes_per_step": d2h,
                    "call": "kt_trace_pixels per rank + NCCL gather + copy to pinned host (rank 0)"},
            "clocks": clocks, "gpu_launches": args.steps * 2}
    if rank == 0:
        print(json.dumps(line), flush=True)
    R.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="knds_bl_dopri5_720p", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the config-3 (bundles) and config-4 (batch) legs of the default line")
    ap.add_argument("--split", default="frames", choices=["frames", "tiles"],
                    help="N>1: 'frames' gives every rank its own frame (weak scaling); 'tiles' "
                         "splits one frame over the ranks by interleaved tiles (strong scaling)")
    args = ap.parse_args()
    sys.path.insert(0, os.path.join(ROOT, "tests"))

    rank = env_int("RANK", 0)
    world = env_int("WORLD_SIZE", 1)
    local_rank = env_int("LOCAL_RANK", 0)
    from kerrtracecpp2_b200 import abi

    wl = dict(WORKLOADS[args.workload])
    calib = wl.pop("cpu_calib_pixels", None)
    if wl.get("solver_mode", 0) != 0:
        # the semi-analytic solver runs in FP64 only; no gradient leg
        args.no_mixed = args.no_adjoint = True
    if wl.get("adjoint"):
        return bench_adjoint(args, rank, world, local_rank)
    if wl.get("batch"):
        base_cfg = {"workload": args.workload, "frames": wl["batch"], "seed": wl["seed"],
                    "sizes": "square, side ~ U{256..1024} step 16", "chart": "KS requested "
                    "(Lambda != 0 frames run in BL, as the reference does)",
                    "integrator": "RK4-doubling", "tol": 1e-7,
                    "parallelism": f"frames{args.gpus}", "l2": "256 MB flush between steps"}
        return bench_batch(args, wl, base_cfg, rank, world, local_rank)
    base_cfg = {"workload": args.workload, "width": wl["width"], "height": wl["height"],
                "chart": "BL" if wl.get("chart", 0) == 1 else "KS",
                "integrator": "DOPRI5" if wl.get("integrator", 0) == 1 else "RK4-doubling",
                "tol": wl.get("tol", 1e-7), "a": wl.get("a"), "Q": wl.get("Q", 0.0),
                "Lambda": wl.get("Lambda", 0.0), "bundles": bool(wl.get("bundles", 0)),
                "solver": ["standard", "semi-analytic", "elliptic-closed"][wl.get("solver_mode", 0)],
                "parallelism": f"frames{args.gpus}", "l2": "256 MB flush between steps"}

    if args.split == "tiles" and args.impl != "reference":
        if "MASTER_PORT" not in os.environ:  # one process, not launched by torchrun
            import socket

            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(sk.getsockname()[1]),
                                  RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
        return bench_tiles(args, wl, base_cfg, rank, world, local_rank)
    if args.impl == "reference":
        if rank != 0:
            return 0
        desc = abi.frame_desc(**wl)
        per_step = max(2.0, 120.0 / max(1, args.steps + args.warmup))
        for _ in range(args.warmup):
            cpu_reference_sample(desc, per_step, calib_pixels=calib)
        rates, secs = [], []
        info = None
        for _ in range(args.steps):
            rate, pix, threads, kind, sample, _, dt = cpu_reference_sample(desc, per_step,
                                                                           calib_pixels=calib)
            rates.append(rate)
            secs.append(dt)
            info = (threads, kind, sample)
        v = float(np.mean(rates)) / 1e6
        # ms_per_step: the time each step took (a bounded sample of the
        # frame, described in cpu_baseline.sample); value: rays per second.
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * float(np.mean(secs)),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (procedural camera frame; no dataset)", "config": base_cfg,
                "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": info[0], "kind": info[1],
                                 "sample": info[2] + ("; reference built -O3 without -ffast-math, "
                                                      "glibc libm" if info[1] == "reference" else "")},
                "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch

    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    import kerrtracecpp2_b200 as kt

    R = kt.Renderer(local_rank)
    if world > 1:
        wl["phi_deg"] = 360.0 * rank / world
    desc = abi.frame_desc(**wl)
    n = desc.width * desc.height
    out = R.alloc(n, counters=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)
    stream = torch.cuda.current_stream(device)

    def step():
        flush.fill_(1)
        R.trace(desc, out, stream)

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize(device)

    clk_path = os.path.join(tempfile.gettempdir(), f"kt_clocks_{os.getpid()}.csv")
    proc, fh = start_clock_sampler(clk_path)
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 2)]
    ev[0].record(stream)
    for i in range(args.steps):
        flush.fill_(1)
        ev[2 + 2 * i].record(stream)
        R.trace(desc, out, stream)
        ev[3 + 2 * i].record(stream)
    ev[1].record(stream)
    torch.cuda.synchronize(device)
    if dist:
        dist.barrier()
    clocks = stop_clock_sampler(proc, fh, clk_path, local_rank)
    total_ms = ev[0].elapsed_time(ev[1])
    kern_ms = [ev[2 + 2 * i].elapsed_time(ev[3 + 2 * i]) for i in range(args.steps)]
    t = torch.tensor([total_ms, float(np.mean(kern_ms))], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    total_ms, kernel_ms = float(t[0]), float(t[1])
    value = world * args.steps * n / (total_ms * 1e-3) / 1e6

    # Mixed precision (KT_PREC_MIXED), timed the same way; its error is taken
    # against this run's FP64 frame, which is bit-identical to the reference.
    def timed_ms(desc_, out_):
        """Device time of args.steps kt_trace calls (L2 flushed before each),
        max over ranks, after warm-up."""
        for _ in range(max(args.warmup, 1)):
            flush.fill_(1)
            R.trace(desc_, out_, stream)
        torch.cuda.synchronize(device)
        if dist:
            dist.barrier()
        tev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        tev[0].record(stream)
        for _ in range(args.steps):
            flush.fill_(1)
            R.trace(desc_, out_, stream)
        tev[1].record(stream)
        torch.cuda.synchronize(device)
        tt = torch.tensor([tev[0].elapsed_time(tev[1])], dtype=torch.float64, device=device)
        if dist:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt[0])

    def error_table(got, ref):
        """Mixed against FP64 (bit-identical to the reference): class
        mismatches over the frame; relative g and hit-radius error over the
        pixels that are disk hits in both."""
        same = ref["outcome"] == got["outcome"]
        disk = same & (ref["outcome"] == 1)
        eg = ((got["redshift"] - ref["redshift"]).abs() / ref["redshift"].abs())[disk]
        er = ((got["r"] - ref["r"]).abs() / ref["r"].abs())[disk]
        q = lambda x, p: float(torch.quantile(x.float(), p)) if x.numel() else None  # noqa: E731
        return {"pixels": n, "class_mismatch_frac": float(1.0 - same.double().mean()),
                "g_rel_p50": q(eg, 0.5), "g_rel_p90": q(eg, 0.9), "g_rel_p99": q(eg, 0.99),
                "g_rel_max": float(eg.max()) if eg.numel() else None,
                "g_rel_frac_above_1e-6": float((eg > 1e-6).double().mean()) if eg.numel() else None,
                "r_hit_rel_p50": q(er, 0.5), "r_hit_rel_p99": q(er, 0.99),
                "r_hit_rel_max": float(er.max()) if er.numel() else None}

    # Mixed precision (KT_PREC_MIXED) on the same frame, timed the same way;
    # its error is taken against this run's FP64 frame, which is
    # bit-identical to the reference.  Below tol 1e-8 the FP32 right-hand
    # side is off (FP32 rounding would be seen by the error control as
    # error): this leg is the analytic FP64 Hamiltonian gradient with the
    # mixed path's reciprocals and sincos.
    mixed = None
    mixed_fp32 = None
    if not args.no_mixed:
        mdesc = abi.frame_desc(**dict(wl, precision=abi.KT_PREC_MIXED))
        mout = R.alloc(n, counters=True)
        mt = timed_ms(mdesc, mout)
        mval = world * args.steps * n / (mt * 1e-3) / 1e6
        fp32_on = kt.frame_derive(mdesc).r_fp32 != float("inf")
        mixed = {"value": mval, "unit": "Mrays/s", "speedup_vs_fp64": mval / value,
                 "ms_per_step": mt / args.steps,
                 "form": ("FP32 right-hand side beyond r_fp32, FP64 near the horizon, at turning "
                          "points and in the integrator" if fp32_on else
                          "analytic FP64 Hamiltonian gradient (FP32 right-hand side off below "
                          "tol 1e-8)"),
                 "error_vs_fp64_oracle": error_table(mout, out),
                 "fp32_rhs": "used beyond r_fp32" if fp32_on
                 else "off at this tolerance (analytic FP64 gradient)"}
        # The same frame at tol 1e-8, where the FP32 right-hand side is taken
        # beyond r_fp32 = max(4M, 2 r+): plain FP64 and mixed, each timed,
        # the error against the FP64 frame at that tolerance.
        if fp32_on is False and wl.get("tol", 1e-7) < 1e-8 and not wl.get("bundles"):
            d8 = abi.frame_desc(**dict(wl, tol=1e-8))
            m8 = abi.frame_desc(**dict(wl, tol=1e-8, precision=abi.KT_PREC_MIXED))
            o8 = R.alloc(n, counters=True)
            t8 = timed_ms(d8, o8)
            t8m = timed_ms(m8, mout)
            v8 = world * args.steps * n / (t8 * 1e-3) / 1e6
            v8m = world * args.steps * n / (t8m * 1e-3) / 1e6
            dv8 = kt.frame_derive(m8)
            mixed_fp32 = {"tol": 1e-8, "value": v8m, "unit": "Mrays/s", "fp64_value": v8,
                          "speedup_vs_fp64_same_tol": v8m / v8, "ms_per_step": t8m / args.steps,
                          "fp64_ms_per_step": t8 / args.steps,
                          "form": "FP32 right-hand side beyond r_fp32, FP64 near the horizon, at "
                                  "radial and polar turning points, in the error estimate, the "
                                  "step-size controller, the constraint reprojection and the disk "
                                  "crossing",
                          "r_fp32": dv8.r_fp32,
                          "error_vs_fp64_oracle_same_tol": error_table(mout, o8)}
            del o8
        del mout

    # Mixed precision, batched: BATCH_720P_FRAMES frames of this workload (the
    # camera at azimuths 360*k/F deg) as one autotuned kt_batch, one graph
    # launch per step.
    mixed_batched = None
    if mixed is not None and not args.no_batch and args.workload == "knds_bl_dopri5_720p":
        descs = [abi.frame_desc(**dict(wl, precision=abi.KT_PREC_MIXED,
                                       phi_deg=wl.get("phi_deg", 0.0) + 360.0 * k / BATCH_720P_FRAMES))
                 for k in range(BATCH_720P_FRAMES)]
        b = R.batch(descs, options=abi.batch_options(autotune=True))
        for _ in range(max(args.warmup, 1)):
            flush.fill_(1)
            b.launch(stream)
        torch.cuda.synchronize(device)
        if dist:
            dist.barrier()
        bev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        bev[0].record(stream)
        for _ in range(args.steps):
            flush.fill_(1)
            b.launch(stream)
        bev[1].record(stream)
        torch.cuda.synchronize(device)
        bt = torch.tensor([bev[0].elapsed_time(bev[1])], dtype=torch.float64, device=device)
        if dist:
            dist.all_reduce(bt, op=dist.ReduceOp.MAX)
        bval = world * args.steps * n * BATCH_720P_FRAMES / (float(bt[0]) * 1e-3) / 1e6
        f0 = b.outs[0]
        same = f0["outcome"] == out["outcome"]
        disk = same & (out["outcome"] == 1)
        eg = ((f0["redshift"] - out["redshift"]).abs() / out["redshift"].abs())[disk]
        mixed_batched = {"value": bval, "unit": "Mrays/s", "frames": BATCH_720P_FRAMES,
                         "speedup_vs_fp64": bval / value,
                         "ms_per_step": float(bt[0]) / args.steps,
                         "groups": [{k: g[k] for k in ("kernel_name", "variant", "block", "min_blocks",
                                                        "grid", "refill_min", "best_ms", "default_ms")}
                                    for g in b.groups()],
                         "error_vs_fp64_oracle_frame0": {
                             "class_mismatch_frac": float(1.0 - same.double().mean()),
                             "g_rel_p50": float(torch.quantile(eg.float(), 0.5)) if eg.numel() else None,
                             "g_rel_p99": float(torch.quantile(eg.float(), 0.99)) if eg.numel() else None}}
        b.close()
        del b

    adjoint = adjoint_dopri5 = adjoint_bundle = None
    if not args.no_adjoint:
        adjoint = adjoint_leg(R, args.steps, args.warmup, stream, flush)
        if args.workload == "knds_bl_dopri5_720p":
            # the DOPRI5 adjoint on this run's own frame (configuration 2, 720p)
            adjoint_dopri5 = adjoint_leg(R, min(args.steps, LEG_STEPS), 1, stream, flush,
                                         frame=WORKLOADS["knds_bl_dopri5_720p"],
                                         target=dict(a=0.92, theta_deg=86.0), fd_check=False)
            if not args.no_legs:
                # the bundle adjoint, magnification in the loss (configuration
                # 3's geometry at 960x540)
                adjoint_bundle = adjoint_leg(R, min(args.steps, LEG_STEPS), 1, stream, flush,
                                             frame=WORKLOADS["bundles_bl_960x540"],
                                             target=dict(a=0.99, theta_deg=61.0), fd_check=False,
                                             w_m=0.01)

    # Configs 3 and 4 as legs of the default line (one GPU).
    bundles = batch64 = None
    if world == 1 and args.workload == "knds_bl_dopri5_720p" and not args.no_legs:
        bundles = bundles_leg(R, stream, flush)
        batch64 = batch_leg(R, stream, flush)

    steps_sum = float(out["steps"].to(torch.int64).sum())
    att_sum = float(out["attempts"].to(torch.int64).sum())
    costs = R.op_costs()
    weights = {k: costs[k] for k in UNIT_WEIGHTS}
    flops = ray_flops(desc, steps_sum, att_sum, weights)
    flops_unit = ray_flops(desc, steps_sum, att_sum)
    peak_gflops = R.fp64_peak_gflops()
    roofline = None
    if flops is not None:
        achieved = flops / (kernel_ms * 1e-3) / 1e12
        peak = peak_gflops / 1e3
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak,
                    "traffic": TRAFFIC_DOPRI5_720P if args.workload == "knds_bl_dopri5_720p" else None,
                    "peak_source": "measured in this run: kt_measure_fp64_peak (dependent FMA chains, all SMs)",
                    "flops_per_frame": flops,
                    "op_weights_flops": {k: round(v, 2) for k, v in weights.items()},
                    "op_weights_source": "measured in this run: kt_measure_op_costs (throughput against FMA)",
                    "frac_unit_weights": flops_unit / (kernel_ms * 1e-3) / 1e12 / peak,
                    "flops_per_frame_unit_weights": flops_unit,
                    "rhs_per_ray": (n + 6.0 * att_sum) / n
                    if desc.integrator == 1 else (n + 10.0 * att_sum + steps_sum) / n,
                    "kernel_ms": kernel_ms}

    # end to end through the public host-buffer call (kt_trace_host): the
    # frame parameters go in, the per-pixel results come back to pinned host
    # memory inside the timed region.
    host = {k: torch.empty(n, dtype={"u1": torch.uint8, "f8": torch.float64}[dt],
                           pin_memory=True).numpy()
            for k, dt in abi.GEO_FIELDS if dt in ("u1", "f8") and k != "status"}
    soa = abi.GeoSoA()
    for k, _ in abi.GEO_FIELDS:
        setattr(soa, k, host[k].ctypes.data_as(ctypes.c_void_p) if k in host else None)
    L = kt.load_library()
    for _ in range(1):
        L.kt_trace_host(R.ctx, ctypes.byref(desc), ctypes.byref(soa))
    e2e_ms = []
    for _ in range(args.steps):
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        st = L.kt_trace_host(R.ctx, ctypes.byref(desc), ctypes.byref(soa))
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        if st != 0:
            raise RuntimeError(L.kt_last_error(R.ctx).decode())
    et = torch.tensor([sum(e2e_ms)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps * n / (float(et[0]) * 1e-3) / 1e6
    d2h = sum(host[k].nbytes for k in host)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle_lib as O  # noqa: E402  (tests/oracle_lib.py)

        rate, pix, threads, kind, sample, res, _ = cpu_reference_sample(desc, args.cpu_seconds,
                                                                        calib_pixels=calib)
        got_out = out["outcome"].cpu().numpy()[pix]
        got_g = out["redshift"].cpu().numpy()[pix]
        disk = (got_out == 1) & (res["outcome"] == 1)
        rel = np.abs(got_g[disk] - res["redshift"][disk]) / np.maximum(np.abs(res["redshift"][disk]), 1e-300)
        cpu = {"value": rate / 1e6, "unit": "Mrays/s", "cores": threads, "kind": kind,
               "sample": sample + ("; reference built -O3 without -ffast-math, glibc libm"
                                   if kind == "reference" else ""),
               "class_mismatch_vs_gpu": int(np.sum(got_out != res["outcome"])),
               "class_mismatch_boundary_distance_px": O.boundary_distance(
                   out["outcome"].cpu().numpy().reshape(desc.height, desc.width),
                   pix[got_out != res["outcome"]]),
               "g_rel_diff_vs_gpu_median": float(np.median(rel)) if rel.size else None}

    # Per-pixel parity of this run's frame with the strict oracle (the C
    # restatement, bit-identical to the reference compiled without
    # contraction and with the renderer's libm on every golden fixture),
    # over the whole frame (Jacobi bundles: every 16th pixel).
    parity = None
    if (rank == 0 and world == 1 and not args.no_parity and wl.get("solver_mode", 0) != 1
            and desc.precision == 0):
        import oracle_lib as O  # noqa: E402  (tests/oracle_lib.py)

        stride = 16 if desc.bundles else 1
        pix = np.arange(0, n, stride, dtype=np.uint32)
        t0 = time.perf_counter()
        want = O.trace_port(desc, pix=None if stride == 1 else pix, counters=True)
        t_oracle = time.perf_counter() - t0
        got = {k: out[k].cpu().numpy() for k in O.GEO_FIELDS}
        got["steps"] = out["steps"].cpu().numpy().view(np.uint32)
        got["attempts"] = out["attempts"].cpu().numpy().view(np.uint32)
        got["status"] = out["status"].cpu().numpy()  # creeping bundle rays: counters stop early
        parity = dict(O.parity_report(got, want, desc.width, desc.height, pix=pix),
                      oracle="oracle/kt_oracle.c (strict: no contraction, the renderer's libm; "
                             "bit-identical to the reference built that way on every golden fixture)",
                      sample="every pixel" if stride == 1 else f"every {stride}th pixel (row-major)",
                      oracle_seconds=t_oracle, oracle_threads=os.cpu_count())

    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (procedural camera frame; no dataset)", "config": base_cfg,
            "mode": "plain FP64, bit-identical to the reference CPU path" if desc.precision == 0
            else ["plain FP64", "mixed precision", "smooth tracer"][desc.precision],
            "roofline": roofline, "cpu_baseline": cpu, "parity_vs_strict": parity,
            "mixed_precision": mixed, "mixed_precision_fp32_tol1e-8": mixed_fp32,
            "mixed_batched": mixed_batched, "adjoint": adjoint, "adjoint_dopri5_720p": adjoint_dopri5,
            "adjoint_bundles_960x540": adjoint_bundle,
            "bundles_1080p": bundles, "batch64": batch64,
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": ctypes.sizeof(desc),
                    "d2h_bytes_per_step": d2h, "call": "kt_trace_host"},
            "clocks": clocks, "gpu_launches": args.steps * trace_launches(kt.frame_derive(desc), desc)
            * (2 + (2 if mixed_fp32 is not None else 0) if mixed is not None else 1)
            + (args.steps * len(mixed_batched["groups"]) if mixed_batched else 0)
            + (args.steps * 9 if adjoint else 0)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    R.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
