"""Mixed-precision kernels on the GPU against the FP64 kernels, which are
bit-identical to the reference (so this is the error against the FP64
oracle), over whole frames of the benchmark configurations."""
import numpy as np
import pytest

from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu

FRAMES = {
    "cfg2_720p_dopri5": dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                             theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=1280, height=720),
    "cfg1_ks_rk4": dict(chart=0, a=0.5, width=320, height=180, r_obs=40.0, theta_deg=80.0,
                        fov_deg=45.0, disk_out=12.0),
    "cfg5_ks_rk4": dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=512,
                        height=512),
    "cfg2_geometry_rk4": dict(chart=1, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
                              fov_deg=30.0, disk_out=20.0, width=640, height=360),
}


def trace(renderer, d):
    import torch

    out = renderer.trace(d)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


# Stated bounds of the mixed tracer's error against the FP64 oracle
# (class-mismatch fraction; relative g error at p50, p99 and max over the
# disk pixels of both).  Configuration 2 carries the target's g bar at the
# median.  These errors are almost entirely the difference between the
# analytic Hamiltonian gradient and the reference's central differences
# (test_mixed_error_decomposition): it moves the adaptive step sequence,
# and the reference's disk crossing is the midpoint of an 8 x 8 bisection
# of the last step (geodesic.hpp:49-140), so two traces whose last steps
# differ disagree by up to 1/4096 of a step in the hit.
# Measured on B200 (class, g p50 / p99 / max): config 2 0, 8.5e-7 / 1.7e-5 /
# 7.1e-2; config 1 0, 2.3e-6 / 2.0e-5 / 8.3e-2; config 5 3.8e-6, 2.0e-6 /
# 4.3e-5 / 6.6e-2; config 2 geometry with RK4 at tol 1e-7 0, 2.1e-6 / 5.1e-5
# / 3.2e-2.  The maxima are pixels by the critical curve.
BOUNDS = {
    "cfg2_720p_dopri5": dict(cls=1e-4, p50=1e-6, p99=5e-5, mx=0.2),
    "cfg1_ks_rk4": dict(cls=1e-4, p50=5e-6, p99=5e-5, mx=0.2),
    "cfg5_ks_rk4": dict(cls=1e-4, p50=5e-6, p99=1e-4, mx=0.2),
    "cfg2_geometry_rk4": dict(cls=1e-4, p50=5e-6, p99=1e-4, mx=0.2),
}


@pytest.mark.parametrize("name", sorted(FRAMES))
def test_mixed_against_fp64(renderer, name):
    import mixed_lib as X

    kw = FRAMES[name]
    ref = trace(renderer, abi.frame_desc(**kw))
    got = trace(renderer, abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw))
    s = X.error_stats(got, ref)
    print(X.fmt(name, s))
    b = BOUNDS[name]
    assert s["class_mismatch"] < b["cls"]
    assert s["g_p50"] <= b["p50"] and s["g_p99"] <= b["p99"] and s["g_max"] <= b["mx"]
    assert s["r_p50"] < 5e-5


@pytest.mark.parametrize("name,tol", [("cfg2_720p_dopri5", 1e-10), ("cfg2_720p_dopri5", 1e-8),
                                      ("cfg1_ks_rk4", None), ("cfg5_ks_rk4", None)],
                         ids=["cfg2_tol1e-10", "cfg2_tol1e-8_fp32", "cfg1_fp32", "cfg5_fp32"])
def test_mixed_error_decomposition(renderer, name, tol):
    """The mixed frame M against the FP64 oracle F (the exact kernel,
    bit-identical to the reference) split through A, the same frame traced
    on the host with the mixed tracer's analytic FP64 gradient alone (exact
    reciprocals and sincos, no FP32, no contraction): M vs A is the mixed
    kernel's own error (FP32 right-hand side, approximate reciprocals and
    sincos, FMA contraction), A vs F the reference's finite-difference
    gradient against the analytic one.  At tol 1e-10 the FP32 right-hand
    side is off and M vs A is the rounding of the mixed path's operations
    (measured p50 9.3e-9, a hundredth of A vs F); with the FP32 right-hand
    side on (tol >= 1e-8) M vs A is of the size of A vs F (p50 2e-6)."""
    import mixed_lib as X

    kw = dict(FRAMES[name])
    if tol is not None:
        kw["tol"] = tol
    F = trace(renderer, abi.frame_desc(**kw))
    dm = abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw)
    M = trace(renderer, dm)
    A = X.trace_fp64_rhs(dm)
    import kerrtracecpp2_b200 as kt

    fp32 = kt.frame_derive(dm).r_fp32 != float("inf")
    mf, ma, af = X.error_stats(M, F), X.error_stats(M, A), X.error_stats(A, F)
    print(f"\n{name} tol {kw.get('tol', 1e-7):g} (FP32 right-hand side {'on' if fp32 else 'off'})")
    for k, v in (("M mixed vs F oracle", mf), ("M mixed vs A analytic FP64", ma),
                 ("A analytic FP64 vs F oracle", af)):
        print(X.fmt(k, v))
    assert mf["class_mismatch"] < 1e-4 and af["class_mismatch"] < 1e-4
    if not fp32:
        assert ma["g_p50"] <= 5e-8 and ma["g_p50"] < 0.05 * af["g_p50"]
        assert ma["class_mismatch"] < 1e-5
    else:
        assert ma["g_p50"] <= 2 * max(af["g_p50"], 1e-6)


def test_mixed_bundles_against_fp64(renderer):
    """Bundle mode (config 3 geometry at 1/100 of the pixels): the analytic
    Hessian-vector products against the reference's finite-difference
    Hessian; magnification compared on the disk pixels."""
    kw = dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=192, height=108)
    ref = trace(renderer, abi.frame_desc(**kw))
    got = trace(renderer, abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw))
    same = got["outcome"] == ref["outcome"]
    disk = same & (ref["outcome"] == 1)
    eg = np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk])
    em = np.abs(got["magnif"][disk] - ref["magnif"][disk]) / np.abs(ref["magnif"][disk])
    print(f"bundles: class mismatch {1 - same.mean():.2e}, g rel p50 {np.median(eg):.2e}, "
          f"magnif rel p50 {np.median(em):.2e} p99 {np.percentile(em, 99):.2e}")
    assert 1 - same.mean() < 1e-3
    assert np.median(eg) < 5e-6 and np.median(em) < 1e-4


def test_mixed_error_table_every_config(renderer):
    """The error of the mixed-precision path against the FP64 oracle for
    every benchmark configuration at its full size: pixel class, g and r_hit
    on the disk pixels of both, and the colour of the pixel (blackbody
    palette, seed-0 star field).  Config 4 is its 64 parameter sets, traced
    as one batch in each precision.  The table is printed."""
    import torch

    import kerrtracecpp2_b200 as kt

    cfgs = {
        "1 KS RK4 320x180": [FRAMES["cfg1_ks_rk4"]],
        "2 KNdS BL DOPRI5 720p": [FRAMES["cfg2_720p_dopri5"]],
        "3 bundles 1080p": [dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=1920, height=1080)],
        "4 64 sets, batch": None,
        "5 KS RK4 512x512": [FRAMES["cfg5_ks_rk4"]],
    }
    bg = torch.from_numpy(np.ascontiguousarray(kt.starfield(0, 2048, 1024))).cuda()
    rows = []
    for name, frames in cfgs.items():
        if frames is None:
            descs = kt.random_parameter_sets(64, seed=1)
            outs = []
            for prec in (abi.KT_PREC_FP64, abi.KT_PREC_MIXED):
                ds = [abi.frame_desc(**{**{f: getattr(d, f) for f, _ in abi.FrameDesc._fields_},
                                        "precision": prec}) for d in descs]
                b = renderer.batch(ds)
                b.launch()
                outs.append((ds, b.outs))
            pairs = [((outs[0][0][i], outs[0][1][i]), (outs[1][0][i], outs[1][1][i]))
                     for i in range(len(descs))]
        else:
            pairs = []
            for kw in frames:
                dp = abi.frame_desc(**kw)
                dm = abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw)
                pairs.append(((dp, renderer.trace(dp)), (dm, renderer.trace(dm))))
        n = mism = 0
        eg_all, er_all, cdiff = [], [], []
        for (dp, op), (dm, om) in pairs:
            rp = renderer.colorize(dp, op, bg=bg)
            rm = renderer.colorize(dm, om, bg=bg)
            torch.cuda.synchronize()
            ref = {k: v.cpu().numpy() for k, v in op.items() if v is not None}
            got = {k: v.cpu().numpy() for k, v in om.items() if v is not None}
            same = got["outcome"] == ref["outcome"]
            disk = same & (ref["outcome"] == 1)
            n += same.size
            mism += int((~same).sum())
            eg_all.append(np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk]))
            er_all.append(np.abs(got["r"][disk] - ref["r"][disk]) / np.abs(ref["r"][disk]))
            d = np.abs(rm.cpu().numpy().astype(int) - rp.cpu().numpy().astype(int)).reshape(-1, 3).max(axis=1)
            cdiff.append(d)
        eg, er, cd = np.concatenate(eg_all), np.concatenate(er_all), np.concatenate(cdiff)
        rows.append((name, n, mism / n, np.median(eg), np.percentile(eg, 99), np.median(er),
                     np.percentile(er, 99), (cd > 0).mean(), np.percentile(cd, 99.9), cd.max()))
    print("\nconfig | pixels | class mismatch | g p50 | g p99 | r_hit p50 | r_hit p99 | "
          "colour: pixels differing | p99.9 diff | max diff")
    for r in rows:
        print(f"{r[0]} | {r[1]} | {r[2]:.1e} | {r[3]:.1e} | {r[4]:.1e} | {r[5]:.1e} | {r[6]:.1e} | "
              f"{r[7]:.2e} | {r[8]:.0f} | {r[9]}")
    for r in rows:
        assert r[2] < 1e-3 and r[3] < 5e-6, r


def test_mixed_reciprocal_and_sincos():
    """mx_rcp (hardware seed + two Newton-Raphson steps) is within one ulp
    of the division on 4 M arguments over the whole exponent range (zero and
    infinity included), and the device sincos of the mixed path (CUDA's) is
    within 4e-16 of the renderer's libm on [-8, 8] and on arguments up to
    3e7."""
    import os
    import subprocess

    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    exe = os.path.join(here, "_build", "mx_rcp_check")
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-I", os.path.join(root, "kerrtracecpp2_b200", "csrc"), "-o", exe,
                    os.path.join(here, "mx_rcp_check.cu")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    vals = dict(zip(out[0::2], out[1::2]))
    print(vals)
    assert vals["status"] == "no"  # "no error"
    assert float(vals["max_rcp_ulp"]) <= 1.0
    assert float(vals["max_sincos_abs"]) <= 4e-16


@pytest.mark.parametrize("kw", [
    dict(chart=1, integrator=1, tol=1e-8, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
         fov_deg=30.0, disk_out=20.0, width=1280, height=720),
    dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=512, height=512),
], ids=["cfg2_dopri5_tol1e-8", "cfg5_ks"])
def test_mixed_fp32_frames_are_reproducible(renderer, kw):
    """With the FP32 right-hand side on (r_fp32 finite), the per-warp
    FP32/FP64 choice depends on which rays share a warp; the single-frame
    kernels refill a warp only when all its lanes are idle, so each warp
    traces a fixed group of 32 consecutive rays and three launches of the
    same frame give the same bits."""
    import kerrtracecpp2_b200 as kt

    d = abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw)
    assert np.isfinite(kt.frame_derive(d).r_fp32)
    runs = [trace(renderer, d) for _ in range(3)]
    for r in runs[1:]:
        for k, v in runs[0].items():
            assert np.array_equal(np.ascontiguousarray(v).view(np.uint8),
                                  np.ascontiguousarray(r[k]).view(np.uint8)), k
