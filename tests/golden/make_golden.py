"""Generate tests/golden/frames.npz from the reference renderer itself.

Runs the reference's own tracers and colour pass, compiled from the
reference tree by oracle/build.py (strict flavour: the renderer's libm bound
in, no FMA contraction), on small frames of every path: the reference's
configurations shrunk to a few thousand pixels, plus edge cases (1x1, 7x3,
pixel offsets, Schwarzschild, retrograde spin, equatorial camera, step cap,
KS+Lambda fallback, KS+DOPRI5 request).  The GPU box has no reference tree,
so the outputs are committed as fixtures.

Stored per case: the frame descriptor, the float64 per-pixel results
(ref_trace_pixels), the reference's own GeoPixel records from
trace_geodesics (float32), and the RGB image from colorize_buffer with the
seed-0 procedural star field as background.  Also the reference's values for
the known-answer checks of its tests/core_tests.cpp.

Usage: python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle_lib as O  # noqa: E402
from kerrtracecpp2_b200 import abi, starfield  # noqa: E402

BG_W, BG_H = 512, 256

CASES = {
    "cfg1_ks_rk4": dict(chart=abi.KT_CHART_KS, a=0.5, width=64, height=36, r_obs=40.0,
                        theta_deg=80.0, phi_deg=0.0, fov_deg=45.0, disk_out=12.0),
    "cfg2_bl_dopri5": dict(chart=abi.KT_CHART_BL, integrator=abi.KT_DOPRI5, tol=1e-10, a=0.9, Q=0.3,
                           Lambda=1e-4, r_obs=60.0, theta_deg=85.0, fov_deg=30.0, disk_out=20.0,
                           width=48, height=27),
    "cfg2_bl_rk4": dict(chart=abi.KT_CHART_BL, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                        theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=48, height=27),
    "cfg3_bundles": dict(chart=abi.KT_CHART_BL, bundles=1, a=0.998, theta_deg=60.0, width=32,
                         height=18),
    "cfg5_ks": dict(chart=abi.KT_CHART_KS, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0,
                    disk_out=15.0, width=48, height=48),
    "ks_dopri5_request": dict(chart=abi.KT_CHART_KS, integrator=abi.KT_DOPRI5, a=0.6, width=24,
                              height=14, fov_deg=40.0),
    "ks_lambda_fallback": dict(chart=abi.KT_CHART_KS, a=0.5, Lambda=2e-4, width=24, height=14),
    # bundles near the equatorial plane: rays that plunge within 0.35 rad of
    # the equator skip the horizon test (ray_bundle.hpp:352-356) and run to
    # the step cap, kept small here
    "bundles_ks_request": dict(chart=abi.KT_CHART_KS, bundles=1, a=0.7, width=16, height=9,
                               fov_deg=40.0, max_steps=3000),
    "one_pixel": dict(chart=abi.KT_CHART_BL, a=0.9, width=1, height=1),
    "seven_by_three": dict(chart=abi.KT_CHART_KS, a=0.3, width=7, height=3, fov_deg=50.0),
    "offsets": dict(chart=abi.KT_CHART_BL, a=0.6, width=20, height=12, pixel_offset_x=0.35,
                    pixel_offset_y=-0.2, fov_deg=40.0),
    "schwarzschild": dict(chart=abi.KT_CHART_BL, a=0.0, width=20, height=12, fov_deg=40.0),
    "retrograde": dict(chart=abi.KT_CHART_KS, a=-0.8, width=20, height=12, fov_deg=40.0),
    "equatorial_camera": dict(chart=abi.KT_CHART_BL, integrator=abi.KT_DOPRI5, a=0.9,
                              theta_deg=90.0, width=20, height=12, fov_deg=40.0),
    "step_cap": dict(chart=abi.KT_CHART_BL, a=0.9, width=16, height=9, max_steps=7),
    "ks_step_cap": dict(chart=abi.KT_CHART_KS, a=0.9, width=16, height=9, max_steps=5),
    "bundle_step_cap": dict(chart=abi.KT_CHART_BL, bundles=1, a=0.9, width=12, height=7, max_steps=6),
    "kn_charged": dict(chart=abi.KT_CHART_KS, a=0.4, Q=0.5, width=24, height=14, fov_deg=35.0),
    "ads_lambda": dict(chart=abi.KT_CHART_BL, a=0.5, Lambda=-1e-4, width=20, height=12),
    "coarse_tol": dict(chart=abi.KT_CHART_BL, a=0.9, tol=1e-4, step_init=5.0, width=24, height=14),
}

FIELDS = ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")


def main():
    if not O.ref_available("strict"):
        sys.exit("oracle/_ref/libktref_strict.so missing: run python oracle/build.py first")
    bg = starfield(0, BG_W, BG_H)
    arrays = {"bg": bg}
    meta = {}
    for name, kw in CASES.items():
        d = abi.frame_desc(**kw)
        out = O.trace_ref(d, "strict")
        geo = O.trace_geodesics_ref(d, "strict")
        r_isco = O.ref("strict").ref_r_isco(d.M, d.a, d.Q, d.Lambda)
        rgb = O.colorize_ref(d, geo, r_isco, bg=bg, flavour="strict")
        for k in FIELDS:
            arrays[f"{name}/{k}"] = out[k]
        arrays[f"{name}/geopixels"] = geo
        arrays[f"{name}/rgb"] = rgb
        meta[name] = kw
        print(f"{name:20s} {d.width}x{d.height} outcomes {np.bincount(out['outcome'], minlength=3)}")
    # Known-answer values (tests/core_tests.cpp:18-96 of the reference).
    R = O.ref("strict")
    cov = np.zeros(16)
    con = np.zeros(16)
    R.ref_covariant_BL(1.0, 0.5, 0.1, 1e-4, 10.0, 1.2, cov.ctypes.data_as(O._P))
    R.ref_contravariant_BL(1.0, 0.5, 0.1, 1e-4, 10.0, 1.2, con.ctypes.data_as(O._P))
    arrays["kat/cov_bl"] = cov
    arrays["kat/con_bl"] = con
    s7 = np.zeros(7)
    R.ref_angle_ray(1.0, -0.5, 0.0, 0.0, 40.0, 80.0, 15.0, 45.0, 640, 360, 0.0, 0.0,
                    s7.ctypes.data_as(O._P))
    arrays["kat/camera_ray"] = s7.copy()
    for dop in (0, 1):
        s = np.zeros(7)
        R.ref_angle_ray(1.0, -0.5, 0.0, 0.0, 40.0, 80.0, 0.0, 45.0, 640, 360, 0.03, -0.02,
                        s.ctypes.data_as(O._P))
        h = np.array([1.0])
        fsal = np.full(4, np.nan)
        acc = 0
        for _ in range(32):
            acc = R.ref_adaptive_step(1.0, -0.5, 0.0, 0.0, s.ctypes.data_as(O._P),
                                      h.ctypes.data_as(O._P), dop, fsal.ctypes.data_as(O._P), 1e-7)
            if acc:
                break
        arrays[f"kat/step_{'dopri5' if dop else 'rk4'}"] = np.concatenate([s, h])
    arrays["kat/omega"] = np.array([R.ref_keplerian_omega(1.0, 0.5, 0.0, 0.0, 8.0),
                                    R.ref_keplerian_omega(1.0, -0.5, 0.0, 0.0, 8.0)])
    xyz = np.zeros(3)
    R.ref_bl_to_ks(8.0, 1.2, 2.1, 0.5, xyz.ctypes.data_as(O._P))
    arrays["kat/ks_xyz"] = xyz
    arrays["kat/ks_r"] = np.array([R.ref_r_ks(xyz[0], xyz[1], xyz[2], 0.5)])
    radii = []
    for (M, a, Q, L) in [(1, 0.5, 0, 0), (1, 0.9, 0.3, 1e-4), (1, 0.998, 0, 0), (1, 0.7, 0.1, 0),
                         (1, -0.8, 0, 0), (1, 0.0, 0, 0), (1, 0.5, 0, -1e-4), (1, 0.5, 0, 2e-4)]:
        radii.append([M, a, Q, L, R.ref_r_horizon(M, a, Q, L), R.ref_r_isco(M, a, Q, L)])
    arrays["kat/radii"] = np.array(radii)
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "frames.npz"), **arrays)
    print("wrote", os.path.join(HERE, "frames.npz"), os.path.getsize(os.path.join(HERE, "frames.npz")), "bytes")


if __name__ == "__main__":
    main()
