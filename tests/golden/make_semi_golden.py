"""Generate tests/golden/semi.npz from the reference renderer itself.

The semi-analytic solver (--semi-analytic / --solver-mode semi): the
reference's trace_single_separable_kerr (main.cpp:578-703) reached through
the dispatch of trace_geodesics (select_solver_mode, main.cpp:235-276),
compiled from the reference tree by oracle/build.py (strict flavour).  Small
Kerr frames in the BL chart, most with a reduced step cap: in this solver a
ray whose radial potential reaches zero stops moving in r (dr is
sqrt(max(R, 0)) and the branch sign flips only on a sampled crossing of
R = 1e-9), so every ray with a radial turning point runs to the step cap.
Two cases keep the default cap of 500000 steps.  Also the frames the solver
hands to the standard tracers (KS chart, charge, Lambda, bundles).

Stored per case: the frame descriptor, the float64 per-pixel results
(ref_trace_pixels) and the reference's GeoPixel records (trace_geodesics).

Usage: python tests/golden/make_semi_golden.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle_lib as O  # noqa: E402
from kerrtracecpp2_b200 import abi  # noqa: E402

SEMI = dict(chart=abi.KT_CHART_BL, solver_mode=abi.KT_SOLVER_SEMI_ANALYTIC)

CASES = {
    "semi_kerr": dict(SEMI, a=0.5, width=32, height=18, fov_deg=40.0, max_steps=4000),
    "semi_default_cap": dict(SEMI, a=0.9, width=8, height=5, fov_deg=40.0),
    # tol 1e-10 at the default cap: phi of a parked ray grows until the
    # step-doubling error of its rounding reaches tol; the controller then
    # shrinks and regrows the step
    "semi_tight_default_cap": dict(SEMI, a=0.9, tol=1e-10, width=8, height=5, fov_deg=40.0),
    "semi_fast_spin": dict(SEMI, a=0.998, theta_deg=60.0, width=24, height=14, max_steps=3000),
    "semi_tight_tol": dict(SEMI, a=0.9, theta_deg=85.0, r_obs=60.0, fov_deg=30.0, disk_out=20.0,
                           tol=1e-10, width=24, height=14, max_steps=3000),
    "semi_dopri5_request": dict(SEMI, integrator=abi.KT_DOPRI5, a=0.7, width=20, height=12,
                                fov_deg=40.0, max_steps=3000),
    "semi_polar_camera": dict(SEMI, a=0.6, theta_deg=5.0, width=20, height=12, fov_deg=60.0,
                              max_steps=3000),
    "semi_equatorial_camera": dict(SEMI, a=0.9, theta_deg=90.0, width=20, height=12, fov_deg=40.0,
                                   max_steps=3000),
    "semi_retrograde": dict(SEMI, a=-0.8, width=20, height=12, fov_deg=40.0, max_steps=3000),
    "semi_schwarzschild": dict(SEMI, a=0.0, width=20, height=12, fov_deg=40.0, max_steps=3000),
    "semi_offsets": dict(SEMI, a=0.6, width=20, height=12, pixel_offset_x=0.35, pixel_offset_y=-0.2,
                         fov_deg=40.0, max_steps=3000),
    "semi_coarse": dict(SEMI, a=0.9, tol=1e-4, step_init=5.0, width=24, height=14, max_steps=3000),
    "semi_step_cap": dict(SEMI, a=0.9, width=16, height=9, max_steps=7),
    "semi_close_camera": dict(SEMI, a=0.95, r_obs=8.0, theta_deg=70.0, fov_deg=90.0, width=24,
                              height=14, max_steps=3000),
    # select_solver_mode hands these to the standard tracers
    "semi_ks_request": dict(SEMI, chart=abi.KT_CHART_KS, a=0.5, width=20, height=12, fov_deg=40.0),
    "semi_charged": dict(SEMI, a=0.5, Q=0.3, width=20, height=12, fov_deg=40.0),
    "semi_lambda": dict(SEMI, a=0.5, Lambda=1e-4, width=20, height=12, fov_deg=40.0),
    "semi_bundles": dict(SEMI, bundles=1, a=0.9, width=12, height=7, max_steps=3000),
}

FIELDS = ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")


def main():
    if not O.ref_available("strict"):
        sys.exit("oracle/_ref/libktref_strict.so missing: run python oracle/build.py first")
    arrays = {}
    meta = {}
    for name, kw in CASES.items():
        d = abi.frame_desc(**kw)
        t0 = time.time()
        out = O.trace_ref(d, "strict")
        geo = O.trace_geodesics_ref(d, "strict")
        for k in FIELDS:
            arrays[f"{name}/{k}"] = out[k]
        arrays[f"{name}/geopixels"] = geo
        meta[name] = kw
        print(f"{name:24s} {d.width}x{d.height} outcomes {np.bincount(out['outcome'], minlength=3)} "
              f"{time.time() - t0:.1f}s", flush=True)
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    path = os.path.join(HERE, "semi.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
