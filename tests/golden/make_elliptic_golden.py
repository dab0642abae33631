"""Generate tests/golden/elliptic.npz from the reference renderer itself.

The elliptic-closed solver (--elliptic-closed / --solver-mode elliptic): the
reference's trace_single_elliptic_closed (main.cpp:1227-1295) reached through
the dispatch of trace_geodesics (select_solver_mode, main.cpp:235-276),
compiled from the reference tree by oracle/build.py (strict flavour: the
renderer's libm, complex arithmetic by the textbook formulas).  Kerr frames
in both charts and with both integrators (a ray the closed form does not
place on the disk, or that the standard tracer ends at the horizon, is the
standard tracer's), edge cases of the camera, and the frames that
select_solver_mode hands to the standard tracers (charge, Lambda, bundles).

Stored per case: the frame descriptor, the float64 per-pixel results
(ref_trace_pixels), the reference's GeoPixel records (trace_geodesics) and
its fallback reason per pixel (EllipticFallbackReason, 0 where the closed
form was taken or checked against the horizon).

Usage: python tests/golden/make_elliptic_golden.py
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

ELL = dict(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED)
BL, KS = abi.KT_CHART_BL, abi.KT_CHART_KS

CASES = {
    "ell_kerr_bl": dict(ELL, chart=BL, a=0.5, width=48, height=27, fov_deg=40.0),
    "ell_kerr_ks": dict(ELL, chart=KS, a=0.5, width=48, height=27, fov_deg=45.0),
    "ell_fast_spin_bl": dict(ELL, chart=BL, a=0.998, theta_deg=60.0, width=40, height=24),
    "ell_fast_spin_ks": dict(ELL, chart=KS, a=0.998, theta_deg=60.0, width=40, height=24),
    "ell_edge_on_dopri5": dict(ELL, chart=BL, integrator=abi.KT_DOPRI5, tol=1e-10, a=0.9,
                               theta_deg=85.0, r_obs=60.0, fov_deg=30.0, disk_out=20.0, width=40,
                               height=24),
    "ell_edge_on_ks": dict(ELL, chart=KS, a=0.9, theta_deg=85.0, r_obs=60.0, fov_deg=30.0,
                           disk_out=20.0, width=40, height=24),
    "ell_retrograde": dict(ELL, chart=BL, integrator=abi.KT_DOPRI5, a=-0.7, width=30, height=20,
                           fov_deg=40.0),
    "ell_polar_camera": dict(ELL, chart=KS, a=0.6, theta_deg=5.0, width=30, height=20, fov_deg=60.0),
    "ell_equatorial_camera": dict(ELL, chart=BL, a=0.9, theta_deg=90.0, width=30, height=20,
                                  fov_deg=40.0),
    "ell_close_camera": dict(ELL, chart=KS, a=0.95, r_obs=8.0, theta_deg=70.0, fov_deg=90.0,
                             width=24, height=14),
    "ell_schwarzschild": dict(ELL, chart=BL, a=0.0, width=20, height=12, fov_deg=40.0),
    "ell_offsets": dict(ELL, chart=BL, a=0.6, width=20, height=12, pixel_offset_x=0.35,
                        pixel_offset_y=-0.2, fov_deg=40.0),
    "ell_step_cap": dict(ELL, chart=BL, a=0.9, width=16, height=9, max_steps=7),
    # select_solver_mode hands these to the standard tracers
    "ell_charged": dict(ELL, chart=BL, a=0.5, Q=0.3, width=20, height=12, fov_deg=40.0),
    "ell_lambda": dict(ELL, chart=KS, a=0.5, Lambda=1e-4, width=20, height=12, fov_deg=40.0),
    "ell_bundles": dict(ELL, chart=BL, bundles=1, a=0.9, width=12, height=7, max_steps=3000),
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
        solver = d.solver_mode if not (d.bundles or abs(d.Q) > 1e-15 or abs(d.Lambda) > 1e-15) else 0
        if solver == abi.KT_SOLVER_ELLIPTIC_CLOSED:
            arrays[f"{name}/reason"] = O.elliptic_reasons_ref(d, "strict")
        meta[name] = kw
        print(f"{name:24s} {d.width}x{d.height} outcomes {np.bincount(out['outcome'], minlength=3)} "
              f"{time.time() - t0:.1f}s", flush=True)
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    path = os.path.join(HERE, "elliptic.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
