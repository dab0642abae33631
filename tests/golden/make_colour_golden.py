"""Generate tests/golden/colour.npz from the reference renderer itself.

The two colour options of render_image that frames.npz does not cover,
produced by the reference's own code compiled from the reference tree by
oracle/build.py (strict flavour):

* the interstellar disk palette of colorize_buffer (main.cpp:1721-1866),
  applied to the reference's own GeoPixel records of frames.npz's cases,
  with the default ColorParams and with every palette field changed;
* camera supersampling, render_image with camera_spp > 1
  (main.cpp:2232-2322): jittered full passes averaged in linear light, on
  small frames of both charts, bundles, both palettes, spp 2 (the
  horizontal pair), 3 and 5 (centre + table pairs), 4 and 17 (table pairs,
  then the golden-angle spiral).

The GPU box has no reference tree, so the images are committed as fixtures.

Usage: python tests/golden/make_colour_golden.py   (after make_golden.py)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import golden_lib as G  # noqa: E402
import oracle_lib as O  # noqa: E402
from kerrtracecpp2_b200 import abi  # noqa: E402

PALETTE_CASES = ["cfg1_ks_rk4", "cfg2_bl_dopri5", "cfg3_bundles", "cfg5_ks", "kn_charged", "offsets"]

COLOUR = {
    "interstellar": dict(palette=abi.KT_PALETTE_INTERSTELLAR),
    "interstellar_custom": dict(palette=abi.KT_PALETTE_INTERSTELLAR, disk_rings=3, disk_sectors=5,
                                disk_sigma=0.8, disk_hue_offset=0.3, exposure=1.7, gamma=2.0),
    "interstellar_one_cell": dict(palette=abi.KT_PALETTE_INTERSTELLAR, disk_rings=1, disk_sectors=1,
                                  disk_sigma=0.2, disk_hue_offset=-0.45),
}

SPP_CASES = {
    "spp2_bl": (dict(chart=abi.KT_CHART_BL, a=0.6, width=40, height=24, theta_deg=75.0, fov_deg=40.0), 2, {}),
    "spp3_ks_interstellar": (dict(chart=abi.KT_CHART_KS, a=0.8, Q=0.2, width=32, height=20, theta_deg=80.0,
                                  fov_deg=35.0), 3, dict(palette=abi.KT_PALETTE_INTERSTELLAR)),
    "spp4_bl_dopri5": (dict(chart=abi.KT_CHART_BL, integrator=abi.KT_DOPRI5, a=0.9, Q=0.3, Lambda=1e-4,
                            r_obs=60.0, theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=32, height=18),
                       4, dict(gamma=1.8, exposure=1.3)),
    "spp5_offset": (dict(chart=abi.KT_CHART_BL, a=0.5, width=24, height=16, pixel_offset_x=0.3,
                         pixel_offset_y=-0.1, fov_deg=40.0), 5, {}),
    "spp17_ks": (dict(chart=abi.KT_CHART_KS, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
                      width=24, height=24, fov_deg=40.0), 17, dict(palette=abi.KT_PALETTE_INTERSTELLAR)),
    "spp3_bundles": (dict(chart=abi.KT_CHART_BL, bundles=1, a=0.998, theta_deg=60.0, width=20, height=12),
                     3, {}),
}


def main():
    if not O.ref_available("strict"):
        sys.exit("oracle/_ref/libktref_strict.so missing: run python oracle/build.py first")
    bg = G.data()["bg"]
    arrays = {}
    meta = {"palette_cases": PALETTE_CASES, "colour": COLOUR, "spp": {}}
    for name in PALETTE_CASES:
        d = G.desc(name)
        geo = G.data()[f"{name}/geopixels"]
        r_isco = O.ref("strict").ref_r_isco(d.M, d.a, d.Q, d.Lambda)
        for cname, ckw in COLOUR.items():
            rgb = O.colorize_ref_cp(d, geo, r_isco, abi.color_params(**ckw), bg)
            arrays[f"{name}/{cname}"] = rgb
            print(f"{name:16s} {cname:22s} lit {int(rgb.any(axis=1).sum())}")
    for name, (kw, spp, ckw) in SPP_CASES.items():
        d = abi.frame_desc(**kw)
        rgb = O.render_ref(d, abi.color_params(**ckw), spp, bg)
        arrays[f"spp/{name}"] = rgb
        meta["spp"][name] = [kw, spp, ckw]
        print(f"{name:22s} {d.width}x{d.height} spp {spp}")
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    path = os.path.join(HERE, "colour.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
