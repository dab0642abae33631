"""The drop-in boundary end to end on the GPU:

  * the CLI (kerrtracecpp2_b200/bin/kerr_tracer) with the reference's flags:
    --geo-only writes the reference's .kgeo file (main.cpp:96-137,
    2897-2914) byte for byte, --color-only colours it as the reference's
    colorize_buffer does (main.cpp:1817-1866, 2722-2752);
  * the reference's spin-orientation regression (its
    tests/spin_orientation_regression.cpp:86-176) run against this CLI;
  * the reference's own main.cpp built with -DUSE_CUDA and linked against
    libkerrtrace.so (oracle/build.py), whose render dispatch
    (main.cpp:2413-2443) calls cuda_render from this library.
"""
import os
import subprocess

import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
from boundary_lib import kgeo_records, orientation, write_ppm
from kerrtracecpp2_b200 import abi
from png_read import read_png

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "kerrtracecpp2_b200", "bin", "kerr_tracer")
REF_CUDA_MAIN = os.path.join(ROOT, "oracle", "_ref", "kerr_tracer_ref_cuda")

# config 1's flags (the reference's spin test frame)
CFG1_FLAGS = ["--ks", "--a", "0.5", "--theta", "80", "--phi", "0", "--r-obs", "40", "--fov", "45",
              "--disk-out", "12", "--solver-mode", "standard"]


def run(cmd, cwd):
    p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def test_cli_geo_only_then_color_only(tmp_path):
    """The golden configuration-1 frame (64x36): --geo-only writes the
    reference's own GeoPixel records byte for byte, with the reference's
    header; --color-only on that file, with the golden star field as
    background, writes the reference's colorize_buffer image."""
    name = "cfg1_ks_rk4"
    d = G.desc(name)
    geo = str(tmp_path / "f.kgeo")
    run([CLI, "--geo-only", "--geo-file", geo, "--custom-res", str(d.width), str(d.height),
         "--out-dir", str(tmp_path)] + CFG1_FLAGS, tmp_path)
    W, H, meta, recs = kgeo_records(geo)
    assert (W, H) == (d.width, d.height)
    assert recs.tobytes() == G.data()[f"{name}/geopixels"].tobytes()
    r_isco = O.derive_port(d).r_isco
    assert list(meta) == [d.M, d.a, d.Q, d.Lambda, r_isco, r_isco, d.disk_out, d.theta_deg,
                          d.phi_deg, d.r_obs]
    bg = str(tmp_path / "bg.ppm")
    write_ppm(bg, G.data()["bg"])
    png = str(tmp_path / "recolor.png")
    run([CLI, "--color-only", geo, "--bg", bg, "--output", png], tmp_path)
    img = read_png(png)
    assert img.shape == (d.height, d.width, 3)
    assert np.array_equal(img.reshape(-1, 3), G.data()[f"{name}/rgb"])


def test_cli_geo_only_config1_full(tmp_path):
    """Configuration 1 at its full 320x180: the .kgeo records equal the
    oracle's per-pixel results stored as the reference stores them (float32
    GeoPixel fields)."""
    d = abi.frame_desc(chart=abi.KT_CHART_KS, a=0.5, width=320, height=180, r_obs=40.0,
                       theta_deg=80.0, fov_deg=45.0, disk_out=12.0)
    geo = str(tmp_path / "c1.kgeo")
    run([CLI, "--geo-only", "--geo-file", geo, "--custom-res", "320", "180",
         "--out-dir", str(tmp_path)] + CFG1_FLAGS, tmp_path)
    _, _, _, recs = kgeo_records(geo)
    want = O.to_geopixels(O.trace_port(d))
    assert recs.tobytes() == want.tobytes()


@pytest.mark.parametrize("spin,bright_right,gap_right", [(0.5, False, False), (-0.5, True, True)])
def test_spin_orientation_regression(tmp_path, spin, bright_right, gap_right):
    """The reference's regression (spin_orientation_regression.cpp:216-226):
    at a = +0.5 the Doppler-bright side of the disk and the wider gap above
    the shadow are on the left, at a = -0.5 on the right."""
    geo = str(tmp_path / "spin.kgeo")
    flags = [f if f != "0.5" else str(spin) for f in CFG1_FLAGS]
    run([CLI, "--geo-only", "--geo-file", geo, "--custom-res", "320", "180",
         "--intersection-hermite", "--out-dir", str(tmp_path)] + flags, tmp_path)
    W, H, meta, recs = kgeo_records(geo)
    assert meta[1] == spin
    assert orientation(recs, W, H) == (bright_right, gap_right)


@pytest.mark.skipif(not os.path.exists(REF_CUDA_MAIN),
                    reason="the reference's main.cpp was not built against the library "
                           "(oracle/build.py needs the reference tree)")
@pytest.mark.parametrize("chart_flag", ["--ks", "--bl"])
def test_reference_main_renders_through_cuda_render(renderer, tmp_path, chart_flag):
    """The reference's main.cpp (-DUSE_CUDA) linked against libkerrtrace.so:
    its CUDA dispatch calls this library's cuda_render and unpacks the RGBA
    words (main.cpp:2437-2443) into the PNG it writes; that image equals
    kt_render_host of the same frame (black background, default colour
    parameters), i.e. the reference CPU algorithm's image."""
    flags = [chart_flag] + [f for f in CFG1_FLAGS if f not in ("--ks",)]
    run([REF_CUDA_MAIN, "--custom-res", "64", "36", "--bg", "none"] + flags, tmp_path)
    pngs = [f for f in os.listdir(tmp_path) if f.endswith(".png")]
    assert len(pngs) == 1, pngs
    img = read_png(str(tmp_path / pngs[0]))
    d = abi.frame_desc(chart=abi.KT_CHART_KS if chart_flag == "--ks" else abi.KT_CHART_BL, a=0.5,
                       width=64, height=36, r_obs=40.0, theta_deg=80.0, fov_deg=45.0, disk_out=12.0)
    want = renderer.render_host(d)
    assert img.shape == want.shape
    assert np.array_equal(img, want)
    assert (want.reshape(-1, 3).max(axis=1) > 0).mean() > 0.05  # the disk is in the picture
