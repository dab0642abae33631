"""Host-side checks of the boundary tests' pieces (no GPU): the reference's
main.cpp built with -DUSE_CUDA resolves cuda_render from libkerrtrace.so,
the PNG reader decodes what the CLI's encoder writes, and the
spin-orientation analysis gives the reference's expected answers on the
oracle's frames."""
import os
import subprocess
import zlib

import numpy as np
import pytest

import oracle_lib as O
from boundary_lib import orientation
from kerrtracecpp2_b200 import abi
from png_read import read_png

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CUDA_MAIN = os.path.join(ROOT, "oracle", "_ref", "kerr_tracer_ref_cuda")
LIB = os.path.join(ROOT, "kerrtracecpp2_b200", "libkerrtrace.so")
MANGLED = "_Z11cuda_renderRK15KNdSParams_CUDARK17CameraParams_CUDAb"


@pytest.mark.skipif(not os.path.exists(REF_CUDA_MAIN),
                    reason="the reference's main.cpp was not built (needs the reference tree)")
def test_reference_main_links_against_library():
    """The reference's renderer built with -DUSE_CUDA takes cuda_render from
    this library: its only undefined CUDA-side symbol is cuda_render, the
    library defines it, and the dynamic loader resolves libkerrtrace.so to
    the in-tree build (the loader only, nothing runs)."""
    und = subprocess.run(["nm", "-D", "--undefined-only", REF_CUDA_MAIN], capture_output=True,
                         text=True, check=True).stdout
    assert MANGLED in und
    assert "cuda" not in und.replace(MANGLED, "").lower()
    defined = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True,
                             check=True).stdout
    assert MANGLED in defined
    env = dict(os.environ, LD_TRACE_LOADED_OBJECTS="1")
    out = subprocess.run([REF_CUDA_MAIN], env=env, capture_output=True, text=True, check=True).stdout
    line = [l for l in out.splitlines() if "libkerrtrace.so" in l]
    assert line and os.path.realpath(line[0].split("=>")[1].split("(")[0].strip()) == os.path.realpath(LIB)


def _stored_png(img):
    """A PNG as the CLI writes it: unfiltered rows in stored deflate blocks."""
    import struct

    H, W, _ = img.shape
    raw = b"".join(b"\0" + img[y].tobytes() for y in range(H))

    def chunk(t, b):
        return struct.pack(">I", len(b)) + t + b + struct.pack(">I", zlib.crc32(t + b))

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, 2, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw, 0)) + chunk(b"IEND", b""))


def test_png_reader(tmp_path):
    rng = np.random.default_rng(3)
    img = rng.integers(0, 256, size=(7, 5, 3), dtype=np.uint8)
    p = tmp_path / "a.png"
    p.write_bytes(_stored_png(img))
    assert np.array_equal(read_png(str(p)), img)


@pytest.mark.parametrize("spin,expect", [(0.5, (False, False)), (-0.5, (True, True))])
def test_spin_orientation_on_oracle(spin, expect):
    """The reference's spin regression (spin_orientation_regression.cpp:
    216-226) holds on the oracle's configuration-1 frames at a = +-0.5, so
    the same analysis on the CLI's .kgeo files (tests/test_gpu_cli.py) tests
    the renderer, not the analysis."""
    d = abi.frame_desc(chart=abi.KT_CHART_KS, a=spin, width=320, height=180, r_obs=40.0,
                       theta_deg=80.0, fov_deg=45.0, disk_out=12.0)
    recs = O.to_geopixels(O.trace_port(d))
    assert orientation(recs, 320, 180) == expect
