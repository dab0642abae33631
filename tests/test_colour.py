"""The interstellar disk palette and camera supersampling in the oracle:
the C restatement (orc_colorize_cp, orc_spp_offsets, orc_spp_combine)
against the reference's own images in tests/golden/colour.npz, the
library's jitter table (kt_camera_spp_offsets, host code, no GPU) against
the oracle's, and -- where the reference tree is built here -- the fixtures
against a live run of the reference."""
import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
from kerrtracecpp2_b200 import abi

C = G.colour_meta()


def geo_of(name):
    """The reference's GeoPixel records as float64 SoA (what colorize_buffer reads)."""
    g = G.data()[f"{name}/geopixels"]
    return {k: np.ascontiguousarray(g[k].astype(np.uint8 if k == "outcome" else np.float64))
            for k in G.FIELDS}


@pytest.mark.parametrize("cname", sorted(C["colour"]))
@pytest.mark.parametrize("name", C["palette_cases"])
def test_port_interstellar_matches_reference(name, cname):
    cp = abi.color_params(**C["colour"][cname])
    rgb = O.colorize_port_cp(G.desc(name), geo_of(name), cp, G.data()["bg"])
    want = G.colour()[f"{name}/{cname}"]
    assert np.array_equal(rgb, want)
    assert want.any(axis=1).sum() > 0


def test_port_blackbody_cp_equals_plain_colour():
    """orc_colorize_cp with the blackbody palette is orc_colorize."""
    name = "cfg1_ks_rk4"
    d, geo, bg = G.desc(name), G.result(name), G.data()["bg"]
    a = O.colorize_port_cp(d, geo, abi.color_params(exposure=1.3, gamma=2.0, temp_scale=0.9), bg)
    b = O.colorize_port(d, geo, bg, exposure=1.3, gamma=2.0, temp_scale=0.9)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("spp", [0, 1, 2, 3, 4, 5, 6, 14, 15, 16, 17, 18, 33, 256])
def test_library_offsets_equal_port(spp):
    import kerrtracecpp2_b200 as kt

    got = kt.camera_spp_offsets(spp)
    want = O.spp_offsets_port(spp)
    assert got.shape == (max(spp, 1), 2)
    assert np.array_equal(G.bits(got), G.bits(want))
    # +/- pairs (the centre first for odd counts above 2)
    if spp > 2:
        k = spp % 2
        assert np.array_equal(got[k + 1::2][: (spp - k) // 2], -got[k::2][: (spp - k) // 2])
        assert np.all(np.hypot(got[:, 0], got[:, 1]) < 0.5)


def test_library_offsets_reject_too_many():
    import ctypes

    import kerrtracecpp2_b200 as kt

    L = kt.load_library()
    xy = np.zeros(2 * (abi.KT_MAX_CAMERA_SPP + 1))
    assert L.kt_camera_spp_offsets(abi.KT_MAX_CAMERA_SPP + 1, xy.ctypes.data_as(ctypes.c_void_p)) \
        == abi.KT_ERR_INVALID_ARGUMENT


def port_render(kw, spp, ckw, bg):
    cp = abi.color_params(**ckw)
    passes = []
    for ox, oy in O.spp_offsets_port(spp):
        d = abi.frame_desc(**dict(kw, pixel_offset_x=kw.get("pixel_offset_x", 0.0) + ox,
                                  pixel_offset_y=kw.get("pixel_offset_y", 0.0) + oy))
        passes.append(O.colorize_port_cp(d, O.trace_port(d), cp, bg))
    return O.spp_combine_port(np.stack(passes), cp.gamma)


@pytest.mark.parametrize("name", sorted(C["spp"]))
def test_port_supersampling_matches_reference(name):
    kw, spp, ckw = C["spp"][name]
    got = port_render(kw, spp, ckw, G.data()["bg"])
    assert np.array_equal(got, G.colour()[f"spp/{name}"])


def test_spp_combine_edges():
    """One pass returns its own image for any gamma (pow round trip at the
    256 channel values); identical passes average to themselves; black and
    white average to the display value of linear 1/2."""
    v = np.arange(256, dtype=np.uint8)
    img = np.stack([v, v[::-1], v], axis=1)
    for gamma in (2.2, 1.0, 1.8):
        assert np.array_equal(O.spp_combine_port(img[None], gamma), img)
        assert np.array_equal(O.spp_combine_port(np.stack([img] * 5), gamma), img)
    bw = np.stack([np.zeros((1, 3), np.uint8), np.full((1, 3), 255, np.uint8)])
    want = int(np.floor(255 * 0.5 ** (1 / 2.2) + 0.5))
    assert np.all(O.spp_combine_port(bw, 2.2) == want)


needs_ref = pytest.mark.skipif(not O.ref_available("strict"), reason="reference tree not built here")


@needs_ref
def test_fixtures_equal_live_reference():
    bg = G.data()["bg"]
    name = "cfg5_ks"
    d = G.desc(name)
    r_isco = O.ref("strict").ref_r_isco(d.M, d.a, d.Q, d.Lambda)
    cp = abi.color_params(**C["colour"]["interstellar_custom"])
    assert np.array_equal(O.colorize_ref_cp(d, G.data()[f"{name}/geopixels"], r_isco, cp, bg),
                          G.colour()[f"{name}/interstellar_custom"])
    kw, spp, ckw = C["spp"]["spp3_ks_interstellar"]
    assert np.array_equal(O.render_ref(abi.frame_desc(**kw), abi.color_params(**ckw), spp, bg),
                          G.colour()["spp/spp3_ks_interstellar"])
