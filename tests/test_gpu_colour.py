"""The interstellar disk palette and camera supersampling on the GPU
(k_colorize with palette 1, kt_render_spp_host): bit-identical to the
reference's images in tests/golden/colour.npz."""
import numpy as np
import pytest

import golden_lib as G
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu
C = G.colour_meta()


@pytest.mark.parametrize("cname", sorted(C["colour"]))
@pytest.mark.parametrize("name", C["palette_cases"])
def test_colorize_interstellar_from_reference_records(renderer, name, cname):
    """kt_colorize on the reference's own GeoPixel records (float32 values)."""
    import torch

    g = G.data()[f"{name}/geopixels"]
    geo = {k: torch.from_numpy(np.ascontiguousarray(g[k].astype(np.uint8 if k == "outcome" else np.float64))).cuda()
           for k in G.FIELDS}
    bg = torch.from_numpy(np.ascontiguousarray(G.data()["bg"])).cuda()
    rgb = renderer.colorize(G.desc(name), geo, abi.color_params(**C["colour"][cname]), bg)
    torch.cuda.synchronize()
    assert np.array_equal(rgb.cpu().numpy().reshape(-1, 3), G.colour()[f"{name}/{cname}"])


@pytest.mark.parametrize("name", ["cfg1_ks_rk4", "cfg2_bl_dopri5", "cfg3_bundles", "cfg5_ks"])
def test_render_interstellar(renderer, name):
    """Trace + colour on the device equals the reference's render."""
    cp = abi.color_params(**C["colour"]["interstellar_custom"])
    rgb = renderer.render_host(G.desc(name), cp, G.data()["bg"])
    assert np.array_equal(rgb.reshape(-1, 3), G.colour()[f"{name}/interstellar_custom"])


@pytest.mark.parametrize("name", sorted(C["spp"]))
def test_render_supersampled(renderer, name):
    kw, spp, ckw = C["spp"][name]
    rgb = renderer.render_host(abi.frame_desc(**kw), abi.color_params(**ckw), G.data()["bg"], spp)
    assert np.array_equal(rgb.reshape(-1, 3), G.colour()[f"spp/{name}"])


def test_render_image_mirror_spp(renderer):
    """The module-level render_image mirror with camera_spp, and spp 1 equal
    to the plain render."""
    import kerrtracecpp2_b200 as kt

    kw, spp, ckw = C["spp"]["spp2_bl"]
    fp = kt.FrameParams(a=kw["a"], theta=kw["theta_deg"], fov=kw["fov_deg"])
    got = kt.render_image(kw["width"], kw["height"], fp, bg=G.data()["bg"], chart=kw["chart"],
                          camera_spp=spp)
    assert np.array_equal(got.reshape(-1, 3), G.colour()["spp/spp2_bl"])
    d = abi.frame_desc(**kw)
    assert np.array_equal(renderer.render_host(d, bg=G.data()["bg"], camera_spp=1),
                          renderer.render_host(d, bg=G.data()["bg"]))


def test_spp_rejects_too_many(renderer):
    d = abi.frame_desc(width=8, height=8)
    with pytest.raises(Exception):
        renderer.render_host(d, camera_spp=abi.KT_MAX_CAMERA_SPP + 1)
