"""The elliptic-closed solver on the GPU (the standard trace, then
k_elliptic): bit-identical to the reference's results in
tests/golden/elliptic.npz through kt_trace, kt_trace_pixels and a
supersampled render and batches."""
import numpy as np
import pytest

import golden_lib as G
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu
NAMES = sorted(G.ell_cases())


def to_np(out):
    import torch

    torch.cuda.synchronize()
    return {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}


@pytest.mark.parametrize("name", NAMES)
def test_trace_matches_reference(renderer, name):
    got = to_np(renderer.trace(G.ell_desc(name)))
    assert G.mismatches(got, G.ell_result(name)) == {k: 0 for k in G.FIELDS}


def test_pixel_list_matches_frame(renderer):
    import torch

    name = "ell_kerr_ks"
    d = G.ell_desc(name)
    n = d.width * d.height
    perm = np.random.default_rng(5).permutation(n).astype(np.int32)
    got = to_np(renderer.trace_pixels(d, torch.from_numpy(perm).cuda()))
    want = G.ell_result(name)
    assert G.mismatches(got, {k: v[perm] for k, v in want.items()}) == {k: 0 for k in G.FIELDS}


def test_supersampled_render_equals_colour_of_passes(renderer):
    """camera_spp 2 with the elliptic solver: each pass gets the closed form
    too, so the render equals the average of the two single-pass renders
    taken at the jitter offsets."""
    import kerrtracecpp2_b200 as kt
    import oracle_lib as O

    kw = dict(G.ell_cases()["ell_offsets"])
    bg = G.data()["bg"]
    cp = abi.color_params()
    passes = []
    for ox, oy in kt.camera_spp_offsets(2):
        d = abi.frame_desc(**dict(kw, pixel_offset_x=kw["pixel_offset_x"] + ox,
                                  pixel_offset_y=kw["pixel_offset_y"] + oy))
        passes.append(renderer.render_host(d, cp, bg).reshape(-1, 3))
    want = O.spp_combine_port(np.stack(passes), cp.gamma)
    got = renderer.render_host(abi.frame_desc(**kw), cp, bg, camera_spp=2)
    assert np.array_equal(got.reshape(-1, 3), want)


def test_elliptic_frames_in_a_batch(renderer):
    """Elliptic-closed frames share a batch with standard frames of the same
    kernels (KS RK4, BL DOPRI5): the graph runs the closed form over the
    elliptic frames only."""
    names = ["ell_kerr_ks", "ell_edge_on_dopri5", "ell_step_cap"]
    descs = [G.ell_desc(n) for n in names] + [G.desc("cfg1_ks_rk4"), G.desc("cfg2_bl_dopri5")]
    wants = [G.ell_result(n) for n in names] + [G.result("cfg1_ks_rk4"), G.result("cfg2_bl_dopri5")]
    b = renderer.batch(descs)
    for _ in range(2):
        b.launch()
        for o, want in zip(b.outs, wants):
            assert G.mismatches(to_np(o), want) == {k: 0 for k in G.FIELDS}
    b.close()


@pytest.mark.parametrize("name", [n for n in NAMES if f"{n}/reason" in G.ell()])
def test_fallback_reasons_match_reference(renderer, name):
    """kt_elliptic_reasons: the reference's --debug-elliptic tag of every pixel."""
    import torch

    got = renderer.elliptic_reasons(G.ell_desc(name))
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), G.ell()[f"{name}/reason"])


def test_fallback_reasons_zero_for_other_solvers(renderer):
    import torch

    got = renderer.elliptic_reasons(G.desc("cfg1_ks_rk4"))
    torch.cuda.synchronize()
    assert not got.cpu().numpy().any()
