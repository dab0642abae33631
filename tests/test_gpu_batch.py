"""Batches on the GPU: many frames of different sizes and kernels in one
CUDA graph launch (kt_batch_*).  Exact frames must be bit-identical to the
reference fixtures and to kt_trace of each frame, for every launch variant
and regroup threshold and after autotuning; mixed-precision frames keep the
mixed tolerance against FP64."""
import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu


def to_np(out):
    import torch

    torch.cuda.synchronize()
    got = {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}
    got["steps"] = got["steps"].view(np.uint32)
    got["attempts"] = got["attempts"].view(np.uint32)
    return got


def golden_batch():
    names = sorted(G.cases())
    return names, [G.desc(n) for n in names]


def single(renderer, d):
    return to_np(renderer.trace(d))


def assert_same(got, want):
    assert G.mismatches(got, want) == {k: 0 for k in G.FIELDS}
    for k in ("steps", "attempts"):
        assert np.array_equal(got[k], want[k]), k


def test_golden_frames_in_one_batch(renderer):
    """All 20 reference fixtures (KS, BL, DOPRI5, bundles, chart fallbacks,
    step caps, a 1x1 and a 7x3 frame) as one batch: each frame bit-identical
    to the reference renderer's output."""
    names, descs = golden_batch()
    b = renderer.batch(descs)
    kernels = {g["kernel_name"] for g in b.groups()}
    assert {"ks_rk4", "bl_rk4", "bl_dopri5", "bundles"} <= kernels
    assert b.n_rays == sum(d.width * d.height for d in descs)
    b.launch()
    for name, out in zip(names, b.outs):
        got = to_np(out)
        assert G.mismatches(got, G.result(name)) == {k: 0 for k in G.FIELDS}, name
    b.close()


@pytest.mark.parametrize("variant", range(abi.KT_BATCH_VARIANTS))
@pytest.mark.parametrize("refill_min", [1, 8, 24])
def test_variants_match_single_frame(renderer, variant, refill_min):
    descs = [
        abi.frame_desc(chart=0, a=0.5, width=160, height=90, fov_deg=45.0),
        abi.frame_desc(chart=0, a=0.3, Q=0.2, Lambda=1e-4, width=72, height=40, theta_deg=30.0),
        abi.frame_desc(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                       theta_deg=85.0, disk_out=20.0, width=96, height=54),
        abi.frame_desc(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
                       width=33, height=65),
        abi.frame_desc(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=40, height=24),
    ]
    b = renderer.batch(descs, options=abi.batch_options(variant=variant, refill_min=refill_min))
    for g in b.groups():
        # variant 3 (two lanes per ray) exists for the FP64 bundle kernel
        # only; other groups given it run their default variant
        paired = g["kernel_name"] == "bundles"
        want_v = variant if variant != 3 or paired else (1 if g["kernel_name"] == "separable_kerr" else 0)
        assert g["variant"] == want_v and g["refill_min"] == refill_min and g["tuned"] == 0
        assert g["rays_per_warp"] == (16 if want_v == 3 else 32)
    b.launch()
    b.launch()  # the graph resets its queues: a second launch is a full trace again
    for d, out in zip(descs, b.outs):
        assert_same(to_np(out), single(renderer, d))
    b.close()


def test_autotuned_bundle_batch_tunes_rays_per_warp(renderer):
    """A bundle group's autotuner also times the two-lanes-per-ray variant
    (16 rays per warp): 4 variants x 4 thresholds; results bit-identical to
    kt_trace whichever wins."""
    # frames whose rays all end within a few thousand attempts (measured on the
    # oracle: at most 2306 and 3020); a bundle frame closer to the equator has
    # rays that creep to the step cap (ray_bundle.hpp:352-356), 500000 steps
    # at the default cap
    descs = [abi.frame_desc(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=96, height=54),
             abi.frame_desc(chart=1, bundles=1, a=0.9, theta_deg=60.0, width=64, height=40,
                            max_steps=3000)]
    b = renderer.batch(descs, options=abi.batch_options(autotune=True, tune_fraction=0.5))
    (g,) = b.groups()
    assert g["kernel_name"] == "bundles" and g["tuned"] == 1 and g["candidates"] == 16
    assert g["rays_per_warp"] == (16 if g["variant"] == 3 else 32)
    b.launch()
    for d, out in zip(descs, b.outs):
        assert_same(to_np(out), single(renderer, d))
    b.close()


def test_autotuned_batch(renderer):
    """Autotuning on a seeded uneven batch: every group tuned over all
    candidates, results bit-identical to kt_trace, and a strided sample of
    one frame bit-identical to the oracle."""
    import kerrtracecpp2_b200 as kt

    descs = kt.random_parameter_sets(n=8, seed=1, side_min=64, side_max=160)
    b = renderer.batch(descs, options=abi.batch_options(autotune=True, tune_fraction=0.25))
    groups = b.groups()
    assert sum(g["n_frames"] for g in groups) == len(descs)
    for g in groups:
        assert g["tuned"] == 1 and g["candidates"] == 12 and g["rays_per_warp"] == 32
        assert g["best_ms"] <= g["default_ms"]
        assert g["block"] in (64, 128) and g["grid"] > 0
    b.launch()
    for d, out in zip(descs, b.outs):
        assert_same(to_np(out), single(renderer, d))
    d = descs[0]
    pix = np.arange(0, d.width * d.height, 37, dtype=np.uint32)
    want = O.trace_port(d, pix=pix)
    got = to_np(b.outs[0])
    assert G.mismatches({k: got[k][pix] for k in G.FIELDS}, want) == {k: 0 for k in G.FIELDS}
    b.close()


def test_mixed_frames_in_batch(renderer):
    """Mixed-precision frames in a batch: the FP32 decision is per warp, so
    results depend on which rays share a warp; they keep the mixed
    tolerance against the FP64 frame."""
    kw = [dict(chart=0, a=0.5, width=320, height=180, fov_deg=45.0),
          dict(chart=1, integrator=1, tol=1e-8, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
               theta_deg=85.0, disk_out=20.0, width=256, height=144)]
    descs = [abi.frame_desc(precision=abi.KT_PREC_MIXED, **k) for k in kw]
    b = renderer.batch(descs)
    assert {g["kernel_name"] for g in b.groups()} == {"ks_rk4_mixed", "bl_dopri5_mixed"}
    b.launch()
    for k, out in zip(kw, b.outs):
        got = to_np(out)
        ref = single(renderer, abi.frame_desc(**k))
        same = got["outcome"] == ref["outcome"]
        disk = same & (ref["outcome"] == 1)
        eg = np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk])
        assert 1 - same.mean() < 1e-3
        assert np.median(eg) < 5e-6
    b.close()


def test_batch_rejects_bad_frames(renderer):
    import kerrtracecpp2_b200 as kt

    good = abi.frame_desc(width=8, height=8)
    bad = abi.frame_desc(width=0, height=8)
    with pytest.raises(kt.KerrTraceError) as e:
        renderer.batch([good, bad], outs=[renderer.alloc(64), renderer.alloc(64)])
    assert e.value.status == abi.KT_ERR_INVALID_ARGUMENT and "frame 1" in str(e.value)
    with pytest.raises(kt.KerrTraceError):
        renderer.batch([good], options=abi.batch_options(variant=abi.KT_BATCH_VARIANTS))
