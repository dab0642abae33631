"""The smooth tracer and its adjoint on the GPU (kt_trace with
KT_PREC_SMOOTH, kt_vjp, kt_l2_grad): bit-identical to the host build of the
same code (smooth_lib), and on config 5 (512x512 KS, a=0.7, Q=0.1,
theta=70, r_obs=50, disk ISCO-15, L2 loss against the same tracer at a=0.72,
theta=71) the gradient against five-point central differences of the loss
restricted to the pixels on which every stencil is smooth (see
test_smooth.py)."""
import numpy as np
import pytest

import smooth_lib as S
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu

CFG5 = dict(chart=0, a=0.7, Q=0.1, Lambda=0.0, theta_deg=70.0, r_obs=50.0, disk_out=15.0)
KNDS = dict(chart=1, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0, disk_out=20.0)
# Jacobi bundles: configuration 3's geometry, and a KNdS bundle frame
CFG3 = dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, r_obs=40.0, fov_deg=30.0, disk_out=12.0,
            max_steps=20000)
BUNDLE = dict(chart=1, bundles=1, a=0.9, Q=0.2, Lambda=1e-5, theta_deg=70.0, r_obs=40.0,
              fov_deg=30.0, disk_out=12.0, max_steps=20000)
FIELDS = ["outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc", "steps",
          "attempts"]


def to_np(out):
    import torch

    torch.cuda.synchronize()
    got = {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}
    got["steps"] = got["steps"].view(np.uint32)
    got["attempts"] = got["attempts"].view(np.uint32)
    return got


def smooth_gpu(renderer, kw):
    return to_np(renderer.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **kw)))


@pytest.mark.parametrize("kw", [dict(CFG5, width=96, height=96), dict(KNDS, width=96, height=54),
                                dict(CFG5, width=77, height=31, tol=1e-10),
                                dict(KNDS, integrator=abi.KT_DOPRI5, tol=1e-10, fov_deg=30.0,
                                     width=96, height=54),
                                dict(CFG3, width=96, height=54), dict(BUNDLE, width=96, height=54)],
                         ids=["cfg5_ks", "knds_bl", "cfg5_tight", "knds_bl_dopri5", "cfg3_bundle",
                              "knds_bundle"])
def test_smooth_trace_gpu_equals_host(renderer, kw):
    got = smooth_gpu(renderer, kw)
    want, _ = S.smooth(abi.frame_desc(**kw))
    for f in FIELDS:
        assert np.array_equal(got[f], want[f]), f


@pytest.mark.parametrize("kw", [dict(CFG5, width=64, height=64), dict(KNDS, width=64, height=36),
                                dict(KNDS, integrator=abi.KT_DOPRI5, tol=1e-10, fov_deg=30.0,
                                     width=64, height=36),
                                dict(BUNDLE, width=64, height=36)],
                         ids=["ks", "bl", "bl_dopri5", "bundle"])
def test_vjp_gpu_equals_host(renderer, kw):
    import torch

    d = abi.frame_desc(**kw)
    n = d.width * d.height
    rng = np.random.default_rng(7)
    cg, cr = rng.normal(size=n), rng.normal(size=n)
    cm = rng.normal(size=n) if kw.get("bundles") else None
    out = renderer.alloc(n)
    grad, st = renderer.vjp(d, torch.from_numpy(cg).cuda(), torch.from_numpy(cr).cuda(), out=out,
                            cot_magnif=torch.from_numpy(cm).cuda() if cm is not None else None)
    fwd, c = S.smooth(d, mode=1, cot_g=cg, cot_r=cr, cot_m=cm)
    got = to_np(out)
    for f in FIELDS:
        assert np.array_equal(got[f], fwd[f]), f
    h = c.sum(axis=1)
    want = [h[0], h[1], h[2], h[3] * np.pi / 180, h[4], 0.0]
    if kw["chart"] == 0:
        _, cl = S.smooth(d, mode=1, cot_g=cg, cot_r=cr, force_bl=True, tangent=2)
        want[2] = cl.sum(axis=1)[2]
    np.testing.assert_allclose(grad, want, rtol=1e-11, atol=1e-12 * np.abs(want).max())
    assert st["grad_pixels"] == int(h[6]) and st["unrecorded"] == 0
    assert st["bl_pixels"] == (0 if kw["chart"] == 0 else n)


def test_config5_l2_gradient_against_central_differences(renderer):
    """512x512, tol 1e-7: kt_l2_grad's loss equals the loss of its own
    forward, and the VJP with the loss's cotangents on the smooth pixels
    agrees with central differences of that loss (tests/grad_lib.py):
    five-point differences with h = 1e-4 (theta in radians; Lambda 1e-6)
    and two-point differences with h = 1e-6 (Lambda 1e-8), the target's
    check, on the same smooth pixels, to 1e-5 relative; on the looser mask
    (every pixel whose class and step sequence survive +-1e-6) the two-point
    differences are reported and bounded at 1e-4."""
    import grad_lib

    base = dict(CFG5, width=512, height=512)
    n = 512 * 512
    wg, wr = grad_lib.W_G, grad_lib.W_R
    tgt_t = renderer.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **dict(base, a=0.72, theta_deg=71.0)))
    tgt = to_np(tgt_t)
    out = renderer.alloc(n)
    loss, grad_l2, st = renderer.l2_grad(abi.frame_desc(**base), tgt_t, wg, wr, out=out)
    b0 = to_np(out)
    m_all = (b0["outcome"] == 1) & (tgt["outcome"] == 1)
    want_loss = np.sum(wg * (b0["redshift"][m_all] - tgt["redshift"][m_all]) ** 2 +
                       wr * (b0["r"][m_all] - tgt["r"][m_all]) ** 2)
    assert loss == pytest.approx(want_loss, rel=1e-12)
    assert st["grad_pixels"] == m_all.sum()
    assert grad_l2[abi.GRAD_NAMES.index("disk_out")] == 0.0

    res = grad_lib.fd_check(renderer, base)
    for name, r in res.items():
        print(f"{name} h={r['h']:g}: {r['pixels']} of {r['disk_pixels']} disk pixels in the loss")
        for k, v in r["per_param"].items():
            print(f"  {k}: adjoint {v['adjoint']:.10g} differences {v['fd']:.10g} rel {v['rel']:.2e}")
    assert res["five_point"]["worst_rel"] <= 1e-5
    assert res["two_point"]["worst_rel"] <= 1e-5
    assert res["two_point_loose"]["worst_rel"] <= 1e-4
    assert res["five_point"]["pixels"] > 0.3 * res["five_point"]["disk_pixels"]
    assert res["two_point"]["pixels"] > 0.3 * res["two_point"]["disk_pixels"]
    assert res["two_point_loose"]["pixels"] > 0.5 * res["two_point_loose"]["disk_pixels"]


def test_config2_dopri5_gradient_against_central_differences(renderer):
    """The DOPRI5 adjoint (the smooth tracer's dopri5_adaptive, its reverse
    with the embedded error norm and the controller differentiated): config
    2's geometry at 320x180, tol 1e-10, L2 loss against a=0.92, theta=86;
    five-point (h = 1e-4) and two-point (h = 1e-6) central differences on the
    smooth pixels to 1e-5 relative, the loose mask to 1e-4."""
    import grad_lib

    res = grad_lib.fd_check(renderer, grad_lib.CFG2_DOPRI5, target=grad_lib.TARGET_CFG2)
    for name, r in res.items():
        print(f"{name} h={r['h']:g}: {r['pixels']} of {r['disk_pixels']} disk pixels in the loss")
        for k, v in r["per_param"].items():
            print(f"  {k}: adjoint {v['adjoint']:.10g} differences {v['fd']:.10g} rel {v['rel']:.2e}")
    assert res["five_point"]["worst_rel"] <= 1e-5
    assert res["two_point"]["worst_rel"] <= 1e-5
    assert res["two_point_loose"]["worst_rel"] <= 1e-4
    assert res["five_point"]["pixels"] > 0.3 * res["five_point"]["disk_pixels"]


def test_bundle_gradient_against_central_differences(renderer):
    """The bundle adjoint (the Jacobi matrix's equation differentiated with
    third derivatives of H by hyper-dual numbers, the magnification's
    dependence on W and on the crossing): a KNdS bundle frame at 320x180,
    tol 1e-9, L2 loss of (g, r_hit, magnification) against a=0.92,
    theta=71: five-point (h = 1e-4) central differences on the smooth
    pixels to 1e-5 relative, two-point (h = 1e-6) on the same pixels to
    1e-4 (the magnification's rounding noise over 2h), the loose mask
    reported and bounded at 1e-3."""
    import grad_lib

    res = grad_lib.fd_check(renderer, grad_lib.BUNDLE, target=grad_lib.TARGET_BUNDLE, w_m=grad_lib.W_M)
    for name, r in res.items():
        print(f"{name} h={r['h']:g}: {r['pixels']} of {r['disk_pixels']} disk pixels in the loss")
        for k, v in r["per_param"].items():
            print(f"  {k}: adjoint {v['adjoint']:.10g} differences {v['fd']:.10g} rel {v['rel']:.2e}")
    assert res["five_point"]["worst_rel"] <= 1e-5
    assert res["two_point"]["worst_rel"] <= 1e-4
    assert res["two_point_loose"]["worst_rel"] <= 1e-3
    assert res["five_point"]["pixels"] > 0.3 * res["five_point"]["disk_pixels"]


def test_pixel_list_gradients_add_up(renderer):
    """A frame's gradient split into the tiles of three ranks
    (kerrtracecpp2_b200.shard.frame_tiles, kt_l2_grad_pixels on each share)
    sums to the whole frame's: the per-pixel work is the same, only the
    summation order differs.  KS frame, so the Lambda tangent pass is split
    too."""
    import torch

    from kerrtracecpp2_b200 import shard

    base = dict(CFG5, width=128, height=96)
    tgt = renderer.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **dict(base, a=0.72, theta_deg=71.0)))
    d = abi.frame_desc(**base)
    loss, grad, st = renderer.l2_grad(d, tgt, 1.0, 0.01)
    tot_loss, tot_grad, tot_pix = 0.0, np.zeros(abi.KT_GRAD_COUNT), 0
    for rank in range(3):
        pix = torch.from_numpy(shard.frame_tiles(d.width, d.height, 3, rank, 16).astype(np.int32)).cuda()
        l_r, g_r, s_r = renderer.l2_grad(d, tgt, 1.0, 0.01, pix=pix)
        tot_loss += l_r
        tot_grad += g_r
        tot_pix += s_r["grad_pixels"]
    assert tot_pix == st["grad_pixels"]
    assert tot_loss == pytest.approx(loss, rel=1e-12)
    np.testing.assert_allclose(tot_grad, grad, rtol=1e-10, atol=1e-12 * np.abs(grad).max())
