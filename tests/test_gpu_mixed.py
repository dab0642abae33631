"""Mixed-precision kernels on the GPU against the FP64 kernels, which are
bit-identical to the reference (so this is the error against the FP64
oracle), over whole frames of the benchmark configurations."""
import numpy as np
import pytest

from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu

FRAMES = {
    "cfg2_720p_dopri5": dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                             theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=1280, height=720),
    "cfg1_ks_rk4": dict(chart=0, a=0.5, width=320, height=180, r_obs=40.0, theta_deg=80.0,
                        fov_deg=45.0, disk_out=12.0),
    "cfg5_ks_rk4": dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=512,
                        height=512),
    "cfg2_geometry_rk4": dict(chart=1, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
                              fov_deg=30.0, disk_out=20.0, width=640, height=360),
}


def trace(renderer, d):
    import torch

    out = renderer.trace(d)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("name", sorted(FRAMES))
def test_mixed_against_fp64(renderer, name):
    kw = FRAMES[name]
    ref = trace(renderer, abi.frame_desc(**kw))
    got = trace(renderer, abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw))
    same = got["outcome"] == ref["outcome"]
    disk = same & (ref["outcome"] == 1)
    eg = np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk])
    er = np.abs(got["r"][disk] - ref["r"][disk]) / np.abs(ref["r"][disk])
    print(f"{name}: class mismatch {1 - same.mean():.2e}, g rel err p50 {np.median(eg):.2e} "
          f"p99 {np.percentile(eg, 99):.2e}, r rel err p50 {np.median(er):.2e}")
    assert 1 - same.mean() < 1e-4
    assert np.median(eg) < 5e-6 and np.median(er) < 5e-5


def test_mixed_bundles_against_fp64(renderer):
    """Bundle mode (config 3 geometry at 1/100 of the pixels): the analytic
    Hessian-vector products against the reference's finite-difference
    Hessian; magnification compared on the disk pixels."""
    kw = dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=192, height=108)
    ref = trace(renderer, abi.frame_desc(**kw))
    got = trace(renderer, abi.frame_desc(precision=abi.KT_PREC_MIXED, **kw))
    same = got["outcome"] == ref["outcome"]
    disk = same & (ref["outcome"] == 1)
    eg = np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk])
    em = np.abs(got["magnif"][disk] - ref["magnif"][disk]) / np.abs(ref["magnif"][disk])
    print(f"bundles: class mismatch {1 - same.mean():.2e}, g rel p50 {np.median(eg):.2e}, "
          f"magnif rel p50 {np.median(em):.2e} p99 {np.percentile(em, 99):.2e}")
    assert 1 - same.mean() < 1e-3
    assert np.median(eg) < 5e-6 and np.median(em) < 1e-4
