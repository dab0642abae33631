"""Mixed-precision tracer (KT_PREC_MIXED) on the CPU (its per-ray code
compiled for the host): analytic Hamiltonian gradient, FP32 right-hand side
in the far field when the tolerance allows, FP64 integrator.  Its results
differ from the FP64 oracle by about the oracle's own finite-difference
noise; the bars below are the ones the GPU tests use."""
import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
from test_hostcheck import hc, run  # noqa: F401  (fixture + runner)
from kerrtracecpp2_b200 import abi


def errors(got, want):
    same = got["outcome"] == want["outcome"]
    disk = same & (want["outcome"] == 1)
    eg = np.abs(got["redshift"][disk] - want["redshift"][disk]) / np.abs(want["redshift"][disk])
    er = np.abs(got["r"][disk] - want["r"][disk]) / np.abs(want["r"][disk])
    return 1.0 - same.mean(), eg, er


CASES = {
    "cfg2_bl_dopri5": dict(width=48, height=27),
    "cfg2_bl_rk4": dict(width=48, height=27),
    "cfg1_ks_rk4": dict(width=64, height=36),
    "cfg5_ks": dict(width=48, height=48),
    "kn_charged": dict(),
    "retrograde": dict(),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_close_to_fp64_oracle(hc, name):  # noqa: F811
    kw = dict(G.cases()[name])
    kw["precision"] = abi.KT_PREC_MIXED
    d = abi.frame_desc(**kw)
    got = run(hc, d)
    mism, eg, er = errors(got, G.result(name))
    n = d.width * d.height
    assert mism * n <= max(1, 1e-3 * n)
    assert np.median(eg) < 1e-5 and np.percentile(eg, 99) < 1e-3
    assert np.median(er) < 1e-4


def test_mixed_uses_fp32_only_for_loose_tolerance():
    import kerrtracecpp2_b200 as kt

    strict = kt.frame_derive(abi.frame_desc(precision=abi.KT_PREC_MIXED, tol=1e-10, width=4, height=4))
    loose = kt.frame_derive(abi.frame_desc(precision=abi.KT_PREC_MIXED, tol=1e-7, width=4, height=4))
    assert strict.r_fp32 == float("inf")
    assert loose.r_fp32 == max(4.0, 2.0 * loose.r_horizon)


@pytest.mark.parametrize("name", ["cfg3_bundles", "bundle_step_cap"])
def test_mixed_bundles_close_to_fp64_oracle(hc, name):  # noqa: F811
    """Bundle mode with the analytic Hessian-vector products (one Dual<2>
    gradient per RHS): class, g and the Jacobi magnification against the
    reference's finite-difference Hessian."""
    kw = dict(G.cases()[name])
    kw["precision"] = abi.KT_PREC_MIXED
    d = abi.frame_desc(**kw)
    got = run(hc, d)
    want = G.result(name)
    mism, eg, er = errors(got, want)
    n = d.width * d.height
    assert mism * n <= max(1, 1e-3 * n)
    disk = (got["outcome"] == want["outcome"]) & (want["outcome"] == 1)
    if disk.any():
        assert np.median(eg) < 1e-5 and np.median(er) < 1e-4
        em = np.abs(got["magnif"][disk] - want["magnif"][disk]) / np.abs(want["magnif"][disk])
        assert np.median(em) < 1e-4


@pytest.mark.parametrize("chart", [abi.KT_CHART_BL, abi.KT_CHART_KS])
def test_constraint_reprojection(hc, chart):
    """The mixed tracer's Hamiltonian-constraint reprojection (host build of
    bl_reproject / ks_reproject): camera rays whose evolved momenta are
    scaled by 1 + eps (H = O(eps)) come back onto H = 0 to rounding when
    the drift is below its 1e-4 bound, and are left alone above it or where
    the FP32 right-hand side is off (tol below 1e-8)."""
    import ctypes

    import numpy as np

    hc.hc_reproject.argtypes = [ctypes.POINTER(abi.FrameDesc), ctypes.c_uint32, ctypes.c_double,
                                ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    hc.hc_reproject.restype = ctypes.c_int
    kw = dict(chart=chart, a=0.7, Q=0.2, width=32, height=18, r_obs=50.0, theta_deg=70.0,
              fov_deg=40.0, precision=abi.KT_PREC_MIXED, tol=1e-7)
    hb, ha = ctypes.c_double(), ctypes.c_double()
    rng = np.random.default_rng(5)
    for pix in rng.integers(0, 32 * 18, 12):
        for eps in (3e-8, -2e-6, 4e-5):
            d = abi.frame_desc(**kw)
            assert hc.hc_reproject(ctypes.byref(d), int(pix), eps, ctypes.byref(hb), ctypes.byref(ha)) == 1
            assert abs(hb.value) > 1e-9 and abs(ha.value) < 1e-13, (pix, eps, hb.value, ha.value)
        d = abi.frame_desc(**kw)
        assert hc.hc_reproject(ctypes.byref(d), int(pix), 1e-3, ctypes.byref(hb), ctypes.byref(ha)) == 0
        assert ha.value == hb.value
        d = abi.frame_desc(**dict(kw, tol=1e-9))
        assert hc.hc_reproject(ctypes.byref(d), int(pix), 1e-5, ctypes.byref(hb), ctypes.byref(ha)) == 0


def test_oracle_and_analytic_gradient_equally_close_to_a_tighter_trace():
    """What the mixed tracer's error against the FP64 oracle measures: at the
    headline tolerance (config 2 geometry, DOPRI5, tol 1e-10, 80x45) the
    oracle F and the analytic-gradient FP64 trace A are about equally far
    from the same frame traced at tol 1e-13 (beyond the clamp a frame
    accepts), and about as far from each other.  The reference's disk
    crossing is the midpoint of an 8 x 8 bisection of the last step
    (geodesic.hpp:49-140), so traces whose step sequences differ disagree at
    the 1e-6 level in the hit radius and g; the finite-difference gradient
    is enough to move the step sequence.  Neither trace is the more exact."""
    import mixed_lib as X

    d = abi.frame_desc(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                       theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=80, height=45)
    T = X.trace_fp64_rhs(d, tol=1e-13)
    A = X.trace_fp64_rhs(d)
    F = O.trace_port(d)
    at, ft, af = X.error_stats(A, T), X.error_stats(F, T), X.error_stats(A, F)
    for k, v in (("A analytic FP64 vs T (tol 1e-13)", at), ("F oracle vs T (tol 1e-13)", ft),
                 ("A vs F", af)):
        print(X.fmt(k, v))
    assert at["class_mismatch"] == 0 and ft["class_mismatch"] == 0
    assert 0.5 < at["g_p50"] / ft["g_p50"] < 2.0
    assert 0.5 < af["g_p50"] / ft["g_p50"] < 2.0
    assert ft["g_p50"] < 2e-6
