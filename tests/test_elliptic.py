"""The elliptic-closed solver (main.cpp:705-1295) on the CPU: the oracle's
restatement and the kernels' code (kt_elliptic.cuh, host build) against the
reference's results in tests/golden/elliptic.npz, the fallback reason of
every pixel against the reference's, solver selection, and the reference's
frame loop against its per-ray results."""
import ctypes

import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
import testlibs
from kerrtracecpp2_b200 import abi

NAMES = sorted(G.ell_cases())


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_reference(name):
    got = O.trace_port(G.ell_desc(name))
    assert G.mismatches(got, G.ell_result(name)) == {k: 0 for k in G.FIELDS}


@pytest.mark.parametrize("name", [n for n in NAMES if f"{n}/reason" in G.ell()])
def test_port_fallback_reasons_match_reference(name):
    got = O.elliptic_reasons_port(G.ell_desc(name))
    assert np.array_equal(got, G.ell()[f"{name}/reason"])


@pytest.fixture(scope="module")
def hc():
    L = ctypes.CDLL(testlibs.HOSTCHECK)
    L.hc_trace_pixels.argtypes = [ctypes.POINTER(abi.FrameDesc), ctypes.c_int64, ctypes.c_void_p] + \
        [ctypes.c_void_p] * 10
    L.hc_trace_pixels.restype = ctypes.c_int
    return L


@pytest.mark.parametrize("name", NAMES)
def test_kernel_code_matches_reference(hc, name):
    import test_hostcheck

    got = test_hostcheck.run(hc, G.ell_desc(name))
    assert G.mismatches(got, G.ell_result(name)) == {k: 0 for k in G.FIELDS}


@pytest.mark.parametrize("name", NAMES)
def test_reference_frame_loop_dispatch(name):
    geo = G.ell()[f"{name}/geopixels"]
    res = G.ell_result(name)
    for k in G.FIELDS:
        want = res[k].astype(np.float32) if k != "outcome" else res[k]
        assert np.array_equal(G.bits(geo[k]), G.bits(want)), k


def test_closed_form_is_exercised():
    """The fixtures hold disk hits that come from the closed form (reason 0
    and a result that differs from the standard tracer's), rays the standard
    tracer keeps at the horizon, and every fallback reason but the
    constants' (the camera's rays always have E > 0)."""
    reasons = np.concatenate([v for k, v in G.ell().items() if k.endswith("/reason")])
    assert set(np.unique(reasons)) >= {0, 2, 4, 5}
    d = G.ell_desc("ell_kerr_bl")
    std = O.trace_port(abi.frame_desc(**dict(G.ell_cases()["ell_kerr_bl"], solver_mode=0)))
    ell = G.ell_result("ell_kerr_bl")
    changed = ell["r"] != std["r"]
    assert changed.sum() > 50 and np.all(ell["outcome"][changed] == 1)
    assert np.all(ell["phi_disk"][changed] == 0.0)
    assert d.width * d.height == len(changed)


@pytest.mark.parametrize("kw,solver", [
    (dict(chart=abi.KT_CHART_BL, a=0.5), abi.KT_SOLVER_ELLIPTIC_CLOSED),
    (dict(chart=abi.KT_CHART_KS, a=0.5), abi.KT_SOLVER_ELLIPTIC_CLOSED),
    (dict(chart=abi.KT_CHART_BL, a=0.5, Q=0.1), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_KS, a=0.5, Lambda=1e-4), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_BL, a=0.5, bundles=1), abi.KT_SOLVER_STANDARD),
])
def test_solver_selection(kw, solver):
    import kerrtracecpp2_b200 as kt

    d = abi.frame_desc(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED, **kw)
    assert kt.frame_derive(d).solver == solver
    out = abi.FrameDerived()
    O.port().orc_frame_derive(ctypes.byref(d), ctypes.byref(out))
    assert out.solver == solver


def test_fp64_only():
    import kerrtracecpp2_b200 as kt

    for prec in (abi.KT_PREC_MIXED, abi.KT_PREC_SMOOTH):
        with pytest.raises(kt.KerrTraceError) as e:
            kt.frame_derive(abi.frame_desc(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED, precision=prec))
        assert e.value.status == abi.KT_ERR_UNSUPPORTED
