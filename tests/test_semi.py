"""The semi-analytic solver (separable Kerr, main.cpp:436-703) on the CPU:
the oracle's restatement and the kernels' per-ray machine (SepRk4, host
build) against the reference's results in tests/golden/semi.npz, the
solver selection of kt_frame_derive, and the reference's own frame loop
against its per-ray results."""
import ctypes

import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
import testlibs
from kerrtracecpp2_b200 import abi

NAMES = sorted(G.semi_cases())
# The default-step-cap cases run 500000 attempts for each ray with a radial
# turning point; the oracle traces only the rays that end early and one of
# the others.
SLOW = ("semi_default_cap", "semi_tight_default_cap")


def pixels(name):
    if name not in SLOW:
        return None
    steps_done = np.flatnonzero(G.semi_result(name)["outcome"] != 0)
    stuck = np.flatnonzero(G.semi_result(name)["outcome"] == 0)[:1]
    return np.concatenate([steps_done, stuck]).astype(np.uint32)


def subset(res, pix):
    return res if pix is None else {k: v[pix] for k, v in res.items()}


@pytest.mark.parametrize("name", NAMES)
def test_port_matches_reference(name):
    pix = pixels(name)
    got = O.trace_port(G.semi_desc(name), pix=pix)
    assert G.mismatches(got, subset(G.semi_result(name), pix)) == {k: 0 for k in G.FIELDS}


@pytest.fixture(scope="module")
def hc():
    L = ctypes.CDLL(testlibs.HOSTCHECK)
    L.hc_trace_pixels.argtypes = [ctypes.POINTER(abi.FrameDesc), ctypes.c_int64, ctypes.c_void_p] + \
        [ctypes.c_void_p] * 10
    L.hc_trace_pixels.restype = ctypes.c_int
    return L


def hc_run(hc, d, pix):
    import test_hostcheck

    return test_hostcheck.run(hc, d, pix)


@pytest.mark.parametrize("name", NAMES)
def test_kernel_code_matches_reference(hc, name):
    """Every pixel, the default-cap frame included: the machine's right-hand
    side memo makes a ray parked at a turning point cheap."""
    got = hc_run(hc, G.semi_desc(name), None)
    assert G.mismatches(got, G.semi_result(name)) == {k: 0 for k in G.FIELDS}


def test_kernel_counters_match_oracle(hc):
    d = G.semi_desc("semi_kerr")
    got = hc_run(hc, d, None)
    want = O.trace_port(d, counters=True)
    assert np.array_equal(got["steps"], want["steps"])
    assert np.array_equal(got["attempts"], want["attempts"])
    # rays with a radial turning point run to the step cap
    cap = got["steps"] == d.max_steps
    assert cap.sum() > 0 and np.all(got["status"][cap] == 1)
    assert np.all(got["outcome"][cap] == abi.KT_OUT_ESCAPED)


@pytest.mark.parametrize("name", NAMES)
def test_reference_frame_loop_dispatch(name):
    """trace_geodesics' records = float32 of the per-ray results: the frame
    loop and the per-ray harness pick the same solver."""
    geo = G.semi()[f"{name}/geopixels"]
    res = G.semi_result(name)
    for k in G.FIELDS:
        want = res[k].astype(np.float32) if k != "outcome" else res[k]
        assert np.array_equal(G.bits(geo[k]), G.bits(want)), k


@pytest.mark.parametrize("kw,solver", [
    (dict(chart=abi.KT_CHART_BL, a=0.5), abi.KT_SOLVER_SEMI_ANALYTIC),
    (dict(chart=abi.KT_CHART_KS, a=0.5), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_BL, a=0.5, Q=0.1), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_BL, a=0.5, Lambda=1e-4), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_BL, a=0.5, bundles=1), abi.KT_SOLVER_STANDARD),
    (dict(chart=abi.KT_CHART_KS, a=0.5, Lambda=1e-4), abi.KT_SOLVER_STANDARD),
])
def test_solver_selection(kw, solver):
    import kerrtracecpp2_b200 as kt

    d = abi.frame_desc(solver_mode=abi.KT_SOLVER_SEMI_ANALYTIC, **kw)
    assert kt.frame_derive(d).solver == solver
    # the oracle applies the same rules
    out = abi.FrameDerived()
    O.port().orc_frame_derive(ctypes.byref(d), ctypes.byref(out))
    assert out.solver == solver


def test_unsupported_solver_requests():
    import kerrtracecpp2_b200 as kt

    with pytest.raises(kt.KerrTraceError) as e:
        kt.frame_derive(abi.frame_desc(solver_mode=abi.KT_SOLVER_SEMI_ANALYTIC, chart=abi.KT_CHART_BL,
                                       precision=abi.KT_PREC_MIXED))
    assert e.value.status == abi.KT_ERR_UNSUPPORTED
    with pytest.raises(kt.KerrTraceError) as e:
        kt.frame_derive(abi.frame_desc(solver_mode=7))
    assert e.value.status == abi.KT_ERR_INVALID_ARGUMENT
    # elliptic-closed with charge falls back to the standard tracers and runs
    assert kt.frame_derive(abi.frame_desc(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED, Q=0.2)).solver == 0
