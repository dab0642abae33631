"""kt_trace_noalloc: tracing for callers that may not allocate device memory
(a host that owns all device memory, or a frame loop that cannot afford
cudaMalloc/cudaFree).  Its results must equal kt_trace's bit for bit, on
two calls in a row (the shared scratch keeps the previous call's contents
and must be cleared by each call).  This file is collected last so that a
run stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

import golden_lib as G
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu


def _alloc(n):
    import torch

    dt = {"u1": torch.uint8, "f8": torch.float64, "u4": torch.int32}
    return {k: torch.empty(n, dtype=dt[d], device="cuda") for k, d in abi.GEO_FIELDS}


def _soa(out):
    s = abi.GeoSoA()
    for k, _ in abi.GEO_FIELDS:
        setattr(s, k, out[k].data_ptr())
    return s


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("kw", [
    dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
         fov_deg=30.0, disk_out=20.0, width=160, height=90),   # BL DOPRI5 (queue counters)
    dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=96,
         height=96),                                           # KS (queue + fallback list)
    dict(chart=0, a=0.7, Q=0.1, theta_deg=0.0, r_obs=50.0, disk_out=15.0, width=48,
         height=48),                                           # KS, every ray in the fallback list
    dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=320,
         height=240),                                          # KS, centre-out order (>= 2^16 pixels)
], ids=["bl_dopri5", "ks_rk4", "ks_polar_fallback", "ks_centre_out"])
def test_noalloc_matches_kt_trace_twice(kw):
    import torch
    import kerrtracecpp2_b200 as kt

    L = kt.load_library()
    d = abi.frame_desc(**kw)
    n = d.width * d.height
    with kt.Renderer(0) as r:
        want = _np(r.trace(d))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        out = _alloc(n)
        assert L.kt_trace_noalloc(ctypes.byref(d), ctypes.byref(_soa(out)), stream) == abi.KT_OK
        torch.cuda.synchronize()
        got = _np(out)
        fields = G.FIELDS + ("status", "steps", "attempts")
        for k in fields:
            assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), k
    if kw["theta_deg"] == 0.0:
        # a camera on the axis: the KS initialisation of every ray fails
        # (main.cpp:1537-1545), so the frame is the BL trace of the same rays
        # (the fallback launch read every entry of the fallback list)
        with kt.Renderer(0) as r:
            bl = _np(r.trace(abi.frame_desc(**dict(kw, chart=1))))
        for k in G.FIELDS + ("steps", "attempts"):
            assert np.array_equal(got[k].view(np.uint8), bl[k].view(np.uint8)), k


def test_noalloc_rejects_frames_beyond_its_scratch():
    import torch
    import kerrtracecpp2_b200 as kt

    L = kt.load_library()
    d = abi.frame_desc(width=1025, height=1024)  # 1 row more than the 2^20-pixel limit
    out = _alloc(1)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.kt_trace_noalloc(ctypes.byref(d), ctypes.byref(_soa(out)), stream) == \
        abi.KT_ERR_INVALID_ARGUMENT
    assert L.kt_trace_noalloc(None, ctypes.byref(_soa(out)), stream) == abi.KT_ERR_INVALID_ARGUMENT
