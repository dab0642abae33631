"""Error statistics of the mixed-precision tracer and the host reference
it is split against (test infrastructure).

trace_fp64_rhs: the mixed tracer's per-ray code compiled for the host
(tests/_build/libkt_hostcheck.so) with its FP32 right-hand side and its
constraint reprojection off: the analytic FP64 Hamiltonian gradient with
correctly rounded reciprocals and the renderer's sincos, no contraction.
Against it, the GPU's mixed frame shows the mixed kernels' own error, and
the FP64 oracle shows the difference between the analytic gradient and
the reference's central differences (geodesic.hpp:143-166)."""
import ctypes

import numpy as np

import testlibs
from kerrtracecpp2_b200 import abi

_P = ctypes.c_void_p
_lib = None

KEYS = ["outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc", "status", "steps",
        "attempts"]


def _hc():
    global _lib
    if _lib is None:
        testlibs.build_all()
        L = ctypes.CDLL(testlibs.HOSTCHECK)
        L.hc_trace_pixels_fp64_rhs.argtypes = ([ctypes.POINTER(abi.FrameDesc), ctypes.c_int64, _P] +
                                               [_P] * 10 + [ctypes.c_double])
        L.hc_trace_pixels_fp64_rhs.restype = ctypes.c_int
        _lib = L
    return _lib


def trace_fp64_rhs(desc, pix=None, tol=0.0):
    """The frame `desc` (its precision is set to KT_PREC_MIXED) traced on the
    host with the mixed tracer's analytic FP64 right-hand side only; tol > 0
    overrides the frame's tolerance (which frames clamp to >= 1e-10)."""
    d = abi.frame_desc(**{**{f: getattr(desc, f) for f, _ in abi.FrameDesc._fields_},
                          "precision": abi.KT_PREC_MIXED})
    n = d.width * d.height
    pix = np.arange(n, dtype=np.uint32) if pix is None else np.ascontiguousarray(pix, np.uint32)
    dts = {"outcome": np.uint8, "status": np.uint8, "steps": np.uint32, "attempts": np.uint32}
    o = {k: np.zeros(len(pix), dts.get(k, np.float64)) for k in KEYS}
    assert _hc().hc_trace_pixels_fp64_rhs(ctypes.byref(d), len(pix), pix.ctypes.data_as(_P),
                                          *[o[k].ctypes.data_as(_P) for k in KEYS], tol) == 0
    return o


def error_stats(got, ref):
    """Per-pixel error of frame `got` against frame `ref` (dicts of numpy
    arrays): class mismatch fraction, and on the pixels that are disk hits
    in both the relative error of g and of the hit radius (quantiles, the
    maximum, and the fraction of pixels with g error above 1e-6)."""
    same = got["outcome"] == ref["outcome"]
    disk = same & (ref["outcome"] == 1)
    eg = np.abs(got["redshift"][disk] - ref["redshift"][disk]) / np.abs(ref["redshift"][disk])
    er = np.abs(got["r"][disk] - ref["r"][disk]) / np.abs(ref["r"][disk])

    def q(x, p):
        return float(np.percentile(x, p)) if x.size else 0.0

    return {"pixels": int(same.size), "class_mismatch": float(1.0 - same.mean()),
            "disk_pixels": int(disk.sum()),
            "g_p50": q(eg, 50), "g_p90": q(eg, 90), "g_p99": q(eg, 99), "g_p999": q(eg, 99.9),
            "g_max": float(eg.max()) if eg.size else 0.0,
            "g_frac_gt_1e-6": float((eg > 1e-6).mean()) if eg.size else 0.0,
            "r_p50": q(er, 50), "r_p99": q(er, 99), "r_max": float(er.max()) if er.size else 0.0}


def fmt(name, s):
    return (f"{name:34s} class {s['class_mismatch']:.1e}  g p50 {s['g_p50']:.1e} p90 {s['g_p90']:.1e} "
            f"p99 {s['g_p99']:.1e} p99.9 {s['g_p999']:.1e} max {s['g_max']:.1e} "
            f"(>1e-6: {s['g_frac_gt_1e-6']:.1%})  r_hit p50 {s['r_p50']:.1e} p99 {s['r_p99']:.1e} "
            f"max {s['r_max']:.1e}")
