"""The smooth tracer and its adjoint compiled for the host
(hc_smooth_pixels in tests/_build/libkt_hostcheck.so): the CPU twin of the
KT_PREC_SMOOTH kernels, used to check them bit for bit and to check the
adjoint against finite differences without a GPU."""
import ctypes

import numpy as np

import testlibs
from kerrtracecpp2_b200.abi import FrameDesc

N_SLOTS = 9  # a, Q, Lambda, theta [rad], r_obs, loss, n_grad, n_bl, n_unrecorded
_lib = None


def lib():
    global _lib
    if _lib is None:
        testlibs.build_all()
        L = ctypes.CDLL(testlibs.HOSTCHECK)
        P = ctypes.c_void_p
        L.hc_smooth_pixels.argtypes = ([ctypes.POINTER(FrameDesc), ctypes.c_int64, P, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int] + [P] * 5 + [ctypes.c_double] * 2 + [P] * 9)
        L.hc_smooth_pixels.restype = ctypes.c_int
        L.hc_smooth_pixels_m.argtypes = ([ctypes.POINTER(FrameDesc), ctypes.c_int64, P, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int] + [P] * 7 +
                                         [ctypes.c_double] * 3 + [P] * 10)
        L.hc_smooth_pixels_m.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def smooth(desc, pix=None, mode=0, cot_g=None, cot_r=None, target=None, w_g=1.0, w_r=0.0,
           force_bl=False, tangent=-1, cot_m=None, w_m=0.0):
    """Trace pixels `pix` (default: all) with the smooth tracer; mode 1/2
    also runs the adjoint (cotangent arrays over the whole frame, or the L2
    loss against `target`, a dict with outcome/redshift/r (and magnif) over
    the frame); with tangent = k (0 a, 1 Q, 2 Lambda, 3 theta, 4 r_obs) the
    derivative along that parameter comes from the forward-mode tangent
    instead.  Bundle frames: cot_m / w_m for the magnification.
    Returns (outputs dict, contrib[N_SLOTS][len(pix)] or None)."""
    n_frame = desc.width * desc.height
    pix = np.arange(n_frame, dtype=np.uint32) if pix is None else np.ascontiguousarray(pix, np.uint32)
    n = len(pix)
    out = {"outcome": np.zeros(n, np.uint8), "r": np.zeros(n), "redshift": np.zeros(n),
           "magnif": np.zeros(n), "phi_disk": np.zeros(n), "theta_esc": np.zeros(n),
           "phi_esc": np.zeros(n), "steps": np.zeros(n, np.uint32),
           "attempts": np.zeros(n, np.uint32)}
    contrib = np.zeros((N_SLOTS, n)) if mode else None
    t = target or {}
    arr = lambda a, dt: None if a is None else np.ascontiguousarray(a, dt)  # noqa: E731
    keep = [arr(cot_g, np.float64), arr(cot_r, np.float64), arr(cot_m, np.float64),
            arr(t.get("outcome"), np.uint8), arr(t.get("redshift"), np.float64),
            arr(t.get("r"), np.float64), arr(t.get("magnif") if w_m else None, np.float64)]
    rc = lib().hc_smooth_pixels_m(ctypes.byref(desc), n, _p(pix), mode, int(force_bl), int(tangent),
                                  *[_p(k) for k in keep], w_g, w_r, w_m,
                                  *[_p(out[k]) for k in ("outcome", "r", "redshift", "magnif",
                                                         "phi_disk", "theta_esc", "phi_esc",
                                                         "steps", "attempts")],
                                  _p(contrib))
    if rc != 0:
        raise ValueError("hc_smooth_pixels: frame rejected")
    return out, contrib
