"""ctypes bindings of the oracle libraries (test infrastructure).

  port   : oracle/_build/liboracle_port.so  -- the C restatement (kt_oracle.c)
  strict : oracle/_ref/libktref_strict.so   -- the reference compiled with the
                                               renderer's libm, no contraction
  stock  : oracle/_ref/libktref_stock.so    -- the reference as shipped (-O3
                                               -ffast-math, glibc libm)
  ieee   : oracle/_ref/libktref_ieee.so     -- the reference at -O3 without
                                               -ffast-math, glibc libm

Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
import ctypes
import os

import numpy as np

from kerrtracecpp2_b200.abi import ColorParams, FrameDerived, FrameDesc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PORT_PATH = os.path.join(ROOT, "oracle", "_build", "liboracle_port.so")
REF_PATHS = {
    "strict": os.path.join(ROOT, "oracle", "_ref", "libktref_strict.so"),
    "stock": os.path.join(ROOT, "oracle", "_ref", "libktref_stock.so"),
    "ieee": os.path.join(ROOT, "oracle", "_ref", "libktref_ieee.so"),
}

_P = ctypes.c_void_p
_D = ctypes.c_double
_cache = {}


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


def port():
    if "port" not in _cache:
        if not os.path.exists(PORT_PATH):
            raise FileNotFoundError(f"{PORT_PATH} missing: run python oracle/build.py")
        L = ctypes.CDLL(PORT_PATH)
        L.orc_trace_pixels.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64, _P] + [_P] * 9 + [ctypes.c_int]
        L.orc_trace_pixels.restype = None
        L.orc_frame_derive.argtypes = [ctypes.POINTER(FrameDesc), ctypes.POINTER(FrameDerived)]
        L.orc_colorize.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64] + [_P] * 6 + [_D] * 3 + [_P, ctypes.c_int, ctypes.c_int, _P]
        L.orc_colorize.restype = None
        PC = ctypes.POINTER(ColorParams)
        L.orc_colorize_cp.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64] + [_P] * 7 + [PC, _P, ctypes.c_int, ctypes.c_int, _P]
        L.orc_colorize_cp.restype = None
        L.orc_spp_offsets.argtypes = [ctypes.c_int, _P]
        L.orc_spp_offsets.restype = None
        L.orc_spp_combine.argtypes = [ctypes.c_int64, ctypes.c_int, _P, _D, _P]
        L.orc_spp_combine.restype = None
        L.orc_elliptic_reasons.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64, _P, _P]
        L.orc_elliptic_reasons.restype = None
        for f in ("orc_r_horizon", "orc_r_isco"):
            getattr(L, f).argtypes = [_D] * 4
            getattr(L, f).restype = _D
        _cache["port"] = L
    return _cache["port"]


def ref_available(flavour="strict"):
    return os.path.exists(REF_PATHS[flavour])


def ref(flavour="strict"):
    key = "ref_" + flavour
    if key not in _cache:
        path = REF_PATHS[flavour]
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run python oracle/build.py (needs the reference tree)")
        L = ctypes.CDLL(path)
        L.ref_trace_pixels.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64, _P] + [_P] * 7 + [ctypes.c_int]
        L.ref_trace_pixels.restype = None
        L.ref_trace_geodesics.argtypes = [ctypes.POINTER(FrameDesc), _P, ctypes.c_int]
        L.ref_elliptic_reasons.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64, _P, _P, ctypes.c_int]
        L.ref_elliptic_reasons.restype = None
        L.ref_colorize.argtypes = [_P, ctypes.c_int, ctypes.c_int, _D, _D, _D, _P, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _P]
        L.ref_colorize.restype = None
        PC = ctypes.POINTER(ColorParams)
        L.ref_colorize_cp.argtypes = [_P, ctypes.c_int, ctypes.c_int, PC, _P, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _P]
        L.ref_colorize_cp.restype = None
        L.ref_render_image.argtypes = [ctypes.POINTER(FrameDesc), PC, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]
        L.ref_render_image.restype = None
        for f in ("ref_r_horizon", "ref_r_isco"):
            getattr(L, f).argtypes = [_D] * 4
            getattr(L, f).restype = _D
        L.ref_libm_probe_cos.argtypes = [_D]
        L.ref_libm_probe_cos.restype = _D
        L.ref_contravariant_BL.argtypes = [_D] * 6 + [_P]
        L.ref_covariant_BL.argtypes = [_D] * 6 + [_P]
        L.ref_angle_ray.argtypes = [_D] * 8 + [ctypes.c_int, ctypes.c_int, _D, _D, _P]
        L.ref_hamiltonian.argtypes = [_D] * 4 + [_P]
        L.ref_hamiltonian.restype = _D
        L.ref_adaptive_step.argtypes = [_D] * 4 + [_P, _P, ctypes.c_int, _P, _D]
        L.ref_adaptive_step.restype = ctypes.c_int
        L.ref_keplerian_omega.argtypes = [_D] * 5
        L.ref_keplerian_omega.restype = _D
        L.ref_bl_to_ks.argtypes = [_D] * 4 + [_P]
        L.ref_ks_to_bl.argtypes = [_D] * 4 + [_P]
        L.ref_r_ks.argtypes = [_D] * 4
        L.ref_r_ks.restype = _D
        _cache[key] = L
    return _cache[key]


def all_pixels(desc):
    return np.arange(desc.width * desc.height, dtype=np.uint32)


def _alloc(n):
    return {
        "outcome": np.zeros(n, np.uint8), "r": np.zeros(n), "redshift": np.zeros(n),
        "magnif": np.zeros(n), "phi_disk": np.zeros(n), "theta_esc": np.zeros(n),
        "phi_esc": np.zeros(n),
    }


def trace_port(desc, pix=None, nthreads=0, counters=False):
    pix = all_pixels(desc) if pix is None else np.ascontiguousarray(pix, np.uint32)
    n = len(pix)
    out = _alloc(n)
    steps = np.zeros(n, np.uint32) if counters else None
    att = np.zeros(n, np.uint32) if counters else None
    port().orc_trace_pixels(ctypes.byref(desc), n, _ptr(pix), *[_ptr(out[k]) for k in
                            ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")],
                            _ptr(steps), _ptr(att), nthreads)
    if counters:
        out["steps"], out["attempts"] = steps, att
    return out


def trace_ref(desc, flavour="strict", pix=None, nthreads=0):
    pix = all_pixels(desc) if pix is None else np.ascontiguousarray(pix, np.uint32)
    n = len(pix)
    out = _alloc(n)
    ref(flavour).ref_trace_pixels(ctypes.byref(desc), n, _ptr(pix), *[_ptr(out[k]) for k in
                                  ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")],
                                  nthreads)
    return out


GEOPIXEL_DTYPE = np.dtype([("outcome", "u1"), ("pad", "u1", 3), ("r", "<f4"), ("redshift", "<f4"),
                           ("magnif", "<f4"), ("phi_disk", "<f4"), ("theta_esc", "<f4"),
                           ("phi_esc", "<f4")])


def elliptic_reasons_ref(desc, flavour="strict", pix=None, nthreads=0):
    """The reference's elliptic-closed fallback reason per pixel (uint8)."""
    pix = all_pixels(desc) if pix is None else np.ascontiguousarray(pix, np.uint32)
    out = np.zeros(len(pix), np.uint8)
    ref(flavour).ref_elliptic_reasons(ctypes.byref(desc), len(pix), _ptr(pix), _ptr(out), nthreads)
    return out


def elliptic_reasons_port(desc, pix=None):
    """The oracle's elliptic-closed fallback reason per pixel (uint8)."""
    pix = all_pixels(desc) if pix is None else np.ascontiguousarray(pix, np.uint32)
    out = np.zeros(len(pix), np.uint8)
    port().orc_elliptic_reasons(ctypes.byref(desc), len(pix), _ptr(pix), _ptr(out))
    return out


def trace_geodesics_ref(desc, flavour="strict", nthreads=0):
    """The reference's own frame loop: GeoPixel records (float32)."""
    out = np.zeros(desc.width * desc.height, GEOPIXEL_DTYPE)
    ref(flavour).ref_trace_geodesics(ctypes.byref(desc), _ptr(out), nthreads)
    return out


def colorize_port(desc, geo, bg=None, exposure=1.0, gamma=2.2, temp_scale=1.0):
    n = len(geo["outcome"])
    rgb = np.zeros((n, 3), np.uint8)
    bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
    bgc = np.ascontiguousarray(bg) if bg is not None else None
    port().orc_colorize(ctypes.byref(desc), n, *[_ptr(np.ascontiguousarray(geo[k])) for k in
                        ("outcome", "r", "redshift", "magnif", "theta_esc", "phi_esc")],
                        exposure, gamma, temp_scale, _ptr(bgc), bw, bh, _ptr(rgb))
    return rgb


def colorize_ref(desc, geopixels, r_isco, bg=None, exposure=1.0, gamma=2.2, temp_scale=1.0,
                 flavour="strict"):
    n = desc.width * desc.height
    rgb = np.zeros((n, 3), np.uint8)
    bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
    bgc = np.ascontiguousarray(bg) if bg is not None else None
    ref(flavour).ref_colorize(_ptr(geopixels), desc.width, desc.height, exposure, gamma, temp_scale,
                              _ptr(bgc), bw, bh, desc.M, r_isco, r_isco, desc.disk_out, _ptr(rgb))
    return rgb


def colorize_port_cp(desc, geo, cp, bg=None):
    """orc_colorize_cp: both palettes (cp a kt_color_params)."""
    n = len(geo["outcome"])
    rgb = np.zeros((n, 3), np.uint8)
    bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
    bgc = np.ascontiguousarray(bg) if bg is not None else None
    port().orc_colorize_cp(ctypes.byref(desc), n, *[_ptr(np.ascontiguousarray(geo[k])) for k in
                           ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")],
                           ctypes.byref(cp), _ptr(bgc), bw, bh, _ptr(rgb))
    return rgb


def colorize_ref_cp(desc, geopixels, r_isco, cp, bg=None, flavour="strict"):
    """The reference's colorize_buffer with every ColorParams field."""
    n = desc.width * desc.height
    rgb = np.zeros((n, 3), np.uint8)
    bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
    bgc = np.ascontiguousarray(bg) if bg is not None else None
    ref(flavour).ref_colorize_cp(_ptr(geopixels), desc.width, desc.height, ctypes.byref(cp), _ptr(bgc),
                                 bw, bh, desc.M, r_isco, r_isco, desc.disk_out, _ptr(rgb))
    return rgb


def render_ref(desc, cp, spp, bg=None, flavour="strict", nthreads=0):
    """The reference's render_image (CPU branch) with camera_spp passes."""
    n = desc.width * desc.height
    rgb = np.zeros((n, 3), np.uint8)
    bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
    bgc = np.ascontiguousarray(bg) if bg is not None else None
    ref(flavour).ref_render_image(ctypes.byref(desc), ctypes.byref(cp), _ptr(bgc), bw, bh, spp,
                                  nthreads, _ptr(rgb))
    return rgb


def spp_offsets_port(spp):
    xy = np.zeros(2 * max(spp, 1))
    port().orc_spp_offsets(spp, _ptr(xy))
    return xy.reshape(-1, 2)


def spp_combine_port(passes, gamma):
    """passes: (spp, n, 3) uint8 -> (n, 3) uint8, the reference's average."""
    spp, n = passes.shape[0], passes.shape[1]
    rgb = np.zeros((n, 3), np.uint8)
    port().orc_spp_combine(n, spp, _ptr(np.ascontiguousarray(passes)), gamma, _ptr(rgb))
    return rgb


def to_geopixels(geo):
    """float64 SoA -> GeoPixel records, as trace_geodesics stores them."""
    n = len(geo["outcome"])
    g = np.zeros(n, GEOPIXEL_DTYPE)
    for k in ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc"):
        g[k] = geo[k]
    return g


def derive_port(desc):
    d = FrameDerived()
    port().orc_frame_derive(ctypes.byref(desc), ctypes.byref(d))
    return d


def boundary_distance(outcome, pix, radius=8):
    """For pixels whose class differs between two renders: the largest, over
    those pixels, of the distance (in pixels) to the nearest pixel of another
    class in `outcome` (H x W) -- how far from a class boundary (critical
    curve, disk edge) a disagreement lies.  None without disagreements;
    radius + 1 when some lies farther than `radius`."""
    if len(pix) == 0:
        return None
    H, W = outcome.shape
    worst = 0.0
    for p in np.asarray(pix, np.int64):
        y, x = divmod(int(p), W)
        y0, y1, x0, x1 = max(0, y - radius), min(H, y + radius + 1), max(0, x - radius), min(W, x + radius + 1)
        yy, xx = np.nonzero(outcome[y0:y1, x0:x1] != outcome[y, x])
        d = float(np.min(np.hypot(yy + y0 - y, xx + x0 - x))) if yy.size else radius + 1.0
        worst = max(worst, d)
    return worst


GEO_FIELDS = ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")


KT_RAY_CREEP = 4  # include/kerrtrace.h: a bundle ray stopped while creeping onto r_+


def creep_mask(got, pix=None):
    """Pixels (of `pix`) that the library stopped while creeping onto the
    horizon (status KT_RAY_CREEP): their records equal the reference's, but
    their step and attempt counts stop early (the oracle, like the
    reference, traces them on to the reject or step cap)."""
    st = got.get("status")
    if st is None:
        return None
    st = np.asarray(st)
    return (st if pix is None else st[np.asarray(pix, np.int64)]) == KT_RAY_CREEP


def counters_agree(got, want, pix=None):
    """(ok, creeping): the step and attempt counters of `got` equal the
    oracle's on every pixel but the creeping ones, where they are no larger."""
    creep = creep_mask(got, pix)
    ok = True
    for f in ("steps", "attempts"):
        a = np.asarray(got[f]) if pix is None else np.asarray(got[f])[np.asarray(pix, np.int64)]
        b = np.asarray(want[f])
        if creep is None:
            ok &= bool(np.array_equal(a, b))
        else:
            ok &= bool(np.array_equal(a[~creep], b[~creep])) and bool(np.all(a[creep] <= b[creep]))
    return ok, (0 if creep is None else int(creep.sum()))


def parity_report(got, want, width, height, pix=None, rel=1e-9):
    """Per-pixel agreement of a GPU frame `got` with the oracle's `want` on
    the pixels `pix` (all of them by default; `got` holds the whole frame,
    `want` one entry per pixel of `pix`):

      pixels_bit_different     pixels where any of the seven fields differs
                               in its bits (the counters too, when both
                               sides carry them, except on bundle rays
                               stopped while creeping onto the horizon,
                               whose counters only have to be no larger)
      creep_pixels             those rays (status KT_RAY_CREEP)
      class_mismatch           pixels whose outcome differs
      class_mismatch_max_boundary_distance_px
                               the largest distance of such a pixel from a
                               class boundary of the GPU frame (None: none)
      g_rel_gt / r_hit_rel_gt  disk pixels (in both) whose redshift / hit
                               radius differs by more than `rel` relative
      g_rel_max / r_hit_rel_max
    """
    n = width * height
    pix = np.arange(n, dtype=np.int64) if pix is None else np.asarray(pix, np.int64)
    fields = list(GEO_FIELDS) + [f for f in ("steps", "attempts") if f in want and f in got
                                 and want[f] is not None and got[f] is not None]
    differ = np.zeros(len(pix), bool)
    creep = creep_mask(got, pix)
    creep = np.zeros(len(pix), bool) if creep is None else creep
    for f in fields:
        a = np.ascontiguousarray(np.asarray(got[f])[pix])
        b = np.ascontiguousarray(np.asarray(want[f], dtype=a.dtype))
        kind = {1: np.uint8, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize]
        if f in ("steps", "attempts"):
            differ |= np.where(creep, a > b, a.view(kind) != b.view(kind))
        else:
            differ |= a.view(kind) != b.view(kind)
    go, wo = np.asarray(got["outcome"])[pix], np.asarray(want["outcome"])
    cls = go != wo
    disk = (go == 1) & (wo == 1)

    def relerr(f):
        a, b = np.asarray(got[f])[pix][disk], np.asarray(want[f])[disk]
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)

    eg, er = relerr("redshift"), relerr("r")
    return {"pixels": int(len(pix)), "fields": fields,
            "pixels_bit_different": int(differ.sum()), "creep_pixels": int(creep.sum()),
            "class_mismatch": int(cls.sum()),
            "class_mismatch_max_boundary_distance_px": boundary_distance(
                np.asarray(got["outcome"]).reshape(height, width), pix[cls]),
            "disk_pixels": int(disk.sum()),
            "rel_threshold": rel,
            "g_rel_gt": int((eg > rel).sum()), "r_hit_rel_gt": int((er > rel).sum()),
            "g_rel_max": float(eg.max()) if eg.size else 0.0,
            "r_hit_rel_max": float(er.max()) if er.size else 0.0}
