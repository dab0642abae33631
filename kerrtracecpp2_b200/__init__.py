"""kerrtracecpp2_b200 -- B200-native per-pixel null-geodesic renderer.

Python host side over the C ABI of libkerrtrace.so (include/kerrtrace.h).
The functions mirror the reference renderer's frame interface:

  trace_geodesics(W, H, fp, use_bundles, chart, intg, ctl, ...)  main.cpp:2014
  colorize_buffer(geo, W, H, cp, bg, ...)                          main.cpp:1817
  render_image(W, H, fp, bg, use_bundles, chart, intg, ctl, ...)   main.cpp:2209

with the same argument meaning (FrameParams in degrees, IntegratorControls,
pixel offsets, M, Q, Lambda).  Tracing runs on the GPU only: loading the
package without the built library, or tracing without a CUDA device, raises.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import (ColorParams, FrameDerived, FrameDesc, GeoSoA, color_params, frame_desc,
                  KT_CHART_BL, KT_CHART_KS, KT_DOPRI5, KT_RK4_DOUBLING, KT_OK)

__all__ = ["FrameParams", "IntegratorControls", "Renderer", "load_library", "trace_geodesics",
           "colorize_buffer", "render_image", "frame_derive", "starfield", "KerrTraceError",
           "frame_desc", "color_params", "FrameDesc", "ColorParams", "Batch",
           "random_parameter_sets"]

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libkerrtrace.so")
_lib = None


class KerrTraceError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


def load_library():
    """Load the in-tree libkerrtrace.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with python kerrtracecpp2_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    P, D, I32 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int32
    PD = ctypes.POINTER(FrameDesc)
    L.kt_abi_version.restype = ctypes.c_int
    L.kt_status_string.restype = ctypes.c_char_p
    L.kt_status_string.argtypes = [ctypes.c_int]
    L.kt_abi_struct_sizes.argtypes = [ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
    L.kt_abi_struct_sizes.restype = ctypes.c_int
    L.kt_create.argtypes = [ctypes.POINTER(P), ctypes.c_int]
    L.kt_create.restype = ctypes.c_int
    L.kt_destroy.argtypes = [P]
    L.kt_destroy.restype = None
    L.kt_last_error.argtypes = [P]
    L.kt_last_error.restype = ctypes.c_char_p
    L.kt_frame_derive.argtypes = [PD, ctypes.POINTER(FrameDerived)]
    L.kt_frame_derive.restype = ctypes.c_int
    L.kt_frame_desc_defaults.argtypes = [PD]
    L.kt_frame_desc_defaults.restype = None
    L.kt_color_params_defaults.argtypes = [ctypes.POINTER(ColorParams)]
    L.kt_color_params_defaults.restype = None
    L.kt_trace.argtypes = [P, PD, ctypes.POINTER(GeoSoA), P]
    L.kt_trace.restype = ctypes.c_int
    L.kt_trace_pixels.argtypes = [P, PD, P, ctypes.c_int64, ctypes.POINTER(GeoSoA), P]
    L.kt_trace_pixels.restype = ctypes.c_int
    L.kt_trace_noalloc.argtypes = [PD, ctypes.POINTER(GeoSoA), P]
    L.kt_trace_noalloc.restype = ctypes.c_int
    L.kt_trace_host.argtypes = [P, PD, ctypes.POINTER(GeoSoA)]
    L.kt_trace_host.restype = ctypes.c_int
    L.kt_colorize.argtypes = [P, PD, ctypes.POINTER(GeoSoA), ctypes.POINTER(ColorParams), P, I32,
                              I32, P, P]
    L.kt_colorize.restype = ctypes.c_int
    L.kt_render_host.argtypes = [P, PD, ctypes.POINTER(ColorParams), P, I32, I32, P]
    L.kt_render_host.restype = ctypes.c_int
    L.kt_render_spp_host.argtypes = [P, PD, ctypes.POINTER(ColorParams), I32, P, I32, I32, P]
    L.kt_render_spp_host.restype = ctypes.c_int
    L.kt_camera_spp_offsets.argtypes = [I32, P]
    L.kt_camera_spp_offsets.restype = ctypes.c_int
    L.kt_elliptic_reasons.argtypes = [P, PD, P, P]
    L.kt_elliptic_reasons.restype = ctypes.c_int
    L.kt_elliptic_reasons_host.argtypes = [P, PD, P]
    L.kt_elliptic_reasons_host.restype = ctypes.c_int
    L.kt_measure_fp64_peak.argtypes = [P, ctypes.POINTER(D)]
    L.kt_measure_fp64_peak.restype = ctypes.c_int
    L.kt_measure_op_costs.argtypes = [P, ctypes.POINTER(abi.OpCosts)]
    L.kt_measure_op_costs.restype = ctypes.c_int
    L.kt_starfield.argtypes = [ctypes.c_uint64, I32, I32, P]
    L.kt_starfield.restype = ctypes.c_int
    L.kt_kgeo_write.argtypes = [ctypes.c_char_p, PD, ctypes.POINTER(GeoSoA)]
    L.kt_kgeo_write.restype = ctypes.c_int
    L.kt_kgeo_read_header.argtypes = [ctypes.c_char_p, ctypes.POINTER(I32), ctypes.POINTER(I32),
                                      ctypes.POINTER(D)]
    L.kt_kgeo_read_header.restype = ctypes.c_int
    L.kt_kgeo_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(GeoSoA), ctypes.c_int64]
    L.kt_kgeo_read.restype = ctypes.c_int
    PB = ctypes.POINTER(abi.BatchOptions)
    L.kt_batch_options_defaults.argtypes = [PB]
    L.kt_batch_options_defaults.restype = None
    L.kt_batch_create.argtypes = [P, PD, ctypes.POINTER(GeoSoA), I32, PB, ctypes.POINTER(P)]
    L.kt_batch_create.restype = ctypes.c_int
    L.kt_batch_launch.argtypes = [P, P]
    L.kt_batch_launch.restype = ctypes.c_int
    L.kt_batch_group_count.argtypes = [P]
    L.kt_batch_group_count.restype = I32
    L.kt_batch_group.argtypes = [P, I32, ctypes.POINTER(abi.BatchGroupInfo)]
    L.kt_batch_group.restype = ctypes.c_int
    L.kt_batch_rays.argtypes = [P]
    L.kt_batch_rays.restype = ctypes.c_uint64
    L.kt_batch_destroy.argtypes = [P]
    L.kt_batch_destroy.restype = None
    PG = ctypes.POINTER(abi.GradStats)
    PDB = ctypes.POINTER(D)
    L.kt_vjp.argtypes = [P, PD, P, P, ctypes.POINTER(GeoSoA), ctypes.c_uint32, PDB, PG, P]
    L.kt_vjp.restype = ctypes.c_int
    L.kt_l2_grad.argtypes = [P, PD, ctypes.POINTER(GeoSoA), D, D, ctypes.POINTER(GeoSoA),
                             ctypes.c_uint32, PDB, PDB, PG, P]
    L.kt_l2_grad.restype = ctypes.c_int
    L.kt_vjp_pixels.argtypes = [P, PD, P, ctypes.c_int64, P, P, ctypes.POINTER(GeoSoA), ctypes.c_uint32,
                                PDB, PG, P]
    L.kt_vjp_pixels.restype = ctypes.c_int
    L.kt_l2_grad_pixels.argtypes = [P, PD, P, ctypes.c_int64, ctypes.POINTER(GeoSoA), D, D,
                                    ctypes.POINTER(GeoSoA), ctypes.c_uint32, PDB, PDB, PG, P]
    L.kt_l2_grad_pixels.restype = ctypes.c_int
    L.kt_vjp_magnif.argtypes = [P, PD, P, ctypes.c_int64, P, P, P, ctypes.POINTER(GeoSoA),
                                ctypes.c_uint32, PDB, PG, P]
    L.kt_vjp_magnif.restype = ctypes.c_int
    L.kt_l2_grad_magnif.argtypes = [P, PD, P, ctypes.c_int64, ctypes.POINTER(GeoSoA), D, D, D,
                                    ctypes.POINTER(GeoSoA), ctypes.c_uint32, PDB, PDB, PG, P]
    L.kt_l2_grad_magnif.restype = ctypes.c_int
    if L.kt_abi_version() != abi.KT_ABI_VERSION:
        raise ImportError("libkerrtrace.so ABI version mismatch")
    _lib = L
    return L


def _check(status, what, ctx=None):
    if status != KT_OK:
        L = load_library()
        msg = L.kt_last_error(ctx).decode() if ctx else L.kt_status_string(status).decode()
        raise KerrTraceError(status, f"{what}: {msg}")


@dataclass
class FrameParams:
    """FrameParams (main.cpp:1885-1893); angles in degrees."""

    a: float = 0.998
    theta: float = 80.0
    phi: float = 0.0
    r_obs: float = 40.0
    disk_out: float = 12.0
    fov: float = 30.0


@dataclass
class IntegratorControls:
    """IntegratorControls (main.cpp:193-197)."""

    max_steps: int = 500000
    step_init: float = 1.0
    tol: float = 1e-7


def make_desc(W, H, fp, use_bundles=False, chart=KT_CHART_KS, intg=KT_RK4_DOUBLING, ctl=None,
              pixel_offset_x=0.0, pixel_offset_y=0.0, M=1.0, Q=0.0, Lam=0.0,
              solver_mode=abi.KT_SOLVER_STANDARD):
    ctl = ctl or IntegratorControls()
    return frame_desc(M=M, a=fp.a, Q=Q, Lambda=Lam, theta_deg=fp.theta, phi_deg=fp.phi,
                      r_obs=fp.r_obs, disk_out=fp.disk_out, fov_deg=fp.fov, width=W, height=H,
                      pixel_offset_x=pixel_offset_x, pixel_offset_y=pixel_offset_y, chart=chart,
                      integrator=intg, bundles=int(bool(use_bundles)), max_steps=ctl.max_steps,
                      step_init=ctl.step_init, tol=ctl.tol, solver_mode=solver_mode)


def frame_derive(desc):
    """kt_frame_derive: per-frame constants (r_+, ISCO, chart fallback...)."""
    L = load_library()
    out = FrameDerived()
    _check(L.kt_frame_derive(ctypes.byref(desc), ctypes.byref(out)), "kt_frame_derive")
    return out


def starfield(seed=0, w=2048, h=1024):
    """Deterministic procedural equirectangular star field, (h, w, 3) uint8."""
    L = load_library()
    img = np.zeros((h, w, 3), np.uint8)
    _check(L.kt_starfield(seed, w, h, img.ctypes.data_as(ctypes.c_void_p)), "kt_starfield")
    return img


def _np_soa(n, counters=True):
    out = {k: np.zeros(n, dt) for k, dt in abi.GEO_FIELDS}
    if not counters:
        for k in ("status", "steps", "attempts"):
            out[k] = None
    return out


def _soa_struct(arrays, ptr):
    s = GeoSoA()
    for k, _ in abi.GEO_FIELDS:
        a = arrays.get(k)
        setattr(s, k, ptr(a) if a is not None else None)
    return s


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _torch_ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Renderer:
    """One kt_context on one CUDA device."""

    def __init__(self, device=0):
        self.L = load_library()
        self.ctx = ctypes.c_void_p()
        _check(self.L.kt_create(ctypes.byref(self.ctx), device), "kt_create")
        self.device = device

    def close(self):
        if self.ctx:
            self.L.kt_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- device-buffer entry points (torch tensors as device memory) --------
    def alloc(self, n, counters=True):
        import torch

        dev = torch.device("cuda", self.device)
        tdt = {"u1": torch.uint8, "f8": torch.float64, "u4": torch.int32}
        out = {k: torch.empty(n, dtype=tdt[dt], device=dev) for k, dt in abi.GEO_FIELDS}
        if not counters:
            for k in ("status", "steps", "attempts"):
                out[k] = None
        return out

    def trace(self, desc, out=None, stream=None):
        """kt_trace into torch device tensors (allocated if out is None)."""
        n = desc.width * desc.height
        out = out if out is not None else self.alloc(n)
        st = self._stream(stream)
        _check(self.L.kt_trace(self.ctx, ctypes.byref(desc), ctypes.byref(_soa_struct(out, _torch_ptr)),
                               st), "kt_trace", self.ctx)
        return out

    def trace_pixels(self, desc, pix, out=None, stream=None):
        n = int(pix.numel())
        out = out if out is not None else self.alloc(n)
        _check(self.L.kt_trace_pixels(self.ctx, ctypes.byref(desc), _torch_ptr(pix), n,
                                      ctypes.byref(_soa_struct(out, _torch_ptr)), self._stream(stream)),
               "kt_trace_pixels", self.ctx)
        return out

    def colorize(self, desc, geo, cp=None, bg=None, rgb=None, stream=None):
        import torch

        cp = cp or color_params()
        n = desc.width * desc.height
        if rgb is None:
            rgb = torch.empty(n * 3, dtype=torch.uint8, device=torch.device("cuda", self.device))
        bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
        _check(self.L.kt_colorize(self.ctx, ctypes.byref(desc), ctypes.byref(_soa_struct(geo, _torch_ptr)),
                                  ctypes.byref(cp), _torch_ptr(bg) if bg is not None else None, bw, bh,
                                  _torch_ptr(rgb), self._stream(stream)), "kt_colorize", self.ctx)
        return rgb

    @staticmethod
    def _stream(stream):
        if stream is None:
            try:
                import torch

                return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            except Exception:
                return None
        return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))

    def fp64_peak_gflops(self):
        """Measured FP64 FMA throughput of this device (GFLOP/s)."""
        v = ctypes.c_double()
        _check(self.L.kt_measure_fp64_peak(self.ctx, ctypes.byref(v)), "kt_measure_fp64_peak", self.ctx)
        return v.value

    def op_costs(self):
        """kt_measure_op_costs: the measured cost, in flops (2 per FMA), of a
        division, x/3, sqrt, sincos and pow on this device, and the FMA
        throughput of the same probe (GFLOP/s)."""
        v = abi.OpCosts()
        _check(self.L.kt_measure_op_costs(self.ctx, ctypes.byref(v)), "kt_measure_op_costs", self.ctx)
        return {f: getattr(v, f) for f, _ in abi.OpCosts._fields_}

    def vjp(self, desc, cot_redshift=None, cot_r=None, out=None, flags=0, stream=None, pix=None,
            cot_magnif=None):
        """kt_vjp: gradient (numpy, kt_frame_desc units, abi.GRAD_NAMES order)
        of sum(cot_redshift * g + cot_r * r_hit) over the disk pixels of the
        smooth tracer; cotangents are float64 device tensors over the frame.
        With `pix` (an int32 device tensor of pixel indices) only those
        pixels are traced; `cot_magnif` adds a bundle frame's magnification
        (kt_vjp_magnif).  Returns (grad, stats dict)."""
        grad = (ctypes.c_double * abi.KT_GRAD_COUNT)()
        st = abi.GradStats()
        _check(self.L.kt_vjp_magnif(self.ctx, ctypes.byref(desc),
                                    _torch_ptr(pix) if pix is not None else None,
                                    int(pix.numel()) if pix is not None else 0,
                                    _torch_ptr(cot_redshift) if cot_redshift is not None else None,
                                    _torch_ptr(cot_r) if cot_r is not None else None,
                                    _torch_ptr(cot_magnif) if cot_magnif is not None else None,
                                    ctypes.byref(_soa_struct(out, _torch_ptr)) if out is not None else None,
                                    flags, grad, ctypes.byref(st), self._stream(stream)), "kt_vjp", self.ctx)
        return np.array(grad[:]), st.as_dict()

    def l2_grad(self, desc, target, w_g=1.0, w_r=0.0, out=None, flags=0, stream=None, pix=None,
                w_m=0.0):
        """kt_l2_grad: (loss, grad, stats) of the L2 loss of (g, r_hit) against
        a target frame (dict of device tensors from a smooth trace); with `pix`,
        over those pixels only; w_m weighs a bundle frame's magnification
        (kt_l2_grad_magnif)."""
        grad = (ctypes.c_double * abi.KT_GRAD_COUNT)()
        loss = ctypes.c_double()
        st = abi.GradStats()
        _check(self.L.kt_l2_grad_magnif(self.ctx, ctypes.byref(desc),
                                        _torch_ptr(pix) if pix is not None else None,
                                        int(pix.numel()) if pix is not None else 0,
                                        ctypes.byref(_soa_struct(target, _torch_ptr)), w_g, w_r, w_m,
                                        ctypes.byref(_soa_struct(out, _torch_ptr)) if out is not None else None,
                                        flags, ctypes.byref(loss), grad, ctypes.byref(st),
                                        self._stream(stream)),
               "kt_l2_grad", self.ctx)
        return loss.value, np.array(grad[:]), st.as_dict()

    def elliptic_reasons(self, desc, stream=None):
        """kt_elliptic_reasons: the elliptic-closed solver's fallback reason
        per pixel (uint8 tensor, 0 = closed form in the disk)."""
        import torch

        out = torch.empty(desc.width * desc.height, dtype=torch.uint8,
                          device=torch.device("cuda", self.device))
        _check(self.L.kt_elliptic_reasons(self.ctx, ctypes.byref(desc), _torch_ptr(out), self._stream(stream)),
               "kt_elliptic_reasons", self.ctx)
        return out

    def batch(self, descs, outs=None, options=None):
        """kt_batch_create over frames `descs` (a list of kt_frame_desc) with
        device outputs `outs` (one dict of tensors per frame; allocated when
        None).  Returns a Batch; Batch.launch() traces every frame with one
        CUDA graph launch."""
        return Batch(self, descs, outs, options)

    # -- host-buffer entry points --------------------------------------------
    def trace_host(self, desc, counters=True):
        out = _np_soa(desc.width * desc.height, counters)
        _check(self.L.kt_trace_host(self.ctx, ctypes.byref(desc), ctypes.byref(_soa_struct(out, _np_ptr))),
               "kt_trace_host", self.ctx)
        return out

    def render_host(self, desc, cp=None, bg=None, camera_spp=1):
        """render_image: trace + colorize into an (H, W, 3) uint8 image;
        camera_spp > 1 averages that many jittered passes in linear light."""
        cp = cp or color_params()
        rgb = np.zeros((desc.height, desc.width, 3), np.uint8)
        bgc = np.ascontiguousarray(bg) if bg is not None else None
        bw, bh = (bg.shape[1], bg.shape[0]) if bg is not None else (0, 0)
        _check(self.L.kt_render_spp_host(self.ctx, ctypes.byref(desc), ctypes.byref(cp), int(camera_spp),
                                         _np_ptr(bgc) if bgc is not None else None, bw, bh, _np_ptr(rgb)),
               "kt_render_spp_host", self.ctx)
        return rgb


class Batch:
    """A kt_batch: frames traced together by one CUDA graph launch."""

    def __init__(self, renderer, descs, outs=None, options=None):
        self.r = renderer
        self.L = renderer.L
        self.descs = list(descs)
        n = len(self.descs)
        self.outs = outs if outs is not None else [renderer.alloc(d.width * d.height)
                                                   for d in self.descs]
        arr_d = (FrameDesc * n)(*self.descs)
        arr_o = (GeoSoA * n)(*[_soa_struct(o, _torch_ptr) for o in self.outs])
        self.handle = ctypes.c_void_p()
        opt = options if options is not None else abi.batch_options()
        _check(self.L.kt_batch_create(renderer.ctx, arr_d, arr_o, n, ctypes.byref(opt),
                                      ctypes.byref(self.handle)), "kt_batch_create", renderer.ctx)

    @property
    def n_rays(self):
        return int(self.L.kt_batch_rays(self.handle))

    def groups(self):
        out = []
        for i in range(self.L.kt_batch_group_count(self.handle)):
            gi = abi.BatchGroupInfo()
            _check(self.L.kt_batch_group(self.handle, i, ctypes.byref(gi)), "kt_batch_group")
            d = gi.as_dict()
            d["kernel_name"] = abi.BATCH_KERNELS[gi.kernel]
            out.append(d)
        return out

    def launch(self, stream=None):
        _check(self.L.kt_batch_launch(self.handle, Renderer._stream(stream)), "kt_batch_launch",
               self.r.ctx)

    def close(self):
        if self.handle:
            self.L.kt_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_parameter_sets(n=64, seed=1, side_min=256, side_max=1024, lambdas=(0.0, 1e-4)):
    """Seeded random frames for batch rendering: a ~ U[0, 0.998], Q ~ U[0, 0.4]
    redrawn until a^2 + Q^2 < 1, Lambda drawn from `lambdas`, theta_obs ~
    U[5, 89] degrees, r_obs ~ U[20, 200], square frames of side ~ U{side_min
    .. side_max} (multiples of 16); KS chart, RK4 step doubling and the CLI's
    other defaults.  Returns a list of kt_frame_desc."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        a = rng.uniform(0.0, 0.998)
        q = rng.uniform(0.0, 0.4)
        while a * a + q * q >= 1.0:
            q = rng.uniform(0.0, 0.4)
        lam = float(lambdas[int(rng.integers(len(lambdas)))])
        th = rng.uniform(5.0, 89.0)
        r_obs = rng.uniform(20.0, 200.0)
        side = int(rng.integers(side_min // 16, side_max // 16 + 1)) * 16
        out.append(frame_desc(a=a, Q=q, Lambda=lam, theta_deg=th, r_obs=r_obs, width=side,
                              height=side, chart=KT_CHART_KS, integrator=KT_RK4_DOUBLING))
    return out


_default = {}


def _renderer(device=0):
    if device not in _default:
        _default[device] = Renderer(device)
    return _default[device]


def trace_geodesics(W, H, fp, use_bundles=False, chart=KT_CHART_KS, intg=KT_RK4_DOUBLING, ctl=None,
                    pixel_offset_x=0.0, pixel_offset_y=0.0, M_bh=1.0, Q_bh=0.0, Lam=0.0, device=0,
                    solver_mode=abi.KT_SOLVER_STANDARD):
    """Phase 1 (main.cpp:2014): per-pixel results as float64 numpy arrays;
    solver_mode as the reference's RaySolverMode (main.cpp:176)."""
    desc = make_desc(W, H, fp, use_bundles, chart, intg, ctl, pixel_offset_x, pixel_offset_y, M_bh,
                     Q_bh, Lam, solver_mode)
    return _renderer(device).trace_host(desc)


def render_image(W, H, fp, bg=None, use_bundles=False, chart=KT_CHART_KS, intg=KT_RK4_DOUBLING,
                 ctl=None, M_bh=1.0, Q_bh=0.0, Lam=0.0, cp=None, pixel_offset_x=0.0,
                 pixel_offset_y=0.0, device=0, camera_spp=1, solver_mode=abi.KT_SOLVER_STANDARD):
    """render_image (main.cpp:2209): trace + colorize; (H, W, 3) uint8.
    camera_spp > 1 renders that many jittered passes and averages them in
    linear light (main.cpp:2232-2322)."""
    desc = make_desc(W, H, fp, use_bundles, chart, intg, ctl, pixel_offset_x, pixel_offset_y, M_bh,
                     Q_bh, Lam, solver_mode)
    return _renderer(device).render_host(desc, cp, bg, camera_spp)


def camera_spp_offsets(camera_spp):
    """kt_camera_spp_offsets: the (spp, 2) pixel jitter of each pass."""
    L = load_library()
    n = max(int(camera_spp), 1)
    xy = np.zeros((n, 2), np.float64)
    _check(L.kt_camera_spp_offsets(int(camera_spp), _np_ptr(xy)), "kt_camera_spp_offsets")
    return xy


def colorize_buffer(geo, desc, cp=None, bg=None, device=0):
    """colorize_buffer (main.cpp:1817) of host results from trace_geodesics."""
    import torch

    r = _renderer(device)
    dev = torch.device("cuda", device)
    g = {k: (torch.from_numpy(np.ascontiguousarray(v)).to(dev) if v is not None else None)
         for k, v in geo.items()}
    bgt = torch.from_numpy(np.ascontiguousarray(bg)).to(dev) if bg is not None else None
    rgb = r.colorize(desc, g, cp, bgt)
    torch.cuda.synchronize(dev)
    return rgb.cpu().numpy().reshape(desc.height, desc.width, 3)
