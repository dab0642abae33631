"""ctypes mirror of include/kerrtrace.h (the renderer's C ABI).

The structures here must match the header field for field; the CPU test
suite checks their sizes against the library's own `kt_abi_sizes`.
"""
import ctypes

KT_ABI_VERSION = 1

KT_OK = 0
KT_ERR_INVALID_ARGUMENT = 1
KT_ERR_UNSUPPORTED = 2
KT_ERR_CUDA = 3
KT_ERR_OUT_OF_MEMORY = 4
KT_ERR_NO_DEVICE = 5
KT_ERR_IO = 6
KT_ERR_INTERNAL = 7

KT_CHART_KS = 0
KT_CHART_BL = 1
KT_RK4_DOUBLING = 0
KT_DOPRI5 = 1
KT_SOLVER_STANDARD = 0
KT_SOLVER_SEMI_ANALYTIC = 1
KT_SOLVER_ELLIPTIC_CLOSED = 2
KT_PREC_FP64 = 0
KT_PREC_MIXED = 1
KT_PREC_SMOOTH = 2
KT_PALETTE_BLACKBODY = 0
KT_PALETTE_INTERSTELLAR = 1
KT_MAX_CAMERA_SPP = 256
KT_OUT_ESCAPED = 0
KT_OUT_DISK = 1
KT_OUT_HORIZON = 2
KT_RAY_EVENT = 0
KT_RAY_STEP_CAP = 1
KT_RAY_REJECT_CAP = 2
KT_RAY_NONFINITE = 3
KT_RAY_CREEP = 4
KT_FLAG_ANGLES_RADIANS = 1
KT_FLAG_BUNDLE_FULL_CREEP = 2


class FrameDesc(ctypes.Structure):
    """kt_frame_desc: FrameParams + IntegratorControls + dispatch arguments."""

    _fields_ = [
        ("M", ctypes.c_double), ("a", ctypes.c_double), ("Q", ctypes.c_double),
        ("Lambda", ctypes.c_double),
        ("theta_deg", ctypes.c_double), ("phi_deg", ctypes.c_double), ("r_obs", ctypes.c_double),
        ("disk_out", ctypes.c_double), ("fov_deg", ctypes.c_double),
        ("width", ctypes.c_int32), ("height", ctypes.c_int32),
        ("pixel_offset_x", ctypes.c_double), ("pixel_offset_y", ctypes.c_double),
        ("chart", ctypes.c_int32), ("integrator", ctypes.c_int32), ("bundles", ctypes.c_int32),
        ("solver_mode", ctypes.c_int32),
        ("max_steps", ctypes.c_int32), ("precision", ctypes.c_int32),
        ("step_init", ctypes.c_double), ("tol", ctypes.c_double),
        ("flags", ctypes.c_uint32), ("reserved0", ctypes.c_int32),
    ]


class FrameDerived(ctypes.Structure):
    _fields_ = [
        ("chart", ctypes.c_int32), ("integrator", ctypes.c_int32),
        ("r_horizon", ctypes.c_double), ("rh_cut", ctypes.c_double), ("r_isco", ctypes.c_double),
        ("r_disk_in", ctypes.c_double), ("r_disk_out", ctypes.c_double),
        ("r_escape", ctypes.c_double),
        ("r_obs", ctypes.c_double), ("theta_obs", ctypes.c_double), ("phi_obs", ctypes.c_double),
        ("fov_h", ctypes.c_double),
        ("dlam0", ctypes.c_double), ("max_steps", ctypes.c_int32), ("solver", ctypes.c_int32),
        ("tol", ctypes.c_double), ("bundle_eps", ctypes.c_double), ("r_fp32", ctypes.c_double),
    ]


class GeoSoA(ctypes.Structure):
    """kt_geo_soa: per-pixel result arrays (device or host pointers)."""

    _fields_ = [
        ("outcome", ctypes.c_void_p), ("r", ctypes.c_void_p), ("redshift", ctypes.c_void_p),
        ("magnif", ctypes.c_void_p), ("phi_disk", ctypes.c_void_p),
        ("theta_esc", ctypes.c_void_p), ("phi_esc", ctypes.c_void_p),
        ("status", ctypes.c_void_p), ("steps", ctypes.c_void_p), ("attempts", ctypes.c_void_p),
    ]


class ColorParams(ctypes.Structure):
    _fields_ = [
        ("exposure", ctypes.c_double), ("gamma", ctypes.c_double),
        ("temp_scale", ctypes.c_double), ("palette", ctypes.c_int32),
        ("reserved0", ctypes.c_int32), ("disk_rings", ctypes.c_int32),
        ("disk_sectors", ctypes.c_int32), ("disk_sigma", ctypes.c_double),
        ("disk_hue_offset", ctypes.c_double),
    ]


KT_BATCH_VARIANTS = 4
KT_BATCH_AUTOTUNE = 1


class BatchOptions(ctypes.Structure):
    _fields_ = [
        ("flags", ctypes.c_uint32), ("variant", ctypes.c_int32), ("refill_min", ctypes.c_int32),
        ("tune_reps", ctypes.c_int32), ("tune_fraction", ctypes.c_double),
    ]


class BatchGroupInfo(ctypes.Structure):
    _fields_ = [
        ("kernel", ctypes.c_int32), ("n_frames", ctypes.c_int32), ("n_rays", ctypes.c_uint64),
        ("variant", ctypes.c_int32), ("block", ctypes.c_int32), ("min_blocks", ctypes.c_int32),
        ("grid", ctypes.c_int32), ("refill_min", ctypes.c_int32), ("rays_per_warp", ctypes.c_int32),
        ("tuned", ctypes.c_int32), ("candidates", ctypes.c_int32),
        ("sample_rays", ctypes.c_double), ("best_ms", ctypes.c_double),
        ("default_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# Kernel of a batch group (kt_batch_group_info.kernel).
BATCH_KERNELS = ["bl_rk4", "bl_dopri5", "ks_rk4", "bundles", "bl_rk4_mixed", "bl_dopri5_mixed",
                 "ks_rk4_mixed", "bundles_mixed", "separable_kerr"]


def batch_options(autotune=False, **kw):
    """kt_batch_options with the library's defaults (per-mode variant,
    refill as soon as one lane is idle, 2 timed repetitions, 1/16 sample)."""
    o = BatchOptions()
    o.flags = KT_BATCH_AUTOTUNE if autotune else 0
    o.variant, o.refill_min, o.tune_reps, o.tune_fraction = -1, 0, 2, 1.0 / 16.0
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(f"kt_batch_options has no field {k!r}")
        setattr(o, k, v)
    return o


# Gradient entries (kt_vjp / kt_l2_grad), in kt_frame_desc units.
GRAD_NAMES = ["a", "Q", "Lambda", "theta_deg", "r_obs", "disk_out"]
KT_GRAD_COUNT = 6
KT_GRAD_SKIP_LAMBDA = 1


class GradStats(ctypes.Structure):
    _fields_ = [
        ("loss", ctypes.c_double), ("grad_pixels", ctypes.c_int64), ("bl_pixels", ctypes.c_int64),
        ("unrecorded", ctypes.c_int64), ("ms_main", ctypes.c_float), ("ms_lambda", ctypes.c_float),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OpCosts(ctypes.Structure):
    """kt_op_costs: measured flops (2 per FMA) of one operation."""
    _fields_ = [
        ("fma_gflops", ctypes.c_double), ("div", ctypes.c_double), ("div3", ctypes.c_double),
        ("sqrt", ctypes.c_double), ("sincos", ctypes.c_double), ("pow", ctypes.c_double),
    ]


# Result arrays of one frame: name -> numpy dtype, in kt_geo_soa order.
GEO_FIELDS = [
    ("outcome", "u1"), ("r", "f8"), ("redshift", "f8"), ("magnif", "f8"), ("phi_disk", "f8"),
    ("theta_esc", "f8"), ("phi_esc", "f8"), ("status", "u1"), ("steps", "u4"),
    ("attempts", "u4"),
]


def frame_desc(**kw):
    """A kt_frame_desc with the reference CLI's defaults (main.cpp:2505-2517,
    2709-2716): KS chart, RK4 doubling, tol 1e-7, step_init 1, max_steps
    500000, a=0.998, theta=80, phi=0, r_obs=40, fov=30, disk_out=12,
    1920x1080, M=1, Q=0, Lambda=0.  Keyword arguments override fields."""
    d = FrameDesc()
    d.M, d.a, d.Q, d.Lambda = 1.0, 0.998, 0.0, 0.0
    d.theta_deg, d.phi_deg, d.r_obs, d.disk_out, d.fov_deg = 80.0, 0.0, 40.0, 12.0, 30.0
    d.width, d.height = 1920, 1080
    d.pixel_offset_x = d.pixel_offset_y = 0.0
    d.chart, d.integrator, d.bundles, d.solver_mode = KT_CHART_KS, KT_RK4_DOUBLING, 0, 0
    d.max_steps, d.precision = 500000, KT_PREC_FP64
    d.step_init, d.tol = 1.0, 1e-7
    d.flags = 0
    for k, v in kw.items():
        if not hasattr(d, k):
            raise KeyError(f"kt_frame_desc has no field {k!r}")
        setattr(d, k, v)
    return d


def color_params(**kw):
    """ColorParams defaults (main.cpp:72-81): exposure 1, gamma 2.2, temp_scale 1,
    blackbody palette; interstellar palette 7 rings x 14 sectors, sigma 0.5,
    hue offset 0."""
    c = ColorParams()
    c.exposure, c.gamma, c.temp_scale, c.palette = 1.0, 2.2, 1.0, 0
    c.disk_rings, c.disk_sectors, c.disk_sigma, c.disk_hue_offset = 7, 14, 0.5, 0.0
    for k, v in kw.items():
        setattr(c, k, v)
    return c
