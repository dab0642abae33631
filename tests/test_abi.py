"""The C ABI library without a GPU: it loads, exports every entry point the
headers declare, its structs match the ctypes mirror, the host-side frame
derivation equals the reference's, .kgeo files are byte-compatible with the
reference's GeoPixel records, and argument errors come back as status codes."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
import kerrtracecpp2_b200 as kt
from kerrtracecpp2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    return kt.load_library()


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kt_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    syms = subprocess.run(["nm", "-D", "--defined-only", kt.LIB_PATH], capture_output=True,
                          text=True, check=True).stdout
    exported = set(re.findall(r" T (\S+)", syms))
    missing = [s for s in declared("kerrtrace.h") if s not in exported]
    assert not missing, missing
    # cuda_render with the reference's C++ signature (gpu/cuda/tracer.cuh:23-26)
    assert "_Z11cuda_renderRK15KNdSParams_CUDARK17CameraParams_CUDAb" in exported


def test_struct_layout(L):
    sizes = (ctypes.c_size_t * 6)()
    assert L.kt_abi_struct_sizes(sizes, 6) == 6
    assert list(sizes) == [ctypes.sizeof(abi.FrameDesc), ctypes.sizeof(abi.FrameDerived),
                           ctypes.sizeof(abi.GeoSoA), ctypes.sizeof(abi.ColorParams),
                           ctypes.sizeof(abi.BatchOptions), ctypes.sizeof(abi.BatchGroupInfo)]


def test_batch_options_defaults(L):
    o = abi.BatchOptions()
    L.kt_batch_options_defaults(ctypes.byref(o))
    ref = abi.batch_options()
    assert [getattr(o, f) for f, _ in o._fields_] == [getattr(ref, f) for f, _ in ref._fields_]


def test_batch_entry_points_reject_null(L):
    d = abi.frame_desc(width=4, height=4)
    h = ctypes.c_void_p()
    assert L.kt_batch_create(None, ctypes.byref(d), None, 1, None, ctypes.byref(h)) == \
        abi.KT_ERR_INVALID_ARGUMENT
    assert L.kt_batch_launch(None, None) == abi.KT_ERR_INVALID_ARGUMENT
    assert L.kt_batch_group_count(None) == 0 and L.kt_batch_rays(None) == 0
    gi = abi.BatchGroupInfo()
    assert L.kt_batch_group(None, 0, ctypes.byref(gi)) == abi.KT_ERR_INVALID_ARGUMENT
    L.kt_batch_destroy(None)


def test_random_parameter_sets():
    a = kt.random_parameter_sets(64, seed=1)
    b = kt.random_parameter_sets(64, seed=1)
    assert [bytes(x) for x in a] == [bytes(x) for x in b]
    assert len(a) == 64
    for d in a:
        assert 0 <= d.a <= 0.998 and 0 <= d.Q <= 0.4 and d.a ** 2 + d.Q ** 2 < 1
        assert d.Lambda in (0.0, 1e-4) and 5 <= d.theta_deg <= 89 and 20 <= d.r_obs <= 200
        assert d.width == d.height and 256 <= d.width <= 1024 and d.width % 16 == 0
        assert d.chart == abi.KT_CHART_KS and d.integrator == abi.KT_RK4_DOUBLING


def test_defaults_match_reference_cli(L):
    d = abi.FrameDesc()
    L.kt_frame_desc_defaults(ctypes.byref(d))
    ref = abi.frame_desc()
    for name, _ in abi.FrameDesc._fields_:
        assert getattr(d, name) == getattr(ref, name), name


def test_frame_derive_radii_match_reference():
    for M, a, Q, Lam, rh, ri in G.data()["kat/radii"]:
        dv = kt.frame_derive(abi.frame_desc(M=M, a=a, Q=Q, Lambda=Lam, chart=1, width=4, height=4))
        assert dv.r_horizon == rh and dv.r_isco == ri


def test_frame_derive_radii_match_reference_random_metrics():
    """Horizon and ISCO of random (M, a, Q, Lambda), both signs of Lambda,
    against the strict reference build's own r_horizon and r_isco (the
    scan's samples are evaluated on several threads here)."""
    if not O.ref_available("strict"):
        pytest.skip("reference build missing")
    ref = O.ref("strict")
    rng = np.random.default_rng(17)
    for _ in range(40):
        M = float(rng.uniform(0.5, 2.0))
        a = float(rng.uniform(-0.99, 0.99)) * M
        Q = float(rng.uniform(0.0, 0.9)) * M * np.sqrt(max(0.0, 1.0 - (a / M) ** 2))
        Lam = float(rng.choice([0.0, 1e-4, 3e-3, -2e-4, -1e-3])) / (M * M)
        dv = kt.frame_derive(abi.frame_desc(M=M, a=a, Q=Q, Lambda=Lam, chart=1, width=4, height=4))
        assert dv.r_horizon == ref.ref_r_horizon(M, a, Q, Lam), (M, a, Q, Lam)
        assert dv.r_isco == ref.ref_r_isco(M, a, Q, Lam), (M, a, Q, Lam)


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_frame_derive_in_forked_child():
    """The frame set-up's threaded sampling after fork(): a child of a
    process that has used it derives the same radii (serially) and exits."""
    import time

    d = abi.frame_desc(chart=1, a=0.9, Q=0.3, Lambda=1e-4, width=4, height=4)
    want = kt.frame_derive(d)
    r, w = os.pipe()
    pid = os.fork()
    if pid == 0:  # child: no pytest machinery, report through the pipe
        try:
            dv = kt.frame_derive(d)
            os.write(w, f"{dv.r_horizon!r} {dv.r_isco!r}".encode())
        finally:
            os._exit(0)
    os.close(w)
    deadline = time.time() + 60
    while time.time() < deadline:
        done, _ = os.waitpid(pid, os.WNOHANG)
        if done:
            break
        time.sleep(0.05)
    else:
        os.kill(pid, 9)
        os.waitpid(pid, 0)
        pytest.fail("frame set-up in a forked child did not finish")
    got = os.read(r, 200).decode().split()
    os.close(r)
    assert [float(x) for x in got] == [want.r_horizon, want.r_isco]


@pytest.mark.parametrize("name", sorted(G.cases()))
def test_frame_derive_matches_oracle(name):
    d = G.desc(name)
    got, want = kt.frame_derive(d), O.derive_port(d)
    for f, _ in abi.FrameDerived._fields_:
        assert getattr(got, f) == getattr(want, f), f


def test_fallback_rules():
    # KS + Lambda != 0 -> BL; bundles -> BL; KS ignores DOPRI5 (main.cpp:2033-2049, 1539-1545)
    assert kt.frame_derive(abi.frame_desc(chart=0, Lambda=1e-4, width=2, height=2)).chart == 1
    assert kt.frame_derive(abi.frame_desc(chart=0, bundles=1, width=2, height=2)).chart == 1
    dv = kt.frame_derive(abi.frame_desc(chart=0, integrator=1, width=2, height=2))
    assert dv.chart == 0 and dv.integrator == 0


@pytest.mark.parametrize("kw,status", [
    (dict(width=0), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(height=-3), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(width=70000, height=70000), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(a=float("nan")), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(tol=float("inf")), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(chart=7), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED, precision=abi.KT_PREC_MIXED), abi.KT_ERR_UNSUPPORTED),
    (dict(solver_mode=9), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(precision=7), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED, precision=abi.KT_PREC_SMOOTH), abi.KT_ERR_UNSUPPORTED),
    (dict(r_obs=-1.0), abi.KT_ERR_INVALID_ARGUMENT),
    (dict(flags=8), abi.KT_ERR_INVALID_ARGUMENT),
])
def test_invalid_frames_return_status(L, kw, status):
    d = abi.frame_desc(**kw)
    out = abi.FrameDerived()
    assert L.kt_frame_derive(ctypes.byref(d), ctypes.byref(out)) == status


def test_no_device_is_an_error_not_a_fallback(L):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = ctypes.c_void_p()
    assert L.kt_create(ctypes.byref(ctx), 0) == abi.KT_ERR_NO_DEVICE
    assert not ctx.value
    with pytest.raises(kt.KerrTraceError):
        kt.Renderer(0)
    # trace calls on a NULL context fail cleanly
    d = abi.frame_desc(width=4, height=4)
    assert L.kt_trace(None, ctypes.byref(d), None, None) == abi.KT_ERR_INVALID_ARGUMENT


def _soa(res, ptr=lambda a: a.ctypes.data_as(ctypes.c_void_p)):
    s = abi.GeoSoA()
    for k in G.FIELDS:
        setattr(s, k, ptr(res[k]))
    return s


@pytest.mark.parametrize("name", ["cfg1_ks_rk4", "cfg3_bundles", "offsets"])
def test_kgeo_bytes_match_reference_records(L, tmp_path, name):
    """kt_kgeo_write writes the reference's GeoPixel records byte for byte
    (main.cpp:84-137) and kt_kgeo_read reads them back."""
    d = G.desc(name)
    res = {k: np.ascontiguousarray(v) for k, v in G.result(name).items()}
    path = str(tmp_path / "f.kgeo").encode()
    assert L.kt_kgeo_write(path, ctypes.byref(d), ctypes.byref(_soa(res))) == 0
    raw = open(path, "rb").read()
    n = d.width * d.height
    assert len(raw) == 8 + 88 + 28 * n and raw[:4] == b"KGEO"
    assert np.frombuffer(raw[4:8], "<u4")[0] == 1
    W, H = np.frombuffer(raw[8:16], "<u4")
    meta = np.frombuffer(raw[16:96], "<f8")
    assert (W, H) == (d.width, d.height)
    dv = kt.frame_derive(d)
    assert list(meta) == [d.M, d.a, d.Q, d.Lambda, dv.r_isco, dv.r_isco, d.disk_out, d.theta_deg,
                          d.phi_deg, d.r_obs]
    recs = np.frombuffer(raw[96:], O.GEOPIXEL_DTYPE)
    assert recs.tobytes() == G.data()[f"{name}/geopixels"].tobytes()
    w, h = ctypes.c_int32(), ctypes.c_int32()
    m10 = (ctypes.c_double * 10)()
    assert L.kt_kgeo_read_header(path, ctypes.byref(w), ctypes.byref(h), m10) == 0
    back = {k: np.zeros(n, dtype=v.dtype) for k, v in res.items()}
    assert L.kt_kgeo_read(path, ctypes.byref(_soa(back)), n) == 0
    for k in G.FIELDS:
        want = res[k].astype(np.float32).astype(np.float64) if k != "outcome" else res[k]
        assert np.array_equal(back[k], want), k
    assert L.kt_kgeo_read(path, ctypes.byref(_soa(back)), n - 1) == abi.KT_ERR_INVALID_ARGUMENT


def test_kgeo_rejects_bad_files(L, tmp_path):
    p = tmp_path / "bad.kgeo"
    p.write_bytes(b"KGEX" + b"\0" * 100)
    w, h = ctypes.c_int32(), ctypes.c_int32()
    assert L.kt_kgeo_read_header(str(p).encode(), ctypes.byref(w), ctypes.byref(h), None) == abi.KT_ERR_IO
    p.write_bytes(b"KGEO" + b"\1\0\0\0" + b"\0" * 10)  # truncated meta
    assert L.kt_kgeo_read_header(str(p).encode(), ctypes.byref(w), ctypes.byref(h), None) == abi.KT_ERR_IO
    assert L.kt_kgeo_read_header(str(tmp_path / "none").encode(), ctypes.byref(w), ctypes.byref(h),
                                 None) == abi.KT_ERR_IO


def test_starfield_deterministic():
    a = kt.starfield(0, 256, 128)
    b = kt.starfield(0, 256, 128)
    c = kt.starfield(1, 256, 128)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.shape == (128, 256, 3) and a.max() > 80 and np.median(a) < 40
    assert np.array_equal(kt.starfield(0, 512, 256), G.data()["bg"])
