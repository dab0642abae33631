"""GPU parity: the CUDA kernels against the reference renderer (golden
fixtures made from its own code) and the oracle, bit for bit, through the
C ABI.  Full-size frames are compared with the oracle pixel for pixel:
config 2 (720p) and config 5 (512x512) whole, config 3 (1080p bundles) on
every 16th pixel."""
import numpy as np
import pytest

import golden_lib as G
import oracle_lib as O
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu


def to_np(out):
    return {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}


def trace(renderer, d):
    import torch

    out = renderer.trace(d)
    torch.cuda.synchronize()
    got = to_np(out)
    got["steps"] = got["steps"].view(np.uint32)
    got["attempts"] = got["attempts"].view(np.uint32)
    return got


@pytest.mark.parametrize("name", sorted(G.cases()))
def test_kernel_matches_reference_fixtures(renderer, name):
    got = trace(renderer, G.desc(name))
    assert G.mismatches(got, G.result(name)) == {k: 0 for k in G.FIELDS}


@pytest.mark.parametrize("kw", [
    dict(chart=0, a=0.5, width=320, height=180, r_obs=40.0, theta_deg=80.0, fov_deg=45.0,
         disk_out=12.0),                                                        # config 1, full
    dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
         fov_deg=30.0, disk_out=20.0, width=160, height=90),                    # config 2 at 1/64
    dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=96, height=54),    # config 3 at 1/400
    dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=128,
         height=128),                                                           # config 5 at 1/16
], ids=["cfg1_full", "cfg2_160x90", "cfg3_96x54", "cfg5_128"])
def test_kernel_matches_oracle_medium(renderer, kw):
    """Every field bit-identical to the oracle; the step and attempt counters
    too, except on bundle rays stopped while creeping onto the horizon
    (status KT_RAY_CREEP), whose counters stop early."""
    d = abi.frame_desc(**kw)
    got = trace(renderer, d)
    want = O.trace_port(d, counters=True)
    assert G.mismatches(got, want) == {k: 0 for k in G.FIELDS}
    ok, creeping = O.counters_agree(got, want)
    assert ok
    assert (creeping > 0) == bool(kw.get("bundles"))


def test_bundle_full_creep_counters_match_oracle(renderer):
    """With KT_FLAG_BUNDLE_FULL_CREEP the bundle rays creeping onto the
    horizon are traced on to the reference's reject or step cap: config 3's
    geometry at 96x54, records and counters bit-identical to the oracle, and
    the records equal to the default trace's (which stops those rays early)."""
    kw = dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=96, height=54)
    d = abi.frame_desc(flags=abi.KT_FLAG_BUNDLE_FULL_CREEP, **kw)
    got = trace(renderer, d)
    want = O.trace_port(d, counters=True)
    assert G.mismatches(got, want) == {k: 0 for k in G.FIELDS}
    assert np.array_equal(got["steps"], want["steps"])
    assert np.array_equal(got["attempts"], want["attempts"])
    assert not np.any(got["status"] == abi.KT_RAY_CREEP)
    early = trace(renderer, abi.frame_desc(**kw))
    assert G.mismatches(early, got) == {k: 0 for k in G.FIELDS}
    assert np.any(early["status"] == abi.KT_RAY_CREEP)


@pytest.mark.parametrize("kw", [
    dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=960, height=540),   # config 3, 1/4
    # closer to the equator: rays that creep to the step cap, capped at 20000
    dict(chart=1, bundles=1, a=0.9, Q=0.2, Lambda=1e-5, theta_deg=70.0, width=480, height=270,
         max_steps=20000),
], ids=["cfg3_960x540", "knds_480x270"])
def test_bundle_creep_end_keeps_every_record(renderer, kw):
    """Whole bundle frames traced with and without KT_FLAG_BUNDLE_FULL_CREEP:
    every record bit-identical; the rays stopped early carry status
    KT_RAY_CREEP and no more steps or attempts than the full trace."""
    full = trace(renderer, abi.frame_desc(flags=abi.KT_FLAG_BUNDLE_FULL_CREEP, **kw))
    early = trace(renderer, abi.frame_desc(**kw))
    assert G.mismatches(early, full) == {k: 0 for k in G.FIELDS}
    creep = early["status"] == abi.KT_RAY_CREEP
    print(f"{int(creep.sum())} of {creep.size} rays stopped creeping; attempts "
          f"{int(early['attempts'].astype(np.int64).sum())} against {int(full['attempts'].astype(np.int64).sum())}")
    assert creep.any()
    assert np.all(early["steps"][creep] <= full["steps"][creep])
    assert np.all(early["attempts"][creep] <= full["attempts"][creep])
    for f in ("steps", "attempts", "status"):
        assert np.array_equal(early[f][~creep], full[f][~creep]), f


CFG2_720P = dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                 theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=1280, height=720)


def test_full_720p_frame_against_oracle(renderer):
    """Config 2 at full size (1280x720 KNdS, BL, DOPRI5 tol 1e-10), every
    one of the 921,600 pixels: the seven per-pixel fields and the step and
    attempt counters bit-identical to the oracle, so no pixel's g or hit
    radius differs by more than 1e-9 and no pixel changes class.  Also
    deterministic across two launches, with valid ranges."""
    d = abi.frame_desc(**CFG2_720P)
    a = trace(renderer, d)
    b = trace(renderer, d)
    assert G.mismatches(a, b, list(G.FIELDS) + ["steps", "attempts"]) == \
        {k: 0 for k in list(G.FIELDS) + ["steps", "attempts"]}
    disk = a["outcome"] == 1
    assert disk.any() and (a["outcome"] == 2).any() and (a["outcome"] == 0).any()
    assert np.all((a["redshift"][disk] >= 0) & (a["redshift"][disk] <= 20))
    assert np.all((a["r"][disk] >= 1.0) & (a["r"][disk] <= 20.0))
    want = O.trace_port(d, counters=True)
    rep = O.parity_report(a, want, d.width, d.height)
    print(rep)
    assert rep["pixels"] == 921600 and rep["disk_pixels"] > 0
    assert rep["pixels_bit_different"] == 0
    assert rep["class_mismatch"] == 0 and rep["g_rel_gt"] == 0 and rep["r_hit_rel_gt"] == 0


@pytest.mark.parametrize("kw,stride", [
    (dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=512,
          height=512), 1),                                                       # config 5, whole
    (dict(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=1920, height=1080), 16),  # config 3
], ids=["cfg5_512_full", "cfg3_1080p_stride16"])
def test_full_size_frames_against_oracle(renderer, kw, stride):
    """Config 5 at full size, every pixel, and config 3 (Jacobi bundles) at
    full size on every 16th pixel (129,600 bundle rays): all fields and the
    counters bit-identical to the oracle (on bundle rays stopped while
    creeping onto the horizon, counters no larger)."""
    d = abi.frame_desc(**kw)
    a = trace(renderer, d)
    pix = np.arange(0, d.width * d.height, stride, dtype=np.uint32)
    want = O.trace_port(d, pix=None if stride == 1 else pix, counters=True)
    rep = O.parity_report(a, want, d.width, d.height, pix=pix)
    print(rep)
    assert rep["pixels_bit_different"] == 0 and rep["class_mismatch"] == 0
    assert rep["g_rel_gt"] == 0 and rep["r_hit_rel_gt"] == 0


def test_trace_pixels_equals_frame(renderer):
    import torch

    d = G.desc("cfg5_ks")
    full = trace(renderer, d)
    pix = np.array([5, 0, 2303, 17, 1000, 1001, 999], np.uint32)
    out = renderer.trace_pixels(d, torch.from_numpy(pix.astype(np.int32)).cuda())
    torch.cuda.synchronize()
    sub = to_np(out)
    for k in G.FIELDS:
        assert np.array_equal(G.bits(sub[k]), G.bits(full[k][pix])), k


def test_trace_host_equals_device(renderer):
    d = G.desc("cfg2_bl_dopri5")
    dev = trace(renderer, d)
    host = renderer.trace_host(d)
    assert G.mismatches(host, dev) == {k: 0 for k in G.FIELDS}


@pytest.mark.parametrize("case", ["cfg1_ks_rk4", "cfg2_bl_dopri5", "elliptic", "partly_pinned"])
def test_trace_host_into_pinned_buffers(renderer, case):
    """kt_trace_host with page-locked host buffers (the kernels write into
    them directly) gives the records of the pageable-buffer call (device
    staging and copies): a KS frame with its BL fallback launch, the DOPRI5
    frame, an elliptic-solver frame (whose closed-form kernel reads and
    rewrites the records), and buffers of which only some are page-locked."""
    import ctypes

    import torch

    import kerrtracecpp2_b200 as kt

    if case == "elliptic":
        d = abi.frame_desc(chart=abi.KT_CHART_KS, a=0.5, width=96, height=54, fov_deg=45.0,
                           solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED)
    else:
        d = G.desc("cfg2_bl_dopri5" if case == "partly_pinned" else case)
    n = d.width * d.height
    ref = renderer.trace_host(d)
    pinned = {k: torch.zeros(n, dtype=getattr(torch, {"u1": "uint8", "u4": "int32", "f8": "float64"}[dt]),
                             pin_memory=True).numpy() for k, dt in abi.GEO_FIELDS}
    if case == "partly_pinned":
        pinned["phi_esc"] = np.zeros(n)
    st = renderer.L.kt_trace_host(renderer.ctx, ctypes.byref(d),
                                  ctypes.byref(kt._soa_struct(pinned, kt._np_ptr)))
    assert st == 0
    for k, dt in abi.GEO_FIELDS:
        got = pinned[k].view(np.uint32) if dt == "u4" else pinned[k]
        assert np.array_equal(G.bits(got), G.bits(ref[k])), k


@pytest.mark.parametrize("name", ["cfg1_ks_rk4", "cfg2_bl_dopri5", "cfg3_bundles", "cfg5_ks",
                                  "seven_by_three", "retrograde", "ads_lambda", "offsets"])
def test_render_matches_reference_colour(renderer, name):
    z = G.data()
    d = G.desc(name)
    rgb = renderer.render_host(d, bg=z["bg"])
    assert np.array_equal(rgb.reshape(-1, 3), z[f"{name}/rgb"])


def test_colorize_device_entry(renderer):
    import torch

    z = G.data()
    d = G.desc("cfg1_ks_rk4")
    out = renderer.trace(d)
    bg = torch.from_numpy(np.ascontiguousarray(z["bg"])).cuda()
    rgb = renderer.colorize(d, out, bg=bg)
    torch.cuda.synchronize()
    assert np.array_equal(rgb.cpu().numpy().reshape(-1, 3), z["cfg1_ks_rk4/rgb"])


def test_status_and_counters(renderer):
    got = trace(renderer, G.desc("step_cap"))
    assert np.all(got["status"] == abi.KT_RAY_STEP_CAP) and np.all(got["steps"] == 7)
    got = trace(renderer, G.desc("cfg1_ks_rk4"))
    assert np.all(got["status"] == abi.KT_RAY_EVENT)


def test_errors_are_status_codes(renderer):
    import kerrtracecpp2_b200 as kt

    with pytest.raises(kt.KerrTraceError) as e:
        renderer.trace(abi.frame_desc(width=0, height=10))
    assert e.value.status == abi.KT_ERR_INVALID_ARGUMENT
    with pytest.raises(kt.KerrTraceError) as e:
        renderer.trace(abi.frame_desc(width=8, height=8, chart=abi.KT_CHART_BL,
                                      solver_mode=abi.KT_SOLVER_ELLIPTIC_CLOSED,
                                      precision=abi.KT_PREC_MIXED))
    assert e.value.status == abi.KT_ERR_UNSUPPORTED
    # the context stays usable after an error
    got = trace(renderer, G.desc("one_pixel"))
    assert G.mismatches(got, G.result("one_pixel")) == {k: 0 for k in G.FIELDS}


def test_fp64_peak_probe(renderer):
    g = renderer.fp64_peak_gflops()
    assert 1e3 < g < 1e6
