"""The GPU kernels' per-ray code (kt_machines.cuh / kt_physics.cuh) compiled
for the host: bit-identical to the reference fixtures on every path.  This
pins the kernels' operation order on the CPU; the GPU tests repeat the
comparison with the device build."""
import ctypes

import numpy as np
import pytest

import golden_lib as G
import testlibs
from kerrtracecpp2_b200.abi import FrameDesc, frame_desc

P = ctypes.c_void_p


@pytest.fixture(scope="module")
def hc():
    L = ctypes.CDLL(testlibs.HOSTCHECK)
    L.hc_trace_pixels.argtypes = [ctypes.POINTER(FrameDesc), ctypes.c_int64, P] + [P] * 10
    L.hc_trace_pixels.restype = ctypes.c_int
    return L


def run(hc, d, pix=None):
    n = d.width * d.height
    pix = np.arange(n, dtype=np.uint32) if pix is None else pix
    n = len(pix)
    o = {k: np.zeros(n, dt) for k, dt in [("outcome", np.uint8), ("r", "f8"), ("redshift", "f8"),
                                           ("magnif", "f8"), ("phi_disk", "f8"), ("theta_esc", "f8"),
                                           ("phi_esc", "f8"), ("status", np.uint8),
                                           ("steps", np.uint32), ("attempts", np.uint32)]}
    keys = ["outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc", "status",
            "steps", "attempts"]
    assert hc.hc_trace_pixels(ctypes.byref(d), n, pix.ctypes.data_as(P),
                              *[o[k].ctypes.data_as(P) for k in keys]) == 0
    return o


@pytest.mark.parametrize("name", sorted(G.cases()))
def test_kernel_code_matches_reference(hc, name):
    got = run(hc, G.desc(name))
    assert G.mismatches(got, G.result(name)) == {k: 0 for k in G.FIELDS}


def test_step_counters_match_oracle(hc):
    import oracle_lib as O

    d = G.desc("cfg2_bl_dopri5")
    got = run(hc, d)
    want = O.trace_port(d, counters=True)
    assert np.array_equal(got["steps"], want["steps"])
    assert np.array_equal(got["attempts"], want["attempts"])


def test_status_codes(hc):
    got = run(hc, G.desc("step_cap"))
    assert np.all(got["status"] == 1) and np.all(got["steps"] == 7)
    got = run(hc, G.desc("cfg1_ks_rk4"))
    assert np.all(got["status"] == 0)


def test_pixel_subset_equals_frame(hc):
    d = G.desc("cfg5_ks")
    full = run(hc, d)
    pix = np.array([0, 7, 100, 1151, 2303, 5], np.uint32)
    sub = run(hc, d, pix)
    for k in G.FIELDS:
        assert np.array_equal(G.bits(sub[k]), G.bits(full[k][pix]))


@pytest.mark.parametrize("shape", [1, 2], ids=["rolled", "unrolled"])
@pytest.mark.parametrize("name", [n for n, kw in sorted(G.cases().items()) if kw.get("bundles")])
def test_bundle_rhs_split_matches_reference(hc, name, shape):
    """The bundle RHS split over two lanes (bundle_rhs_half for each lane,
    in either code shape, and bundle_rhs_combine), as the paired bundle
    kernel evaluates it, traced on the host: bit-identical to the
    reference's bundle fixtures."""
    hc.hc_set_bundle_split.argtypes = [ctypes.c_int]
    hc.hc_set_bundle_split(shape)
    try:
        got = run(hc, G.desc(name))
    finally:
        hc.hc_set_bundle_split(0)
    assert G.mismatches(got, G.result(name)) == {k: 0 for k in G.FIELDS}


@pytest.mark.parametrize("full_creep", [False, True], ids=["creep_end", "full_creep"])
def test_bundle_rhs_split_matches_oracle_medium(hc, full_creep):
    """Config 3's geometry at 96x54 through the split bundle RHS on the host:
    all fields bit-identical to the oracle; the counters too, but for the
    rays stopped while creeping onto the horizon (status KT_RAY_CREEP, whose
    counters stop early), and for every ray with KT_FLAG_BUNDLE_FULL_CREEP."""
    import oracle_lib as O
    from kerrtracecpp2_b200 import abi

    d = abi.frame_desc(chart=1, bundles=1, a=0.998, theta_deg=60.0, width=96, height=54,
                       flags=abi.KT_FLAG_BUNDLE_FULL_CREEP if full_creep else 0)
    hc.hc_set_bundle_split.argtypes = [ctypes.c_int]
    hc.hc_set_bundle_split(1)
    try:
        got = run(hc, d)
    finally:
        hc.hc_set_bundle_split(0)
    want = O.trace_port(d, counters=True)
    assert G.mismatches(got, want) == {k: 0 for k in G.FIELDS}
    ok, creeping = O.counters_agree(got, want)
    assert ok
    if full_creep:
        assert creeping == 0
        assert np.array_equal(got["steps"], want["steps"]) and np.array_equal(got["attempts"], want["attempts"])
    else:
        assert creeping > 0  # this frame has rays plunging near the equator
        creep = got["status"] == abi.KT_RAY_CREEP
        assert np.all(got["outcome"][creep] == 0) and np.all(got["r"][creep] == 0.0)
        print(f"{creeping} creeping rays; attempts {got['attempts'].sum()} against the "
              f"oracle's {want['attempts'].sum()}")


@pytest.mark.parametrize("wh", [(1280, 720), (1920, 1080), (1283, 721), (77, 31), (7, 10000), (1, 70000),
                                (8, 4), (512, 512)])
def test_centre_out_order_input_map(hc, wh):
    """ring_item, the input order of the centre-out sort, maps the items
    0..W*H-1 one to one onto the pixels: 8 x 4 blocks of the top-left region
    whose 32 pixels share one ring, then the strips row-major."""
    W, H = wh
    n = W * H
    p = np.zeros(n, np.uint32)
    c = np.zeros(n, np.int32)
    hc.hc_ring_items.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    hc.hc_ring_items(W, H, p.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p))
    assert np.array_equal(np.sort(p), np.arange(n, dtype=np.uint32))
    assert c.min() >= 0 and c.max() < 512
    n_int = (W // 8 * 8) * (H // 4 * 4)
    if n_int:
        blocks = p[:n_int].reshape(-1, 32)
        x, y = blocks % W, blocks // W
        assert np.all(x.max(1) - x.min(1) == 7) and np.all(y.max(1) - y.min(1) == 3)
        assert np.all(c[:n_int].reshape(-1, 32) == c[:n_int].reshape(-1, 32)[:, :1])
    # the rings grow outward: the sorted order starts at the image centre
    order = p[np.argsort(c, kind="stable")]
    cx, cy = (W - 1) / 2, (H - 1) / 2
    d0 = np.hypot(order[:32] % W - cx, order[:32] // W - cy).max()
    ring_w = max(4.0, (np.hypot(cx, cy) + 1) / 512)
    assert d0 <= ring_w + 9.0
