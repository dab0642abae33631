"""The semi-analytic solver on the GPU (k_trace<ModeSepRk4> and the BL RK4
launch over the rays it gives up on): bit-identical to the reference's
results in tests/golden/semi.npz, through kt_trace, kt_trace_pixels and
batches, with the same step counters as the host build of the kernel
code."""
import ctypes

import numpy as np
import pytest

import golden_lib as G
from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu
NAMES = sorted(G.semi_cases())


def to_np(out):
    import torch

    torch.cuda.synchronize()
    got = {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}
    got["steps"] = got["steps"].view(np.uint32)
    got["attempts"] = got["attempts"].view(np.uint32)
    return got


@pytest.mark.parametrize("name", NAMES)
def test_trace_matches_reference(renderer, name):
    got = to_np(renderer.trace(G.semi_desc(name)))
    assert G.mismatches(got, G.semi_result(name)) == {k: 0 for k in G.FIELDS}


def test_counters_match_host_build(renderer):
    import test_hostcheck
    import testlibs

    L = ctypes.CDLL(testlibs.HOSTCHECK)
    L.hc_trace_pixels.argtypes = [ctypes.POINTER(abi.FrameDesc), ctypes.c_int64, ctypes.c_void_p] + \
        [ctypes.c_void_p] * 10
    d = G.semi_desc("semi_kerr")
    got = to_np(renderer.trace(d))
    want = test_hostcheck.run(L, d)
    for k in ("steps", "attempts", "status"):
        assert np.array_equal(got[k], want[k]), k


def test_pixel_list_matches_frame(renderer):
    """A shuffled pixel list through kt_trace_pixels: rays that the
    separable tracer gives up on reach their own output slots through the
    fallback list."""
    import torch

    d = G.semi_desc("semi_close_camera")
    n = d.width * d.height
    perm = np.random.default_rng(3).permutation(n).astype(np.int32)
    got = to_np(renderer.trace_pixels(d, torch.from_numpy(perm).cuda()))
    want = G.semi_result("semi_close_camera")
    assert G.mismatches(got, {k: v[perm] for k, v in want.items()}) == {k: 0 for k in G.FIELDS}


def test_batch_with_semi_frames(renderer):
    """Separable-Kerr frames share a batch with standard frames, including a
    KS frame that asked for DOPRI5 (its BL pass keeps DOPRI5) and a
    separable frame that asked for DOPRI5 (its BL pass uses RK4)."""
    names = ["semi_kerr", "semi_dopri5_request", "semi_close_camera", "semi_charged",
             "semi_ks_request"]
    descs = [G.semi_desc(n) for n in names] + [G.desc("ks_dopri5_request"), G.desc("cfg2_bl_dopri5")]
    wants = [G.semi_result(n) for n in names] + [G.result("ks_dopri5_request"), G.result("cfg2_bl_dopri5")]
    b = renderer.batch(descs)
    b.launch()
    for d, o, want in zip(descs, b.outs, wants):
        assert G.mismatches(to_np(o), want) == {k: 0 for k in G.FIELDS}
    b.close()
