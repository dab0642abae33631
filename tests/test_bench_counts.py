"""The algorithmic flop count of bench.py's roofline: the per-unit counts
with unit operation weights reproduce the totals stated beside them (BL RHS
453, DOPRI5 attempt 447, RK4-doubling attempt 335 flops), measured weights
enter linearly, and only the standard BL single-ray integrators are
counted."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from kerrtracecpp2_b200 import abi  # noqa: E402


def test_unit_weight_totals():
    w = bench.UNIT_WEIGHTS
    assert bench.weighted(bench.RHS_COUNTS, w) == 453.0
    assert bench.weighted(bench.DOPRI5_ATTEMPT_COUNTS, w) == 447.0
    assert bench.weighted(bench.RK4_ATTEMPT_COUNTS, w) == 335.0


def test_frame_flops_from_counters():
    d = abi.frame_desc(**bench.WORKLOADS["knds_bl_dopri5_720p"])
    n = d.width * d.height
    att = 100.0 * n
    assert bench.ray_flops(d, 0.0, att) == pytest.approx((n + 6 * att) * 453 + att * 447)
    w = dict(bench.UNIT_WEIGHTS, div=26.0)  # a division at 13 FMA slots
    extra = (n + 6 * att) * 26 * 25.0 + att * 5 * 25.0
    assert bench.ray_flops(d, 0.0, att, w) == pytest.approx(bench.ray_flops(d, 0.0, att) + extra)
    rk4 = abi.frame_desc(**dict(bench.WORKLOADS["knds_bl_dopri5_720p"], integrator=0))
    assert bench.ray_flops(rk4, 50.0 * n, att) == pytest.approx((n + 10 * att + 50 * n) * 453 + att * 335)
    assert bench.ray_flops(abi.frame_desc(chart=0, a=0.5), 1.0, 1.0) is None
    assert bench.ray_flops(abi.frame_desc(chart=1, bundles=1), 1.0, 1.0) is None
