"""The device probes behind the roofline: FP64 FMA throughput and the
measured cost of the weighted operations (division, x/3, sqrt, sincos,
pow), in flops of FMA-pipe time."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp64_peak_and_op_costs(renderer):
    peak = renderer.fp64_peak_gflops()
    c = renderer.op_costs()
    print(f"FP64 FMA {peak:.0f} GFLOP/s; op costs (flops): " +
          ", ".join(f"{k} {v:.1f}" for k, v in c.items() if k != "fma_gflops"))
    assert 1e3 < peak < 1e5
    assert 0.8 < c["fma_gflops"] / peak < 1.25
    # a correctly rounded division or square root takes several FMA times;
    # x/3 in three operations is cheaper than a division; sincos and pow are
    # polynomial evaluations of tens of operations
    assert 4.0 < c["div"] < 100.0 and 4.0 < c["sqrt"] < 100.0
    assert 2.0 < c["div3"] < c["div"]
    assert 40.0 < c["sincos"] < 500.0 and 60.0 < c["pow"] < 800.0
