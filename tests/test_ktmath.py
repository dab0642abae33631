"""The renderer's libm (ktmath.h) against mpmath: accuracy bounds stated in
its header, special values, and determinism of the host build."""
import ctypes
import math
import random

import mpmath
import pytest

import testlibs

mpmath.mp.prec = 120


@pytest.fixture(scope="module")
def L():
    lib = ctypes.CDLL(testlibs.SHIM)
    for n in ("sin", "cos", "exp", "log", "log10", "cbrt", "acos", "atan", "asin"):
        f = getattr(lib, "kts_" + n)
        f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double]
    for n in ("pow", "atan2", "hypot"):
        f = getattr(lib, "kts_" + n)
        f.restype, f.argtypes = ctypes.c_double, [ctypes.c_double] * 2
    return lib


def ulp_err(got, exact):
    exact = mpmath.mpf(exact)
    if exact == 0:
        return 0.0 if got == 0 else float("inf")
    e = math.frexp(float(exact))[1]
    return float(abs(mpmath.mpf(got) - exact) / mpmath.mpf(2) ** max(e - 53, -1074))  # subnormal spacing


CASES = [
    ("sin", mpmath.sin, lambda r: (r.uniform(-10, 10),), 0.75),
    ("sin", mpmath.sin, lambda r: (r.uniform(-1e5, 1e5),), 0.75),
    ("cos", mpmath.cos, lambda r: (r.uniform(-10, 10),), 0.75),
    ("exp", mpmath.exp, lambda r: (r.uniform(-700, 700),), 1.0),
    ("log", mpmath.log, lambda r: (math.exp(r.uniform(-700, 700)),), 0.6),
    ("log10", mpmath.log10, lambda r: (r.uniform(1, 100),), 0.6),
    ("pow", lambda x, y: x ** y, lambda r: (r.uniform(1e-3, 1e3), r.choice([0.2, 0.25, 4.0, 1 / 2.2])), 1.1),
    ("cbrt", mpmath.cbrt, lambda r: (math.exp(r.uniform(-50, 50)),), 0.6),
    ("atan2", mpmath.atan2, lambda r: (r.uniform(-10, 10), r.uniform(-10, 10)), 2.0),
    ("acos", mpmath.acos, lambda r: (r.uniform(-1, 1),), 2.0),
    ("atan", mpmath.atan, lambda r: (r.uniform(-50, 50),), 2.0),
    ("atan", mpmath.atan, lambda r: (r.uniform(-1, 1),), 2.0),
    ("asin", mpmath.asin, lambda r: (r.uniform(-1, 1),), 2.0),
    ("asin", mpmath.asin, lambda r: (1.0 - math.exp(r.uniform(-30, -1)),), 2.0),
    ("hypot", lambda x, y: mpmath.sqrt(x * x + y * y), lambda r: (r.uniform(-10, 10), r.uniform(-10, 10)), 1.0),
    ("hypot", lambda x, y: mpmath.sqrt(x * x + y * y),
     lambda r: (math.ldexp(r.uniform(1, 2), r.randint(-1070, 1020)), math.ldexp(r.uniform(1, 2), r.randint(-1070, 1020))), 1.0),
]


@pytest.mark.parametrize("name,ref,gen,bound", CASES, ids=[c[0] for c in CASES])
def test_accuracy(L, name, ref, gen, bound):
    rng = random.Random(7)
    f = getattr(L, "kts_" + name)
    worst = 0.0
    for _ in range(3000):
        args = gen(rng)
        worst = max(worst, ulp_err(f(*args), ref(*[mpmath.mpf(a) for a in args])))
    assert worst <= bound, f"{name}: {worst:.3f} ulp > {bound}"


def test_special_values(L):
    assert L.kts_pow(0.0, 0.45) == 0.0
    assert L.kts_pow(-2.0, 3.0) == -8.0
    assert math.isnan(L.kts_pow(-2.0, 0.5))
    assert L.kts_pow(5.0, 0.0) == 1.0
    assert L.kts_pow(1.0, float("nan")) == 1.0
    assert L.kts_atan2(0.0, -1.0) == math.pi
    assert math.copysign(1, L.kts_atan2(-0.0, 1.0)) < 0
    assert L.kts_atan2(1.0, 0.0) == math.pi / 2
    assert math.isnan(L.kts_sin(float("inf")))
    assert L.kts_log(0.0) == -math.inf
    assert math.isnan(L.kts_log(-1.0))
    assert L.kts_exp(-800.0) == 0.0 and L.kts_exp(800.0) == math.inf
    assert L.kts_cbrt(-27.0) == -3.0
    assert L.kts_acos(1.0) == 0.0
    assert math.isnan(L.kts_acos(1.5))
    assert L.kts_asin(1.0) == math.pi / 2 and L.kts_asin(-0.0) == 0.0
    assert math.isnan(L.kts_asin(1.5))
    assert L.kts_atan(math.inf) == math.pi / 2 and L.kts_atan(0.0) == 0.0
    assert L.kts_hypot(3.0, 4.0) == 5.0 and L.kts_hypot(-0.0, 2.5) == 2.5
    assert L.kts_hypot(math.inf, math.nan) == math.inf
    assert L.kts_hypot(1e308, 1e308) == pytest.approx(math.sqrt(2) * 1e308, rel=1e-15)
    assert L.kts_hypot(3e-320, 4e-320) == pytest.approx(5e-320, rel=1e-3)


def test_exact_points(L):
    # powers and roots the renderer hits: pow(x, 4) for the disk intensity,
    # log10(50) for the blackbody ramp, cos(pi/2) for the equatorial metric
    for x in (0.5, 1.5, 2.0, 3.0, 10.0):
        assert L.kts_pow(x, 4.0) == x ** 4
    assert abs(L.kts_log10(50.0) - math.log10(50.0)) <= 2.3e-16 * 2
    assert L.kts_cos(math.pi / 2) == pytest.approx(6.123233995736766e-17, rel=1e-15)


def test_div3_is_the_ieee_quotient(L):
    """ktm_div3 (three operations) returns the bits of x / 3.0 for every
    binade, sign and the special values, and for every pattern of the low 20
    significand bits at a few exponents."""
    import numpy as np

    rng = np.random.default_rng(3)
    bits = rng.integers(0, 2 ** 63, 4_000_000, dtype=np.uint64) | (
        rng.integers(0, 2, 4_000_000, dtype=np.uint64) << np.uint64(63))
    low = np.arange(2 ** 20, dtype=np.uint64)
    patterns = [np.uint64(e) << np.uint64(52) | np.uint64(m) << np.uint64(32) | low
                for e in (1, 64, 1021, 1023, 1024, 1999, 2045) for m in (0, 0x55555, 0xaaaaa, 0xfffff)]
    x = np.concatenate([bits] + patterns).view(np.float64)
    x = np.concatenate([x, np.array([0.0, -0.0, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308,
                                     np.inf, -np.inf, np.nan, 3.0, -3.0, 1.0, 0.1])])
    q = np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    L.kts_div3_n(x.ctypes.data_as(dp), q.ctypes.data_as(dp), ctypes.c_long(x.size))
    with np.errstate(all="ignore"):
        ref = x / 3.0
    same = (q.view(np.uint64) == ref.view(np.uint64)) | (np.isnan(q) & np.isnan(ref))
    assert same.all(), x[~same][:5]
