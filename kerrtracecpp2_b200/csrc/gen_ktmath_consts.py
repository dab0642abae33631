"""Generate the constant table of ktmath.h (the renderer's own FP64 libm).

Every constant is a mathematical quantity evaluated at 200-bit precision with
mpmath and rounded to IEEE binary64 (hex-float literals, so the value is exact
in the source).  Nothing here is taken from another library: the polynomial
coefficients are plain Taylor coefficients (1/n!, 1/(2k+1)), and the
argument-reduction constants are multi-part splits of pi/2, ln 2 and atan(i/8).

Run:  python kerrtracecpp2_b200/csrc/gen_ktmath_consts.py > kerrtracecpp2_b200/csrc/ktmath_consts.h
"""
import mpmath

mpmath.mp.prec = 200


def d(x):
    """Round an mpmath value to binary64 and format it as a hex literal."""
    return float(x).hex()


def split(x, parts, bits=None):
    """Split x into `parts` doubles whose sum approximates x to ~53*parts bits.

    With bits=None each part is the nearest double to the remainder (for use
    with fma-based reduction).  With bits=k the leading parts keep only k
    significant bits, so n*part is exact for |n| < 2^(53-k).
    """
    out = []
    rem = mpmath.mpf(x)
    for i in range(parts):
        if bits is not None and i < parts - 1:
            e = mpmath.floor(mpmath.log(abs(rem), 2))
            q = mpmath.mpf(2) ** (e - bits + 1)
            p = mpmath.nint(rem / q) * q
        else:
            p = mpmath.mpf(float(rem))
        out.append(float(p))
        rem = rem - mpmath.mpf(float(p))
    return out


def main():
    pi = mpmath.pi
    lines = []
    emit = lines.append
    emit("/* Generated by gen_ktmath_consts.py: binary64 roundings of exact constants. */")
    emit("#pragma once")
    # pi/2 in three full-width parts for fma-based Cody-Waite reduction.
    p1, p2, p3 = split(pi / 2, 3)
    emit(f"#define KTM_PIO2_1 {p1.hex()}")
    emit(f"#define KTM_PIO2_2 {p2.hex()}")
    emit(f"#define KTM_PIO2_3 {p3.hex()}")
    emit(f"#define KTM_2_OVER_PI {d(2 / pi)}")
    # pi, pi/2, pi/4 as double-double (hi, lo)
    for name, v in (("PI", pi), ("PIO2", pi / 2), ("PIO4", pi / 4)):
        hi, lo = split(v, 2)
        emit(f"#define KTM_{name}_HI {hi.hex()}")
        emit(f"#define KTM_{name}_LO {lo.hex()}")
    # ln2 with a short high part (k*LN2_HI exact for |k| < 2^21) + full low part
    l1, l2 = split(mpmath.log(2), 2, bits=32)
    emit(f"#define KTM_LN2_HI {l1.hex()}")
    emit(f"#define KTM_LN2_LO {l2.hex()}")
    emit(f"#define KTM_INV_LN2 {d(1 / mpmath.log(2))}")
    h, lo = split(1 / mpmath.log(10), 2)
    emit(f"#define KTM_INV_LN10_HI {h.hex()}")
    emit(f"#define KTM_INV_LN10_LO {lo.hex()}")
    emit(f"#define KTM_SQRT2_OVER_2 {d(mpmath.sqrt(2) / 2)}")
    # Taylor coefficients
    emit("/* sin(r) = r + r^3 * sum_k KTM_SIN[k] * r^(2k),  KTM_SIN[k] = (-1)^(k+1)/(2k+3)! */")
    sin_c = [(-1) ** (k + 1) / mpmath.factorial(2 * k + 3) for k in range(9)]
    emit("#define KTM_SIN_COEFFS {" + ", ".join(d(c) for c in sin_c) + "}")
    emit("/* cos(r) = 1 - r^2/2 + r^4 * sum_k KTM_COS[k] * r^(2k),  KTM_COS[k] = (-1)^k/(2k+4)! */")
    cos_c = [(-1) ** k / mpmath.factorial(2 * k + 4) for k in range(9)]
    emit("#define KTM_COS_COEFFS {" + ", ".join(d(c) for c in cos_c) + "}")
    emit("/* exp(r) - 1 - r = r^2 * sum_k KTM_EXP[k] * r^k,  KTM_EXP[k] = 1/(k+2)! */")
    exp_c = [1 / mpmath.factorial(k + 2) for k in range(13)]
    emit("#define KTM_EXP_COEFFS {" + ", ".join(d(c) for c in exp_c) + "}")
    emit("/* 2*atanh(s) - 2s = s^3 * sum_k KTM_LOG[k] * s^(2k),  KTM_LOG[k] = 2/(2k+3) */")
    log_c = [mpmath.mpf(2) / (2 * k + 3) for k in range(12)]
    emit("#define KTM_LOG_COEFFS {" + ", ".join(d(c) for c in log_c) + "}")
    emit("/* atan(t) - t = t^3 * sum_k KTM_ATAN[k] * t^(2k),  KTM_ATAN[k] = (-1)^(k+1)/(2k+3) */")
    atan_c = [mpmath.mpf((-1) ** (k + 1)) / (2 * k + 3) for k in range(9)]
    emit("#define KTM_ATAN_COEFFS {" + ", ".join(d(c) for c in atan_c) + "}")
    emit("/* atan(i/8), i = 0..8, as double-double */")
    hi_l, lo_l = [], []
    for i in range(9):
        hi, lo = split(mpmath.atan(mpmath.mpf(i) / 8), 2)
        hi_l.append(hi.hex())
        lo_l.append(lo.hex())
    emit("#define KTM_ATAN_TAB_HI {" + ", ".join(hi_l) + "}")
    emit("#define KTM_ATAN_TAB_LO {" + ", ".join(lo_l) + "}")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
