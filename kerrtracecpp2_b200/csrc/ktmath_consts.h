/* Generated by gen_ktmath_consts.py: binary64 roundings of exact constants. */
#pragma once
#define KTM_PIO2_1 0x1.921fb54442d18p+0
#define KTM_PIO2_2 0x1.1a62633145c07p-54
#define KTM_PIO2_3 -0x1.f1976b7ed8fbcp-110
#define KTM_2_OVER_PI 0x1.45f306dc9c883p-1
#define KTM_PI_HI 0x1.921fb54442d18p+1
#define KTM_PI_LO 0x1.1a62633145c07p-53
#define KTM_PIO2_HI 0x1.921fb54442d18p+0
#define KTM_PIO2_LO 0x1.1a62633145c07p-54
#define KTM_PIO4_HI 0x1.921fb54442d18p-1
#define KTM_PIO4_LO 0x1.1a62633145c07p-55
#define KTM_LN2_HI 0x1.62e42ff000000p-1
#define KTM_LN2_LO -0x1.718432a1b0e26p-35
#define KTM_INV_LN2 0x1.71547652b82fep+0
#define KTM_INV_LN10_HI 0x1.bcb7b1526e50ep-2
#define KTM_INV_LN10_LO 0x1.95355baaafad3p-57
#define KTM_SQRT2_OVER_2 0x1.6a09e667f3bcdp-1
/* sin(r) = r + r^3 * sum_k KTM_SIN[k] * r^(2k),  KTM_SIN[k] = (-1)^(k+1)/(2k+3)! */
#define KTM_SIN_COEFFS {-0x1.5555555555555p-3, 0x1.1111111111111p-7, -0x1.a01a01a01a01ap-13, 0x1.71de3a556c734p-19, -0x1.ae64567f544e4p-26, 0x1.6124613a86d09p-33, -0x1.ae7f3e733b81fp-41, 0x1.952c77030ad4ap-49, -0x1.2f49b46814157p-57}
/* cos(r) = 1 - r^2/2 + r^4 * sum_k KTM_COS[k] * r^(2k),  KTM_COS[k] = (-1)^k/(2k+4)! */
#define KTM_COS_COEFFS {0x1.5555555555555p-5, -0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-16, -0x1.27e4fb7789f5cp-22, 0x1.1eed8eff8d898p-29, -0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-45, -0x1.6827863b97d97p-53, 0x1.e542ba4020225p-62}
/* exp(r) - 1 - r = r^2 * sum_k KTM_EXP[k] * r^k,  KTM_EXP[k] = 1/(k+2)! */
#define KTM_EXP_COEFFS {0x1.0000000000000p-1, 0x1.5555555555555p-3, 0x1.5555555555555p-5, 0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26, 0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37}
/* 2*atanh(s) - 2s = s^3 * sum_k KTM_LOG[k] * s^(2k),  KTM_LOG[k] = 2/(2k+3) */
#define KTM_LOG_COEFFS {0x1.5555555555555p-1, 0x1.999999999999ap-2, 0x1.2492492492492p-2, 0x1.c71c71c71c71cp-3, 0x1.745d1745d1746p-3, 0x1.3b13b13b13b14p-3, 0x1.1111111111111p-3, 0x1.e1e1e1e1e1e1ep-4, 0x1.af286bca1af28p-4, 0x1.8618618618618p-4, 0x1.642c8590b2164p-4, 0x1.47ae147ae147bp-4}
/* atan(t) - t = t^3 * sum_k KTM_ATAN[k] * t^(2k),  KTM_ATAN[k] = (-1)^(k+1)/(2k+3) */
#define KTM_ATAN_COEFFS {-0x1.5555555555555p-2, 0x1.999999999999ap-3, -0x1.2492492492492p-3, 0x1.c71c71c71c71cp-4, -0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, -0x1.1111111111111p-4, 0x1.e1e1e1e1e1e1ep-5, -0x1.af286bca1af28p-5}
/* atan(i/8), i = 0..8, as double-double */
#define KTM_ATAN_TAB_HI {0x0.0p+0, 0x1.fd5ba9aac2f6ep-4, 0x1.f5b75f92c80ddp-3, 0x1.6f61941e4def1p-2, 0x1.dac670561bb4fp-2, 0x1.1e00babdefeb4p-1, 0x1.4978fa3269ee1p-1, 0x1.700a7c5784634p-1, 0x1.921fb54442d18p-1}
#define KTM_ATAN_TAB_LO {0x0.0p+0, -0x1.cd37686760c17p-59, 0x1.8ab6e3cf7afbdp-57, -0x1.c63aae6f6e918p-56, 0x1.a2b7f222f65e2p-56, -0x1.928df287a668fp-58, 0x1.2419a87f2a458p-56, -0x1.8c34d25aadef6p-56, 0x1.1a62633145c07p-55}
