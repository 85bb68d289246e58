// fpmath.h -- exp and pow in IEEE binary64 arithmetic that give the same
// bits on the host and on the device.
//
// The per-step path raises to real powers in the drag law (drag.f:60-157),
// the gas-particle heat transfer (hvs.f:9-83), the collision integral of
// the gas viscosity (visc.f:37-148, with exp), the particle repulsion
// (tilde.f:362-416) and the sub-grid filter (turbo.f).  The C library and
// CUDA's math library may round these last bits differently, and one last
// bit is enough to put a corrector cell whose |dg| lies within a rounding
// error of conv on the other side of the convergence test, after which two
// runs differ at the level of delg.  The routines below use only +, -, *, /,
// fma, rint and ldexp -- each exactly specified by IEEE 754, so the same on
// the host (C++, no FMA contraction) and the device (CUDA, -fmad=false) --
// and tables written out as hexadecimal literals (fpmath_tables.h, made by
// gen_fpmath_tables.py).  The engine's kernels and the CPU oracle both call
// them, so both compute the same bits.
//
// Methods: P. T. P. Tang, "Table-driven implementation of the exponential
// function in IEEE floating-point arithmetic", ACM TOMS 15 (1989) 144-157
// (exp = 2^m * 2^(j/32) * exp(r), |r| <= ln2/64), and "Table-driven
// implementation of the logarithm function in IEEE floating-point
// arithmetic", ACM TOMS 16 (1990) 378-400 (log x = m ln2 + log F +
// log1p(f/F), F = 1 + j/128).  pow(x, y) = exp(y log x) with log x carried
// as a double-double and y log x formed with fma, so the result is within
// about one unit in the last place (tests/test_fpmath.py checks it against
// the C library over the ranges the path uses).
#pragma once
#include <cmath>
#include <limits>

#include "fpmath_tables.h"

#ifdef __CUDACC__
#define PDAC_FP_FN __host__ __device__ __forceinline__
#else
#define PDAC_FP_FN inline
#endif

namespace pdac_fp {

#ifdef __CUDACC__
__constant__ const double kExp2Tab[64] = PDAC_EXP2_TABLE;
__constant__ const double kLogTab[258] = PDAC_LOG_TABLE;
#endif
static const double hExp2Tab[64] = PDAC_EXP2_TABLE;
static const double hLogTab[258] = PDAC_LOG_TABLE;

PDAC_FP_FN double exp2_tab(int q) {
#ifdef __CUDA_ARCH__
    return kExp2Tab[q];
#else
    return hExp2Tab[q];
#endif
}
PDAC_FP_FN double log_tab(int q) {
#ifdef __CUDA_ARCH__
    return kLogTab[q];
#else
    return hLogTab[q];
#endif
}

PDAC_FP_FN double fma_(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
PDAC_FP_FN double rint_(double x) {
#ifdef __CUDA_ARCH__
    return rint(x);
#else
    return std::nearbyint(x);
#endif
}
PDAC_FP_FN double ldexp_(double x, int e) {
#ifdef __CUDA_ARCH__
    return ldexp(x, e);
#else
    return std::ldexp(x, e);
#endif
}
PDAC_FP_FN double frexp_(double x, int *e) {
#ifdef __CUDA_ARCH__
    return frexp(x, e);
#else
    return std::frexp(x, e);
#endif
}

// exp(zh + zl) for |zl| no larger than an ulp or so of zh
PDAC_FP_FN double exp_dd(double zh, double zl) {
    if (zh != zh) return zh;
    if (zh > 709.782712893384) return std::numeric_limits<double>::infinity();
    if (zh < -745.2) return 0.0;
    const double N = rint_(zh * PDAC_INV_LN2_32);
    const int n = (int)N, j = n & 31, m = (n - j) / 32;
    double r = fma_(-N, PDAC_LN2_32_HI, zh);
    r = fma_(-N, PDAC_LN2_32_LO, r) + zl;
    // exp(r) - 1 to degree 6; |r| <= ln2/64, so the first term left out is
    // below 4e-18 of the result
    const double q = r * r * (0x1.0p-1 + r * (0x1.5555555555555p-3 + r * (0x1.5555555555555p-5 +
                                                                     r * (0x1.1111111111111p-7 +
                                                                          r * 0x1.6c16c16c16c17p-10))));
    const double p = r + q;
    const double th = exp2_tab(2 * j), tl = exp2_tab(2 * j + 1);
    const double s = th + tl;
    return ldexp_(th + (tl + s * p), m);
}

PDAC_FP_FN double exp(double x) { return exp_dd(x, 0.0); }

// log x as hi + lo, for finite x > 0
PDAC_FP_FN void log_dd(double x, double &hi, double &lo) {
    int e;
    double y = frexp_(x, &e);  // y in [0.5, 1)
    y = y * 2.0;
    e = e - 1;  // x = 2^e y, y in [1, 2)
    int j = (int)rint_((y - 1.0) * 128.0);
    j = j < 0 ? 0 : (j > 128 ? 128 : j);  // y in [1, 2) gives 0 .. 128; the table has 129 entries
    const double F = 1.0 + (double)j * 0x1.0p-7;
    const double f = y - F;                    // exact: |f| <= 1/256
    const double g = f / F;                    // f/F = g + gl
    const double gl = fma_(-g, F, f) / F;
    // log1p(g) - g to degree 6 in g; |g| <= 1/256, the first term left out is
    // below 3e-18
    const double poly = g * g * (-0x1.0p-1 + g * (0x1.5555555555555p-2 + g * (-0x1.0p-2 + g * (0x1.999999999999ap-3 +
                                                                                       g * -0x1.5555555555555p-3))));
    const double a = (double)e * PDAC_LN2_HI;  // exact: the table's ln2 keeps 42 significant bits
    const double b = log_tab(2 * j);
    // two exact sums (Knuth's TwoSum), then the small parts
    double s1 = a + b, bb = s1 - a, t1 = (a - (s1 - bb)) + (b - bb);
    double s2 = s1 + g;
    bb = s2 - s1;
    double t2 = (s1 - (s2 - bb)) + (g - bb);
    double l = t1 + t2 + ((double)e * PDAC_LN2_LO + log_tab(2 * j + 1) + gl + poly);
    hi = s2 + l;
    lo = l - (hi - s2);
}

// x^y for the path's arguments: x >= 0 (x < 0 gives NaN unless y is an
// integer), with the IEEE special cases the path can meet.  Written without
// recursion: a recursive device function leaves the kernel's stack size to
// the runtime's default limit instead of the size the compiler computes.
PDAC_FP_FN double pow(double x, double y) {
    if (y == 0.0 || x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    bool negate = false;
    if (x < 0.0) {
        if (y != rint_(y)) return std::numeric_limits<double>::quiet_NaN();
        negate = rint_(y * 0.5) * 2.0 != y;  // an odd integer power keeps the sign
        x = -x;
    }
    double r;
    if (x == 0.0) r = y > 0.0 ? 0.0 : std::numeric_limits<double>::infinity();
    else if (x == std::numeric_limits<double>::infinity()) r = y > 0.0 ? x : 0.0;
    else {
        double lh, ll;
        log_dd(x, lh, ll);
        const double zh = y * lh;
        const double zl = fma_(y, lh, -zh) + y * ll;
        r = exp_dd(zh, zl);
    }
    return negate ? -r : r;
}

}  // namespace pdac_fp
