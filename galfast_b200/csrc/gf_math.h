/*
 * gf_math.h -- portable elementary functions with identical results on the
 * host (g++, -ffp-contract=off) and on sm_100a (nvcc, -fmad=false).
 *
 * Why: galfast's catalog draws are bit-exact functions of the float values of
 * expf/powf/logf/tanf/... evaluated per (pixel, distance, Mr) bin.  The CUDA
 * and glibc implementations of those functions differ in the last ulp, so a
 * GPU build that called them could never reproduce a CPU run draw for draw.
 * Every function below is evaluated with the same sequence of IEEE-754
 * double operations (add, mul, div, sqrt, fma, rint -- all correctly rounded
 * on both targets), so host and device agree bit for bit.
 *
 * Methods (all from the mathematics; constants in gf_math_consts.h are
 * generated by gen_math_consts.py from arbitrary-precision arithmetic):
 *   exp   Cody-Waite reduction x = n ln2 + r (two-piece ln2), Taylor series of
 *         degree 13 on |r| <= ln2/2, scaling by 2^n through the exponent field.
 *   log   x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
 *         s = (m-1)/(m+1), odd series of atanh to s^23.
 *   sin/cos  Cody-Waite reduction by pi/2 (three 33-bit pieces), Taylor series
 *         to r^19 / r^18 on |r| <= pi/4, quadrant selection.
 *   atan  table of atan(i/8) (double-double) and the addition formula
 *         atan t = atan c + atan((t-c)/(1+tc)), Taylor series to u^15;
 *         atan2 and asin are built on it.
 * The float entry points evaluate the double kernel and round once, so they
 * are correctly rounded except within ~2^-50 of a rounding boundary.
 */
#pragma once
#include <stdint.h>
#include <math.h>
#if !defined(__CUDACC__)
#include <string.h>
#endif
#include "gf_math_consts.h"

#if defined(__CUDACC__)
#define GFM_HD __host__ __device__ __forceinline__
#else
#define GFM_HD static inline
#endif

namespace gfm {

GFM_HD uint64_t d2u(double x)
{
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u; memcpy(&u, &x, 8); return u;
#endif
}
GFM_HD double u2d(uint64_t u)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x; memcpy(&x, &u, 8); return x;
#endif
}
GFM_HD uint32_t f2u(float x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__float_as_uint(x);
#else
    uint32_t u; memcpy(&u, &x, 4); return u;
#endif
}
GFM_HD float u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x; memcpy(&x, &u, 4); return x;
#endif
}

GFM_HD double dfma(double a, double b, double c) { return ::fma(a, b, c); }
GFM_HD double drint(double x) { return ::rint(x); }   /* round half to even */
GFM_HD bool disnan(double x) { return x != x; }
GFM_HD double dinf() { return u2d(0x7ff0000000000000ull); }
GFM_HD double dnan() { return u2d(0x7ff8000000000000ull); }
GFM_HD float finf() { return u2f(0x7f800000u); }
GFM_HD float fnan() { return u2f(0x7fc00000u); }

/* 2^n for n in [-1022, 1023] */
GFM_HD double pow2i(int n) { return u2d((uint64_t)(n + 1023) << 52); }

/* exp(x) for double x */
GFM_HD double exp_d(double x)
{
    if (disnan(x)) return x;
    if (x > 709.782712893384) return dinf();
    if (x < -745.2) return 0.0;
    double n = drint(x * GFM_INV_LN2);
    double r = dfma(-n, GFM_LN2_HI, x);
    r = dfma(-n, GFM_LN2_LO, r);
    double p = GFM_EXP_C13;
    p = dfma(p, r, GFM_EXP_C12);
    p = dfma(p, r, GFM_EXP_C11);
    p = dfma(p, r, GFM_EXP_C10);
    p = dfma(p, r, GFM_EXP_C9);
    p = dfma(p, r, GFM_EXP_C8);
    p = dfma(p, r, GFM_EXP_C7);
    p = dfma(p, r, GFM_EXP_C6);
    p = dfma(p, r, GFM_EXP_C5);
    p = dfma(p, r, GFM_EXP_C4);
    p = dfma(p, r, GFM_EXP_C3);
    p = dfma(p, r, GFM_EXP_C2);
    p = dfma(p, r, GFM_EXP_C1);
    p = dfma(p, r, GFM_EXP_C0);
    int ni = (int)n;
    int n1 = ni / 2;
    int n2 = ni - n1;
    return (p * pow2i(n1)) * pow2i(n2);
}

/* natural log for double x */
GFM_HD double log_d(double x)
{
    if (disnan(x) || x < 0.0) return dnan();
    if (x == 0.0) return -dinf();
    if (x == dinf()) return x;
    uint64_t u = d2u(x);
    int e = (int)((u >> 52) & 0x7ff);
    if (e == 0) {                       /* subnormal: renormalise */
        x = x * 18014398509481984.0;    /* 2^54 */
        u = d2u(x);
        e = (int)((u >> 52) & 0x7ff) - 54;
    }
    e -= 1023;
    double m = u2d((u & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double s = (m - 1.0) / (m + 1.0);
    double z = s * s;
    double p = GFM_LOG_C11;
    p = dfma(p, z, GFM_LOG_C10);
    p = dfma(p, z, GFM_LOG_C9);
    p = dfma(p, z, GFM_LOG_C8);
    p = dfma(p, z, GFM_LOG_C7);
    p = dfma(p, z, GFM_LOG_C6);
    p = dfma(p, z, GFM_LOG_C5);
    p = dfma(p, z, GFM_LOG_C4);
    p = dfma(p, z, GFM_LOG_C3);
    p = dfma(p, z, GFM_LOG_C2);
    p = dfma(p, z, GFM_LOG_C1);
    p = dfma(p, z, GFM_LOG_C0);
    double lm = s * p;
    double de = (double)e;
    return dfma(de, GFM_LN2_HI, dfma(de, GFM_LN2_LO, lm));
}

/* sin(r), cos(r) for |r| <= pi/4 (plus rounding slack) */
GFM_HD double sin_poly(double r)
{
    double z = r * r;
    double p = GFM_SIN_C9;
    p = dfma(p, z, GFM_SIN_C8);
    p = dfma(p, z, GFM_SIN_C7);
    p = dfma(p, z, GFM_SIN_C6);
    p = dfma(p, z, GFM_SIN_C5);
    p = dfma(p, z, GFM_SIN_C4);
    p = dfma(p, z, GFM_SIN_C3);
    p = dfma(p, z, GFM_SIN_C2);
    p = dfma(p, z, GFM_SIN_C1);
    return dfma(r * z, p, r);           /* r + r^3 (C1 + C2 z + ...) */
}
GFM_HD double cos_poly(double r)
{
    double z = r * r;
    double p = GFM_COS_C9;
    p = dfma(p, z, GFM_COS_C8);
    p = dfma(p, z, GFM_COS_C7);
    p = dfma(p, z, GFM_COS_C6);
    p = dfma(p, z, GFM_COS_C5);
    p = dfma(p, z, GFM_COS_C4);
    p = dfma(p, z, GFM_COS_C3);
    p = dfma(p, z, GFM_COS_C2);
    p = dfma(p, z, GFM_COS_C1);
    return dfma(z, p, 1.0);
}

/* sin and cos of x (|x| < 2^19 pi/2 for full accuracy) */
GFM_HD void sincos_d(double x, double *s, double *c)
{
    if (disnan(x) || x == dinf() || x == -dinf()) { *s = dnan(); *c = dnan(); return; }
    double n = drint(x * GFM_TWO_OVER_PI);
    double r = dfma(-n, GFM_PIO2_1, x);
    r = dfma(-n, GFM_PIO2_2, r);
    r = dfma(-n, GFM_PIO2_3, r);
    double sr = sin_poly(r), cr = cos_poly(r);
    long long q = ((long long)n) & 3;
    if (q == 0)      { *s = sr;  *c = cr;  }
    else if (q == 1) { *s = cr;  *c = -sr; }
    else if (q == 2) { *s = -sr; *c = -cr; }
    else             { *s = -cr; *c = sr;  }
}
GFM_HD double sin_d(double x) { double s, c; sincos_d(x, &s, &c); return s; }
GFM_HD double cos_d(double x) { double s, c; sincos_d(x, &s, &c); return c; }

#if defined(__CUDACC__)
static __constant__ double gfm_atan_tab_hi_dev[9] = GFM_ATAN_TAB_HI_LIST;
static __constant__ double gfm_atan_tab_lo_dev[9] = GFM_ATAN_TAB_LO_LIST;
#endif

/* atan(t) for 0 <= t <= 1 */
GFM_HD double atan01(double t)
{
#if defined(__CUDA_ARCH__)
    const double *tab_hi = gfm_atan_tab_hi_dev;
    const double *tab_lo = gfm_atan_tab_lo_dev;
#else
    static const double tab_hi[9] = GFM_ATAN_TAB_HI_LIST;
    static const double tab_lo[9] = GFM_ATAN_TAB_LO_LIST;
#endif
    int i = (int)drint(t * 8.0);
    double c = (double)i * 0.125;
    double u = (t - c) / dfma(t, c, 1.0);
    double z = u * u;
    double p = GFM_ATAN_C7;
    p = dfma(p, z, GFM_ATAN_C6);
    p = dfma(p, z, GFM_ATAN_C5);
    p = dfma(p, z, GFM_ATAN_C4);
    p = dfma(p, z, GFM_ATAN_C3);
    p = dfma(p, z, GFM_ATAN_C2);
    p = dfma(p, z, GFM_ATAN_C1);
    double au = dfma(u * z, p, u);
    return tab_hi[i] + (tab_lo[i] + au);
}

GFM_HD double atan2_d(double y, double x)
{
    if (disnan(x) || disnan(y)) return dnan();
    bool ny = (d2u(y) >> 63) != 0;
    bool nx = (d2u(x) >> 63) != 0;
    double ay = ny ? -y : y, ax = nx ? -x : x;
    double a;
    if (ay == 0.0 && ax == 0.0) {
        a = 0.0;
    } else if (ax == dinf() && ay == dinf()) {
        a = atan01(1.0);                /* pi/4 */
    } else if (ay <= ax) {
        a = atan01(ay / ax);
    } else {
        a = (GFM_PIO2_HI - atan01(ax / ay)) + GFM_PIO2_LO;
    }
    if (nx) a = (GFM_PI_HI - a) + GFM_PI_LO;
    return ny ? -a : a;
}

GFM_HD double atan_d(double x)
{
    return atan2_d(x, 1.0);
}

GFM_HD double asin_d(double x)
{
    if (disnan(x) || x > 1.0 || x < -1.0) return dnan();
    double c = sqrt((1.0 - x) * (1.0 + x));
    return atan2_d(x, c);
}

/* ---------------- single-precision entry points ---------------- */

GFM_HD float expf_(float x) { return (float)exp_d((double)x); }
GFM_HD float logf_(float x) { return (float)log_d((double)x); }
GFM_HD float log10f_(float x) { return (float)(log_d((double)x) * GFM_INV_LN10); }
GFM_HD float exp10f_(float x) { return (float)exp_d((double)x * GFM_LN10_HI); }
GFM_HD float sinf_(float x) { return (float)sin_d((double)x); }
GFM_HD float cosf_(float x) { return (float)cos_d((double)x); }
GFM_HD float tanf_(float x)
{
    double s, c;
    sincos_d((double)x, &s, &c);
    return (float)(s / c);
}

/* true if the float y is an integer, and whether that integer is odd */
GFM_HD bool f_is_int(float y, bool *odd)
{
    float ay = y < 0.f ? -y : y;
    if (ay >= 16777216.f) { *odd = false; return true; }   /* >= 2^24: even integer */
    float t = (float)(int)ay;
    if (t != ay) { *odd = false; return false; }
    *odd = (((int)ay) & 1) != 0;
    return true;
}

/* powf(x, y) with the C99 special cases */
GFM_HD float powf_(float x, float y)
{
    if (y == 0.f) return 1.f;
    if (x == 1.f) return 1.f;
    if (x != x || y != y) return fnan();
    bool odd = false;
    bool yint = f_is_int(y, &odd);
    bool xneg = (f2u(x) >> 31) != 0;
    float ax = xneg ? -x : x;
    if (ax == 0.f) {
        float r = (y > 0.f) ? 0.f : finf();
        return (xneg && yint && odd) ? -r : r;
    }
    if (ax == finf()) {
        if (xneg) {
            float r = (y > 0.f) ? finf() : 0.f;
            return (yint && odd) ? -r : r;
        }
        return (y > 0.f) ? finf() : 0.f;
    }
    if (y == finf() || y == -finf()) {
        if (ax == 1.f) return 1.f;
        bool big = ax > 1.f;
        return ((y > 0.f) == big) ? finf() : 0.f;
    }
    if (xneg && !yint) return fnan();
    float r = (float)exp_d((double)y * log_d((double)ax));
    return (xneg && odd) ? -r : r;
}

} /* namespace gfm */
