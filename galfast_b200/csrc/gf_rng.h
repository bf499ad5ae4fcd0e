/*
 * gf_rng.h -- galfast's multiply-with-carry streams and the samplers built on
 * them, for host and device.
 *
 * Stream state (a, c, x) follows src/common/cuda_rng.h:414-463: one step is
 *     t = a*x + c (64-bit);  c = t >> 32;  x = t mod 2^32;
 * and returns the float 2.32830643708e-10f * (float)x.  With v = c*2^32 + x
 * the step is v' = a*x + c, and since a*2^32 = p + 1 with the safe prime
 * p = a*2^32 - 1, v' == a*v (mod p) with v' in [1, p-1] whenever v is: the
 * stream is a Lehmer generator modulo p.  That makes jump-ahead cheap:
 * after n steps v_n = a^n v_0 mod p.  mwc_mulmod() reduces a 128-bit product
 * modulo p with the same "a*lo + hi" folding the generator itself performs.
 *
 * The samplers restate src/common/cuda_rng.h:158-376 (GSL-derived Poisson,
 * Gaussian by the polar Box-Muller method, gamma, beta, binomial) with the
 * portable functions of gf_math.h, so host and device results agree.
 */
#pragma once
#include <stdint.h>
#include "gf_math.h"

#if defined(__CUDACC__)
#define GFR_HD __host__ __device__ __forceinline__
#else
#define GFR_HD static inline
#endif

namespace gfr {

/* The range of mu (and relative margin) within which the hardware __expf(-mu)
 * brackets the correctly rounded exp(-mu) (see poisson_small). */
#define GF_FASTEXP_MIN_MU (-0.01f)
#define GF_FASTEXP_MAX_MU 10.5f
#define GF_FASTEXP_MARGIN 1.0e-5f

/* 2.32830643708e-10f == 2^-32 exactly */
#define GF_MWC_SCALE 2.32830643708e-10f

struct Mwc {
    uint32_t a, c, x;
    uint32_t used;          /* uniforms drawn since the caller last cleared it */

    GFR_HD float uniform()
    {
        used++;
        uint64_t t = (uint64_t)a * x + c;
        c = (uint32_t)(t >> 32);
        x = (uint32_t)t;
        return GF_MWC_SCALE * (float)x;
    }
    GFR_HD uint64_t v() const { return ((uint64_t)c << 32) | x; }
    GFR_HD void set_v(uint64_t v) { c = (uint32_t)(v >> 32); x = (uint32_t)v; }
    GFR_HD uint64_t p() const { return ((uint64_t)a << 32) - 1; }

    /* uniform_pos: cuda_rng.h:158-163 */
    GFR_HD float uniform_pos()
    {
        float u;
        do { u = uniform(); } while (u == 0.f);
        return u;
    }

    /* gaussian: cuda_rng.h:165-182 (polar Box-Muller) */
    GFR_HD float gaussian(const float sigma)
    {
        float x, y, r2;
        do {
            x = -1.f + 2.f * uniform();
            y = -1.f + 2.f * uniform();
            r2 = x * x + y * y;
        } while (r2 > 1.0f || r2 == 0.f || r2 == 4.f);
        return sigma * y * sqrtf(-2.0f * gfm::logf_(r2) / r2);
    }

    /* gamma_large: cuda_rng.h:185-208 */
    GFR_HD float gamma_large(const float a_)
    {
        float sqa, xx, yy, vv;
        sqa = sqrtf(2 * a_ - 1);
        do {
            do {
                yy = gfm::tanf_((float)(3.14159265358979323846 * uniform()));
                xx = sqa * yy + a_ - 1;
            } while (xx <= 0);
            vv = uniform();
        } while (vv > (1 + yy * yy) * gfm::expf_((a_ - 1) * gfm::logf_(xx / (a_ - 1)) - sqa * yy));
        return xx;
    }

    /* gamma_int: cuda_rng.h:211-235 */
    GFR_HD float gamma_int(const unsigned int a_)
    {
        if (a_ < 3) {
            float prod = 1;
            for (unsigned int i = 0; i < a_; i++) prod *= uniform_pos();
            return -gfm::logf_(prod);
        }
        return gamma_large((float)a_);
    }

    /* gamma_frac: cuda_rng.h:238-264 (evaluated in double as in the reference's host build) */
    GFR_HD float gamma_frac(const float a_)
    {
        float p_, q, xx, u, vv;
        p_ = (float)(2.71828182845904523536 / (a_ + 2.71828182845904523536));
        do {
            u = uniform();
            vv = uniform_pos();
            if (u < p_) {
                xx = (float)gfm::exp_d((1 / a_) * gfm::log_d(vv));
                q = (float)gfm::exp_d(-xx);
            } else {
                xx = (float)(1 - gfm::log_d(vv));
                q = (float)gfm::exp_d((a_ - 1) * gfm::log_d(xx));
            }
        } while (uniform() >= q);
        return xx;
    }

    /* gamma: cuda_rng.h:276-297 */
    GFR_HD float gamma(const float a_, const float b_)
    {
        unsigned int na = (unsigned int)floorf(a_);
        if (a_ >= 4294967295.f) {
            return b_ * (gamma_large(floorf(a_)) + gamma_frac(a_ - floorf(a_)));
        } else if (a_ == (float)na) {
            return b_ * gamma_int(na);
        } else if (na == 0) {
            return b_ * gamma_frac(a_);
        } else {
            return b_ * (gamma_int(na) + gamma_frac(a_ - na));
        }
    }

    /* beta: cuda_rng.h:299-305 */
    GFR_HD float beta(const float a_, const float b_)
    {
        float x1 = gamma(a_, 1.0f);
        float x2 = gamma(b_, 1.0f);
        return x1 / (x1 + x2);
    }

    /* binomial (Knuth, via GSL): cuda_rng.h:308-340 */
    GFR_HD unsigned int binomial(float p_, unsigned int n)
    {
        unsigned int i, aa, bb, k = 0;
        while (n > 10) {
            float X;
            aa = 1 + (n / 2);
            bb = 1 + n - aa;
            X = beta((float)aa, (float)bb);
            if (X >= p_) {
                n = aa - 1;
                p_ /= X;
            } else {
                k += aa;
                n = bb - 1;
                p_ = (p_ - X) / (1 - X);
            }
        }
        for (i = 0; i < n; i++) {
            float u = uniform();
            if (u < p_) k++;
        }
        return k;
    }

    /* poisson: cuda_rng.h:344-376 */
    GFR_HD unsigned int poisson(float mu)
    {
        unsigned int k = 0;
        while (mu > 10) {
            unsigned int m = (unsigned int)(mu * (7.0 / 8.0));
            float X = gamma_int(m);
            if (X >= mu) {
                return k + binomial(mu / X, m - 1);
            } else {
                k += m;
                mu -= X;
            }
        }
        return k + poisson_small(mu);
    }

    /* the sampler's last stage (mu <= 10): multiply uniforms until the product
     * falls to exp(-mu) or below (cuda_rng.h:370-375) */
    GFR_HD unsigned int poisson_small(float mu)
    {
#ifdef __CUDA_ARCH__
        if (mu >= GF_FASTEXP_MIN_MU && mu <= GF_FASTEXP_MAX_MU) {
            /* exp(-mu) lies within GF_FASTEXP_MARGIN (relative) of the hardware
             * __expf(-mu) for every float mu in this range (checked exhaustively by
             * tests/cpp/expf_margin_check.cu), so a product outside the bracket is
             * decided without it; the correctly rounded value is formed only for a
             * product inside the bracket */
            const float ea = __expf(-mu);
            const float lo = ea * (1.0f - GF_FASTEXP_MARGIN), hi = ea * (1.0f + GF_FASTEXP_MARGIN);
            float prod = 1.0f, emu = -1.0f;
            unsigned int k = 0;
            for (;;) {
                prod *= uniform();
                k++;
                if (prod > hi) continue;
                if (prod <= lo) break;
                if (emu < 0.0f) emu = gfm::expf_(-mu);
                if (!(prod > emu)) break;
            }
            return k - 1;
        }
#endif
        const float emu = gfm::expf_(-mu);
        float prod = 1.0f;
        unsigned int k = 0;
        do {
            prod *= uniform();
            k++;
        } while (prod > emu);
        return k - 1;
    }
};

#ifdef __CUDACC__
/* u > exp(-mu), the sampler's first test (a bin has stars), decided with the
 * bracket of poisson_small when mu is in its range */
__device__ __forceinline__ bool exceeds_exp_neg(float u, float mu)
{
    if (mu >= GF_FASTEXP_MIN_MU && mu <= GF_FASTEXP_MAX_MU) {
        const float ea = __expf(-mu);
        if (u > ea * (1.0f + GF_FASTEXP_MARGIN)) return true;
        if (u <= ea * (1.0f - GF_FASTEXP_MARGIN)) return false;
    }
    return u > gfm::expf_(-mu);
}
#endif

/* The largest x in [0, 2^32) whose uniform 2^-32 * (float)x (x rounded to float,
 * to nearest even, then scaled exactly) is <= thr, or -1 when none is: a test
 * u <= thr on the next uniform becomes x <= threshold on the integer state,
 * without the conversion. */
GFR_HD int64_t uniform_threshold(float thr)
{
    if (!(thr >= 0.f)) return -1;
    const float T = thr * 4294967296.0f;               /* exact: scaling by 2^32 */
    if (T >= 4294967296.0f) return 0xffffffffll;
    if (T < 16777216.0f) return (int64_t)T;             /* below 2^24 every integer is a float */
    union { float f; uint32_t u; } cv;
    cv.f = T;
    const uint32_t bits = cv.u;
    const int e = (int)(bits >> 23) - 127;              /* 24 <= e <= 31 */
    const int64_t half = (int64_t)1 << (e - 24);        /* half the spacing of floats above T */
    /* x in (T, T + half) rounds down to T; x = T + half is a tie, kept by an even mantissa */
    return (int64_t)T + half - 1 + ((bits & 1u) ? 0 : 1);
}

/* A cheaper threshold for tests that only need to be safe: x <= X implies
 * 2^-32 * (float)x <= thr (X at most 3.6e-7 relative below uniform_threshold's);
 * -1 when thr <= 0.  For 0 < thr < 1: the scaling by 2^32 is exact, the factor
 * 1 - 2^-22 (rounded product within 2^-24) keeps X * (1 + 2^-24), the largest
 * float x rounds to, below thr * 2^32. */
GFR_HD int64_t uniform_threshold_lower(float thr)
{
    if (!(thr > 0.f)) return -1;
    if (thr >= 1.f) return 0xffffffffll;
    return (int64_t)(uint32_t)(thr * 4294967296.0f * 0.99999976f);
}

/* (a * b) mod p for the stream prime p = A*2^32 - 1, a, b < p.
 * The 128-bit product N is folded with N -> A*(N mod 2^32) + (N >> 32), which
 * multiplies the residue by 2^-32 (mod p); the caller pre-scales one operand
 * by 2^96 (three folds).  Result in [0, p). */
GFR_HD uint64_t mwc_fold3(uint64_t lo, uint64_t hi, uint32_t A, uint64_t p)
{
    /* N = hi*2^64 + lo  (< 2^127) */
    /* fold 1: A*(N mod 2^32) + (N >> 32): N >> 32 is 96 bits = (hi << 32) | (lo >> 32) */
    uint64_t l0 = lo & 0xffffffffull;
    uint64_t s_lo = (lo >> 32) | (hi << 32);     /* low 64 bits of N >> 32 */
    uint64_t s_hi = hi >> 32;                    /* bits 64..95 of N >> 32 */
    uint64_t prod = (uint64_t)A * l0;
    uint64_t r_lo = s_lo + prod;
    uint64_t r_hi = s_hi + (r_lo < prod ? 1 : 0);
    /* fold 2: value (r_hi, r_lo) < 2^97 */
    l0 = r_lo & 0xffffffffull;
    s_lo = (r_lo >> 32) | (r_hi << 32);
    s_hi = r_hi >> 32;
    prod = (uint64_t)A * l0;
    r_lo = s_lo + prod;
    r_hi = s_hi + (r_lo < prod ? 1 : 0);
    /* fold 3: value < 2^66 */
    l0 = r_lo & 0xffffffffull;
    s_lo = (r_lo >> 32) | (r_hi << 32);
    prod = (uint64_t)A * l0;
    uint64_t r = s_lo + prod;                    /* < A*2^32 + 2^34 <= p + 2^34 + 1, fits 64 bits */
    if (r >= p) r -= p;
    return r;
}

GFR_HD void mul64x64(uint64_t a, uint64_t b, uint64_t *lo, uint64_t *hi)
{
#if defined(__CUDA_ARCH__)
    *lo = a * b;
    *hi = __umul64hi(a, b);
#else
    unsigned __int128 t = (unsigned __int128)a * b;
    *lo = (uint64_t)t;
    *hi = (uint64_t)(t >> 64);
#endif
}

/* (m * v) mod p where m_s = m * 2^96 mod p is the pre-scaled multiplier */
GFR_HD uint64_t mwc_mulmod_scaled(uint64_t m_s, uint64_t v, uint32_t A, uint64_t p)
{
    uint64_t lo, hi;
    mul64x64(m_s, v, &lo, &hi);
    return mwc_fold3(lo, hi, A, p);
}

/* plain modular multiply (slow path, host setup): (x * y) mod p */
GFR_HD uint64_t mulmod_generic(uint64_t x, uint64_t y, uint64_t p)
{
#if defined(__CUDA_ARCH__)
    /* double-and-add; only used off the hot path */
    uint64_t r = 0;
    x %= p; y %= p;
    while (y) {
        if (y & 1) { r += x; if (r >= p || r < x) r -= p; }
        uint64_t x2 = x + x;
        if (x2 >= p || x2 < x) x2 -= p;
        x = x2;
        y >>= 1;
    }
    return r;
#else
    return (uint64_t)((unsigned __int128)x * y % p);
#endif
}

} /* namespace gfr */
