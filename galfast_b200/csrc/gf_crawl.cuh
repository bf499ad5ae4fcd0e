/*
 * gf_crawl.cuh -- device functions of the skygen crawl: the (pixel, m, M) bin
 * enumeration, the per-diagonal anchor quantities and the per-bin expected
 * count, written for lane-parallel evaluation on sm_100a.
 *
 * The bin order, anchors and float expressions follow
 * src/skygen/skygen.cu.h:216-358 and :469-565 exactly; the arrangement (one
 * warp per stream, one lane per block of 10 bins) is this library's.
 */
#pragma once
#include "gf_internal.h"
#include "gf_math.h"

namespace gfc {

/* diagIndexToIJ (skygen.cu.h:257-300) for a local index 0 <= k < x*y. */
__device__ __forceinline__ void diag_to_ij(int k, const int x, const int y, int &i, int &j)
{
    int l = x < y ? x : y;
    int m = x < y ? y : x;
    int d;
    if (2 * k < l * (l - 1)) {
        d = int(0.5 * (double)(sqrtf((float)(1 + 8 * k)) - 1));
        i = k - d * (d + 1) / 2;
    } else if (2 * k < l * (2 * m + 1 - l)) {
        if (x >= y) {
            int ka = k - y * (y - 1) / 2;
            d = ka / y + (y - 1);
            i = (ka % y) + d - (y - 1);
        } else {
            int ka = k - x * (x - 1) / 2;
            d = ka / x + (x - 1);
            i = ka % x;
        }
    } else {
        int ka = x * y - k - 1;
        int dd = int(0.5 * (double)(sqrtf((float)(1 + 8 * ka)) - 1));
        d = (x + y - 2) - dd;
        i = (x - 1) - (ka - dd * (dd + 1) / 2);
    }
    j = d - i;
}

/* advance (skygen.cu.h:307-358) without the pixel reload: returns whether the
 * step moved to a new diagonal; *pix_inc is set when the pixel index grows. */
__device__ __forceinline__ bool advance(int &i, int &j, const int x, const int y, bool &pix_inc)
{
    pix_inc = false;
    i++; j--;
    if (j < 0) {
        if (i < y) { j += i + 1; i = 0; }
        else { i -= (y - 1); j += y; }
    } else if (i >= x) {
        if (x > y) {
            i -= y - j - 2; j = y - 1;
        } else {
            if (j + 1 < y - x) { i -= x; j += x + 1; }
            else { i = x - y + j + 2; j = y - 1; }
        }
        if (i == x) pix_inc = true;
    } else {
        return false;
    }
    return true;
}

/* Number of pixel increments inside the block starting at local index k0
 * (nonzero only when the block runs past the end of a pixel, which happens
 * when nm*nM is not a multiple of 10). */
__device__ __forceinline__ int block_drift(int k0, const int x, const int y)
{
    if (k0 + GF_BLOCK - 1 < x * y) return 0;
    int i, j, drift = 0;
    diag_to_ij(k0, x, y, i, j);
    for (int s = 1; s < GF_BLOCK; s++) {
        bool inc;
        advance(i, j, x, y, inc);
        drift += inc ? 1 : 0;
    }
    return drift;
}

/* Anchor quantities of a bin (compute_pos + Model::setpos, skygen.cu.h:216-229,
 * model_expDisk.h:71-115, model_powerLawEllipsoid.h:60-99). */
struct Anchor {
    float D, Am, ms;
};

__device__ __forceinline__ float beam_extinction(const SkyGeom &g, const gf_pencil_beam &pix)
{
    if (g.ext_kind == GF_EXT_NONE || g.ammin == nullptr) return 0.f;
    return g.ammin[pix.extIdx];
}

__device__ __forceinline__ float model_rho(const SkyModel &m, float x, float y, float z)
{
    float vx = x + m.T[0], vy = y + m.T[1], vz = z + m.T[2];
    float wx = m.M[0] * vx + m.M[1] * vy + m.M[2] * vz;
    float wy = m.M[3] * vx + m.M[4] * vy + m.M[5] * vz;
    float wz = m.M[6] * vx + m.M[7] * vy + m.M[8] * vz;
    if (m.type == GF_MODEL_EXP_DISK) {
        float r2 = wx * wx + wy * wy;
        if (m.r_cut2 != 0.f && r2 + wz * wz > m.r_cut2) return 0.f;
        float r = sqrtf(r2);
        return m.f * gfm::expf_(-r / m.l - fabsf(wz) / m.h);
    } else {
        float DSq = wx * wx + wy * wy + wz * wz;
        if (m.rmaxSq != 0.f && (DSq < m.rminSq || DSq >= m.rmaxSq)) return 0.f;
        float ty = wy / m.ba, tz = wz / m.ca;
        float rSq = wx * wx + ty * ty + tz * tz;
        return m.f * gfm::powf_(rSq, 0.5f * m.n);
    }
}

__device__ __forceinline__ Anchor compute_anchor(const SkyModel &m, const SkyGeom &g, const gf_pencil_beam &pix, int im, float M)
{
    Anchor a;
    float mm = m.m0 + (float)im * m.dm;
    float DM = mm - M;
    a.D = gfm::powf_(10.f, 0.2f * DM + 1.f);
    a.Am = beam_extinction(g, pix);
    float x = a.D * pix.cl * pix.cb;
    float y = a.D * pix.sl * pix.cb;
    float z = a.D * pix.sb;
    a.ms = model_rho(m, x, y, z);
    return a;
}

/* Nearest-texel LF lookup (cux.h:778-792, 849-855) from an LF copy in shared memory. */
__device__ __forceinline__ float lf_sample(const SkyModel &m, const float *lf, float Mabs)
{
    float xi = (Mabs - m.lf_x0) * m.lf_inv_dx + 0.5f;
    if (xi < 0.f) xi = 0.f;
    else if (xi >= (float)m.lf_n) xi = (float)m.lf_n - 1;
    return lf[(uint32_t)xi];
}

/* A cut bin is marked with a NaN payload that no arithmetic produces: a real
 * bin's mu can be a tiny negative number (LF extrapolation) or a computed NaN. */
__device__ __forceinline__ float cut_marker() { return __int_as_float(0x7fc0dead); }
__device__ __forceinline__ bool is_cut(float mu) { return __float_as_int(mu) == 0x7fc0dead; }

/* Expected count of a bin, or the cut marker if the bin is cut (skygen.cu.h:551-565). */
__device__ __forceinline__ float bin_mu(const SkyModel &m, const float *lf, const Anchor &a, float dA, int im, float M)
{
    if ((m.dmin != 0.f || m.dmax != 0.f) && (m.dmin > a.D || m.dmax <= a.D)) return cut_marker();
    float mm = m.m0 + m.dm * (float)im + a.Am;
    if (mm > m.m1) return cut_marker();
    float rho = lf_sample(m, lf, M) * a.ms;
    rho *= m.norm;
    rho *= a.D * a.D * a.D;
    rho *= dA * GF_POGSON * m.dm * m.dM;
    return rho;
}


}  // namespace gfc
