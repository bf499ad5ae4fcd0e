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

/* diag_to_ij with the divisions of the middle region done by FastDiv. */
__device__ __forceinline__ void diag_to_ij_fast(int k, const int x, const int y, const FastDiv &fx, const FastDiv &fy,
                                                int &i, int &j)
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
            int q = (int)((__umulhi((uint32_t)ka, fy.mul) + (uint32_t)ka) >> fy.shift);
            d = q + (y - 1);
            i = (ka - q * y) + d - (y - 1);
        } else {
            int ka = k - x * (x - 1) / 2;
            int q = (int)((__umulhi((uint32_t)ka, fx.mul) + (uint32_t)ka) >> fx.shift);
            d = q + (x - 1);
            i = ka - q * x;
        }
    } else {
        int ka = x * y - k - 1;
        int dd = int(0.5 * (double)(sqrtf((float)(1 + 8 * ka)) - 1));
        d = (x + y - 2) - dd;
        i = (x - 1) - (ka - dd * (dd + 1) / 2);
    }
    j = d - i;
}

/* One step along the bin order inside a pixel: the next bin on the diagonal,
 * or the first bin of the next diagonal d+1 = i+j+1, which starts at
 * i = max(0, d+1 - (y-1)) (the same successor advance() computes, minus the
 * pixel change).  Returns whether a new diagonal starts. */
__device__ __forceinline__ bool step_in_pixel(int &i, int &j, const int x, const int y)
{
    int ni = i + 1, nj = j - 1;
    bool wrap = (nj < 0) | (ni >= x);
    if (wrap) {
        int d1 = i + j + 1;
        ni = d1 - (y - 1);
        ni = ni > 0 ? ni : 0;
        nj = d1 - ni;
    }
    i = ni;
    j = nj;
    return wrap;
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
__device__ __forceinline__ float beam_extinction(const SkyGeom &g, const gf_pencil_beam &pix)
{
    if (g.ext_kind == GF_EXT_NONE || g.ammin == nullptr) return 0.f;
    return g.ammin[pix.extIdx];
}

/* nearest texel index of coordinate v on an axis of n texels (cux.h:800-809, 860-874) */
__host__ __device__ __forceinline__ uint32_t tex_index(float v, float x0, float inv_dx, int n)
{
    float t = (v - x0) * inv_dx + 0.5f;
    if (t < 0.f) t = 0.f;
    else if (t >= (float)n) t = (float)(n - 1);
    return (uint32_t)t;
}

/* the anchor's extinction at distance modulus DM (compute_pos, skygen.cu.h:216-229):
 * the beam's row of minima at the nearest DM texel with 3-D maps, else the beam's value */
__device__ __forceinline__ float beam_extinction_dm(const SkyGeom &g, const gf_pencil_beam &pix, float DM)
{
    if (g.ext_kind != GF_EXT_MAPS) return beam_extinction(g, pix);
    if (g.ammin == nullptr) return 0.f;
    const uint32_t k = tex_index(DM, g.ext_tcz[0], g.ext_tcz[1], g.ext_nz);
    return g.ammin[(size_t)pix.extIdx * (size_t)g.ext_nz + k];
}

/* sampleExtinction (skygen.cu.h:199-208): the map of hemisphere proj at (X, Y, DM) */
__device__ __forceinline__ float map_extinction(const SkyGeom &g, int proj, float X, float Y, float DM)
{
    const float *A = g.map[proj];
    if (A == nullptr) return 0.f;
    const int32_t *n = g.map_n[proj];
    const uint32_t i = tex_index(X, g.map_tc[proj][0][0], g.map_tc[proj][0][1], n[0]);
    const uint32_t j = tex_index(Y, g.map_tc[proj][1][0], g.map_tc[proj][1][1], n[1]);
    const uint32_t k = tex_index(DM, g.map_tc[proj][2][0], g.map_tc[proj][2][1], n[2]);
    return A[((size_t)k * (size_t)n[1] + j) * (size_t)n[0] + i];
}

/* nearest-texel sample of a model's density cube (cux.h:800-809, 860-874) */
__host__ __device__ __forceinline__ float cube_sample(const SkyModel &m, float x, float y, float z)
{
    const float c[3] = {x, y, z};
    uint32_t ix[3];
    for (int a = 0; a < 3; a++) {
        float t = (c[a] - m.cube_tc[a][0]) * m.cube_tc[a][1] + 0.5f;
        if (t < 0.f) t = 0.f;
        else if (t >= (float)m.cube_n[a]) t = (float)(m.cube_n[a] - 1);
        ix[a] = (uint32_t)t;
    }
    return m.cube[((size_t)ix[2] * (size_t)m.cube_n[1] + ix[1]) * (size_t)m.cube_n[0] + ix[0]];
}

/* Model density at the heliocentric position (x, y, z); MODEL is the
 * compile-time model kind (GF_MODEL_EXP_DISK or GF_MODEL_POWER_LAW_ELLIPSOID). */
template <int MODEL>
__device__ __forceinline__ float model_rho(const SkyModel &m, float x, float y, float z)
{
    float vx = x + m.T[0], vy = y + m.T[1], vz = z + m.T[2];
    float wx = m.M[0] * vx + m.M[1] * vy + m.M[2] * vz;
    float wy = m.M[3] * vx + m.M[4] * vy + m.M[5] * vz;
    float wz = m.M[6] * vx + m.M[7] * vy + m.M[8] * vz;
    if (MODEL == GF_MODEL_EXP_DISK) {
        float r2 = wx * wx + wy * wy;
        if (m.r_cut2 != 0.f && r2 + wz * wz > m.r_cut2) return 0.f;
        float r = sqrtf(r2);
        return m.f * gfm::expf_(-r / m.l - fabsf(wz) / m.h);
    } else if (m.type == GF_MODEL_DENSITY_CUBE) {
        /* densityCube::setpos (model_densityCube.h:60-66): the frame gives (Rg - x, -y, z);
         * nearest texel of the grid */
        return m.f * cube_sample(m, wx, wy, wz);
    } else if (m.type == GF_MODEL_LCBULGE) {
        /* LCBulge::rho (model_LCBulge.h:79-92): no density factor (the LF carries f) */
        const float t = gfm::powf_(gfm::powf_(wx, m.n) + gfm::powf_(wy / m.ba, m.n) + gfm::powf_(wz / m.ca, m.n),
                                   (float)(1. / m.n));
        return gfm::expf_(-t / m.l);
    } else {
        /* powerLawEllipsoid::rho (model_powerLawEllipsoid.h:60-92) and brokenPowerLaw::rho
         * (model_brokenPowerLaw.h:55-82): f fArr[k] rSq^(nArr[k] / 2) beyond k breaks */
        float DSq = wx * wx + wy * wy + wz * wz;
        if (m.rmaxSq != 0.f && (DSq < m.rminSq || DSq >= m.rmaxSq)) return 0.f;
        float ty = wy / m.ba, tz = wz / m.ca;
        float rSq = wx * wx + ty * ty + tz * tz;
        int k = 0;
        while (k != m.nbreaks && rSq > m.rbreakSq[k]) k++;
        return m.f * m.fArr[k] * gfm::powf_(rSq, 0.5f * m.nArr[k]);
    }
}

/* Distance of the bin (im, iM): DM = (m0 + im dm) - (M1 - iM dM), D = powf(10, 0.2 DM + 1)
 * (skygen.cu.h:219-222).  After advance() leaves a pixel the reference keeps
 * crawling with im >= nm ("garbage" bins of a block that straddles two pixels);
 * those are evaluated directly instead of from the table. */
__device__ __forceinline__ float bin_distance(const SkyModel &m, const float *Dtab, int im, int iM)
{
    if ((unsigned)im < (unsigned)m.nm && (unsigned)iM < (unsigned)m.nM) return Dtab[im * m.nM + iM];
    const float M = m.M1 - (float)iM * m.dM;
    const float mm = m.m0 + (float)im * m.dm;
    return gfm::powf_(10.f, 0.2f * (mm - M) + 1.f);
}

/* Anchor quantities in the per-bin form (AnchorX) for the bin (ilb, im, iM). */
template <int MODEL>
__device__ __forceinline__ AnchorX anchor_x(const SkyModel &m, const SkyGeom &g, const float *Dtab, int ilb, int im, int iM)
{
    const gf_pencil_beam pix = g.pixels[ilb];
    AnchorX a;
    const float D = bin_distance(m, Dtab, im, iM);
    float Am;
    if (g.ext_kind == GF_EXT_MAPS) {
        /* the distance modulus as compute_pos forms it: m = m0 + im dm, DM = m - M */
        const float M = m.M1 - (float)iM * m.dM;
        const float mm = m.m0 + (float)im * m.dm;
        Am = beam_extinction_dm(g, pix, mm - M);
    } else {
        Am = beam_extinction(g, pix);
    }
    float x = D * pix.cl * pix.cb;
    float y = D * pix.sl * pix.cb;
    float z = D * pix.sb;
    a.ms = model_rho<MODEL>(m, x, y, z);
    const bool dcut = (m.dmin != 0.f || m.dmax != 0.f) && (m.dmin > D || m.dmax <= D);
    a.Am = dcut ? __int_as_float(0x7f800000) : Am;
    a.D3 = D * D * D;
    a.K = pix.dA * GF_POGSON * m.dm * m.dM;
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

/* Expected count of a bin from its anchor, the LF value at its absolute
 * magnitude and m0 + dm*im (the two per-model tables), or the cut marker. */
__device__ __forceinline__ float bin_mu_x(const AnchorX &a, float lfv, float mrow, float norm, float m1)
{
    float rho = lfv * a.ms;
    rho *= norm;
    rho *= a.D3;
    rho *= a.K;
    return (mrow + a.Am > m1) ? cut_marker() : rho;
}

}  // namespace gfc
