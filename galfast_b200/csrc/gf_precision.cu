/*
 * gf_precision.cu -- the precision form: the expected counts of every
 * (pixel, m, M) bin evaluated twice, as the catalog path evaluates them (FP32,
 * the reference's float expressions) and in FP64, over the same
 * discretisation (the same LF texels, the same anchor bins: block starts and
 * diagonal starts of the crawl, skygen.cu.h:216-229, 541-565).  The per-bin
 * statistics cover the bins with at least 1e-30 expected stars.
 *
 * One warp per pixel; lane l takes the pixel's blocks l, l + 32, ...  Per pixel
 * the FP32 values are summed with Kahan compensation in FP32 and the FP64
 * values in FP64; per bin the relative difference is accumulated (max, sum,
 * count) and the FP64 counts are histogrammed by distance-modulus row
 * (d = im + iM, constant DM along a diagonal when dm = dM).
 */
#include "gf_crawl.cuh"
#include "gf_launch.h"

namespace gfk {

namespace {

/* x^y in double, with pow's result for a negative x and an integer y */
__device__ __forceinline__ double pow_fp64(double x, double y)
{
    if (x == 0.0) return y > 0.0 ? 0.0 : __longlong_as_double(0x7ff0000000000000ll);
    if (x > 0.0) return gfm::exp_d(y * gfm::log_d(x));
    if (y != rint(y)) return __longlong_as_double(0x7ff8000000000000ll);
    const double r = gfm::exp_d(y * gfm::log_d(-x));
    return fmod(fabs(y), 2.0) == 1.0 ? -r : r;
}

/* the anchor quantities of the bin (ilb, im, iM) in FP64 */
template <int MODEL>
__device__ void anchor_fp64(const SkyModel &m, const SkyGeom &g, int ilb, int im, int iM, double &ms, double &D3, double &K)
{
    const gf_pencil_beam pix = g.pixels[ilb];
    const double M = (double)m.M1 - (double)iM * (double)m.dM;
    const double mm = (double)m.m0 + (double)im * (double)m.dm;
    const double D = gfm::exp_d((0.2 * (mm - M) + 1.0) * 2.30258509299404568401799145468);
    const double x = D * (double)pix.cl * (double)pix.cb, y = D * (double)pix.sl * (double)pix.cb, z = D * (double)pix.sb;
    const double vx = x + m.T[0], vy = y + m.T[1], vz = z + m.T[2];
    const double wx = m.M[0] * vx + m.M[1] * vy + m.M[2] * vz;
    const double wy = m.M[3] * vx + m.M[4] * vy + m.M[5] * vz;
    const double wz = m.M[6] * vx + m.M[7] * vy + m.M[8] * vz;
    if (MODEL == GF_MODEL_EXP_DISK) {
        const double r2 = wx * wx + wy * wy;
        if (m.r_cut2 != 0.f && r2 + wz * wz > (double)m.r_cut2) ms = 0.0;
        else ms = (double)m.f * gfm::exp_d(-sqrt(r2) / (double)m.l - fabs(wz) / (double)m.h);
    } else if (m.type == GF_MODEL_DENSITY_CUBE) {
        /* the grid holds float values: the same texel as the float path */
        ms = (double)m.f * (double)gfc::cube_sample(m, (float)wx, (float)wy, (float)wz);
    } else if (m.type == GF_MODEL_LCBULGE) {
        const double n = (double)m.n;
        const double t = pow_fp64(pow_fp64(wx, n) + pow_fp64(wy / (double)m.ba, n) + pow_fp64(wz / (double)m.ca, n), 1.0 / n);
        ms = gfm::exp_d(-t / (double)m.l);
    } else {
        const double DSq = wx * wx + wy * wy + wz * wz;
        if (m.rmaxSq != 0.f && (DSq < (double)m.rminSq || DSq >= (double)m.rmaxSq)) {
            ms = 0.0;
        } else {
            const double ty = wy / (double)m.ba, tz = wz / (double)m.ca;
            const double rSq = wx * wx + ty * ty + tz * tz;
            int k = 0;
            while (k != m.nbreaks && rSq > (double)m.rbreakSq[k]) k++;
            ms = (double)m.f * (double)m.fArr[k] * gfm::exp_d(0.5 * (double)m.nArr[k] * gfm::log_d(rSq));
        }
    }
    D3 = D * D * D;
    K = (double)pix.dA * 0.46051701859880913680 * (double)m.dm * (double)m.dM;
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v)
{
    /* non-negative doubles order like their bit patterns */
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

template <int MODEL>
__global__ void __launch_bounds__(128) precision_kernel(SkyModel m, SkyGeom g, const float *Dtab, FastDiv fx, FastDiv fy,
                                                         double *pix32, double *pix64, double *hist64,
                                                         unsigned long long *max_rel, double *sum_rel,
                                                         unsigned long long *nbins)
{
    extern __shared__ double s_hist[];
    const int x = m.nm, y = m.nM, kmax = x * y, nd = x + y - 1;
    for (int q = threadIdx.x; q < nd; q += blockDim.x) s_hist[q] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    double rel_max = 0.0, rel_sum = 0.0;
    unsigned long long count = 0;
    for (int ilb = warp; ilb < g.npixels; ilb += nwarps) {
        float s32 = 0.f, c32 = 0.f;          /* Kahan sum of the FP32 counts */
        double s64 = 0.0;
        for (int k0 = GF_BLOCK * lane; k0 < kmax; k0 += GF_BLOCK * 32) {
            int ci, cj;
            gfc::diag_to_ij_fast(k0, x, y, fx, fy, ci, cj);
            AnchorX A;
            double ms64 = 0, D364 = 0, K64 = 0;
            for (int s = 0; s < GF_BLOCK; s++) {
                bool anchor = (s == 0);
                if (s > 0) anchor = gfc::step_in_pixel(ci, cj, x, y);
                if (anchor) {
                    A = gfc::anchor_x<MODEL>(m, g, Dtab, ilb, ci, cj);
                    anchor_fp64<MODEL>(m, g, ilb, ci, cj, ms64, D364, K64);
                }
                const float M = m.M1 - (float)cj * m.dM;
                const float lfv = gfc::lf_sample(m, m.lf, M);
                const float mrow = m.m0 + m.dm * (float)ci;
                const float mu = gfc::bin_mu_x(A, lfv, mrow, m.norm, m.m1);
                if (gfc::is_cut(mu)) continue;
                const double mu64 = (double)lfv * ms64 * (double)m.norm * D364 * K64;
                /* Kahan: s32 + mu with the lost low part carried in c32 */
                const float yk = mu - c32;
                const float tk = s32 + yk;
                c32 = (tk - s32) - yk;
                s32 = tk;
                s64 += mu64;
                /* relative error over bins with at least 1e-30 expected stars: below that the
                 * reference's float expressions pass through subnormal intermediates (the model
                 * density far out in the disk), which keep only a few significant bits */
                if (fabs(mu64) >= 1e-30) {
                    const double r = fabs((double)mu - mu64) / fabs(mu64);
                    rel_max = r > rel_max ? r : rel_max;
                    rel_sum += r;
                    count++;
                }
                atomicAdd(&s_hist[ci + cj], mu64);
            }
        }
        double t32 = (double)s32 - (double)c32, t64 = s64;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            t32 += __shfl_xor_sync(0xffffffffu, t32, o);
            t64 += __shfl_xor_sync(0xffffffffu, t64, o);
        }
        if (lane == 0) {
            pix32[ilb] = t32;
            pix64[ilb] = t64;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double om = __shfl_xor_sync(0xffffffffu, rel_max, o);
        rel_max = om > rel_max ? om : rel_max;
        rel_sum += __shfl_xor_sync(0xffffffffu, rel_sum, o);
        count += __shfl_xor_sync(0xffffffffu, count, o);
    }
    if (lane == 0) {
        atomic_max_pos(max_rel, rel_max);
        atomicAdd(sum_rel, rel_sum);
        atomicAdd(nbins, count);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nd; q += blockDim.x)
        if (s_hist[q] != 0.0) atomicAdd(&hist64[q], s_hist[q]);
}

}  // namespace

cudaError_t launch_precision(const SkyModel &m, const SkyGeom &g, const float *Dtab, double *pix32, double *pix64,
                             double *hist64, unsigned long long *max_rel, double *sum_rel, unsigned long long *nbins,
                             cudaStream_t s)
{
    const int nd = m.nm + m.nM - 1;
    const size_t smem = sizeof(double) * (size_t)nd;
    if (smem > 48 * 1024) return cudaErrorInvalidValue;
    int blocks = (int)std::min<int64_t>(((int64_t)g.npixels + 3) / 4, (int64_t)sm_count() * 8);
    if (blocks < 1) blocks = 1;
    const FastDiv fx = make_fastdiv((uint32_t)m.nm), fy = make_fastdiv((uint32_t)m.nM);
    if (m.type == GF_MODEL_EXP_DISK)
        precision_kernel<GF_MODEL_EXP_DISK><<<blocks, 128, smem, s>>>(m, g, Dtab, fx, fy, pix32, pix64, hist64, max_rel, sum_rel, nbins);
    else
        precision_kernel<GF_MODEL_POWER_LAW_ELLIPSOID><<<blocks, 128, smem, s>>>(m, g, Dtab, fx, fy, pix32, pix64, hist64, max_rel, sum_rel, nbins);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace gfk
