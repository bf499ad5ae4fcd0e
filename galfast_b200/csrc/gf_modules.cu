/*
 * gf_modules.cu -- sm_100a kernels of the postprocessing modules on the
 * catalog path.  Each restates the reference kernel named beside it with the
 * portable math of gf_math.h; expressions keep the reference's types and
 * evaluation order (the library is compiled with -fmad=false).
 *
 *   clipper_kernel     os_clipper::process (src/skygen/os_skygen.cpp:999-1044), analytic footprints
 *   fixedfeh_kernel    os_fixedFeH_kernel (src/modules/fixedFeH_gpu.cu.h:34-50)
 *   feh_kernel<0>      os_FeH_kernel (src/modules/FeH_gpu.cu.h:43-87)
 *   feh_kernel<1>      os_GaussianFeH_kernel (src/modules/GaussianFeH_gpu.cu.h:42-73)
 *   bond2010_kernel    os_Bond2010_kernel (src/modules/Bond2010_gpu.cu.h:81-218)
 *   photometry_kernel  os_photometry_kernel (src/modules/photometry_gpu.cu.h:87-174)
 *   photoerr_kernel    os_photometricErrors::process (photometricErrors_host.cpp:112-131)
 *   vel2pm_kernel      os_vel2pm_kernel (src/modules/vel2pm_gpu.cu.h:253-301)
 *   gal2other_kernel   os_gal2other_kernel (src/modules/gal2other_gpu.cu.h:62-96)
 */
#include "gf_launch.h"
#include "gf_math.h"
#include "gf_rng.h"
#include "gf_footprint.h"

namespace gfk {

static const double D2R = 0.01745329251994329576923691;

static int grid_for(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    int64_t cap = (int64_t)sm_count() * 32;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

/* ---------------- sampler check: Poisson deviates of one stream ---------------- */
/* rng_t::poisson (cuda_rng.h:344-376) applied to mu[0..n) one after another on a
 * single stream: the device form of the sampler, including the gamma_int /
 * binomial reduction for mu > 10 that catalog bins rarely reach. */
__global__ void poisson_stream_kernel(uint32_t *st, const float *mu, int32_t n, uint32_t *out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    gfr::Mwc r;
    r.a = st[0]; r.c = st[1]; r.x = st[2]; r.used = 0;
    for (int32_t i = 0; i < n; i++) out[i] = r.poisson(mu[i]);
    st[0] = r.a; st[1] = r.c; st[2] = r.x;
}

cudaError_t launch_poisson_stream(uint32_t *st, const float *mu, int32_t n, uint32_t *out, cudaStream_t s)
{
    poisson_stream_kernel<<<1, 32, 0, s>>>(st, mu, n, out);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- clipper ---------------- */
__device__ __forceinline__ void clip_row(const gf_footprint &foot, gf_table &t, int64_t row)
{
    const int64_t P = t.capacity;
    if (t.hidden[row]) return;
    bool in = true;
        if (foot.kind == GF_FOOT_LAMBERT_RECT) {
            float x = t.projXY[row], y = t.projXY[P + row];
            in = t.projIdx[row] == foot.proj && x >= foot.a && x < foot.b && y >= foot.c && y < foot.d;
        } else if (foot.kind == GF_FOOT_CAP) {
            double l = t.lb[row] * D2R, b = t.lb[P + row] * D2R;
            double l0 = foot.a * D2R, b0 = foot.b * D2R;
            double cosd = gfm::sin_d(b) * gfm::sin_d(b0) + gfm::cos_d(b) * gfm::cos_d(b0) * gfm::cos_d(l - l0);
            in = cosd >= gfm::cos_d(foot.c * D2R);
        } else if (foot.kind == GF_FOOT_LATCUT) {
            in = fabs(t.lb[P + row]) > foot.a;
        } else if (foot.kind == GF_FOOT_LB_RECT) {
            const double l = t.lb[row], b = t.lb[P + row];
            in = b >= foot.c && b < foot.d && ((foot.a <= foot.b) ? (l >= foot.a && l < foot.b) : (l >= foot.a || l < foot.b));
        } else if (foot.kind == GF_FOOT_REGIONS) {
            in = gff::regions_inside(foot, t.lb[row], t.lb[P + row]);
        }
        if (!in) t.hidden[row] = 1;
}

__global__ void clipper_kernel(gf_footprint foot, gf_table t, int64_t begin, int64_t end)
{
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x)
        clip_row(foot, t, row);
}

/* each row clipped by its own request's footprint */
__global__ void clipper_multi_kernel(const gf_footprint *foot_by_job, MultiRows R, gf_table t, int64_t begin, int64_t end)
{
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        const gf_footprint &f = foot_by_job[R.slot_job[R.row_slot[row]]];
        if (f.kind != GF_FOOT_ALL) clip_row(f, t, row);
    }
}

cudaError_t launch_clipper_multi(const gf_footprint *foot_by_job, MultiRows R, gf_table t, int64_t begin, int64_t end,
                                 cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    clipper_multi_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(foot_by_job, R, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_clipper(const gf_footprint &foot, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin || foot.kind == GF_FOOT_ALL) return cudaSuccess;
    clipper_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(foot, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- fixedFeH ---------------- */
__global__ void fixedfeh_kernel(gf_fixedfeh_config c, gf_table t, int64_t begin, int64_t end)
{
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        if (t.hidden[row]) continue;
        int cmp = t.comp[row];
        if (!((c.comp_mask >> cmp) & 1u)) continue;
        t.FeH[row] = c.FeH;
    }
}

cudaError_t launch_fixedfeh(const gf_fixedfeh_config &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    fixedfeh_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(c, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- Bond2010 kinematics ---------------- */
__device__ __forceinline__ float modfun(float Rsquared, float Z, const float *val)
{
    /* a + b|Z|^c + d R^e, Bond2010_gpu.cu.h:106-110 */
    return val[0] + val[1] * gfm::powf_(fabsf(Z), val[2]) + val[3] * gfm::powf_(Rsquared, (float)(0.5 * (double)val[4]));
}

__device__ __forceinline__ void trivar_gauss(float y[3], const float sg[6], gfr::Mwc &rng)
{
    /* Cholesky draw, Bond2010_gpu.cu.h:81-103 */
    float s11 = sg[0], s12 = sg[1], s13 = sg[2], s22 = sg[3], s23 = sg[4], s33 = sg[5];
    float b10 = s12;      float b11 = s22 * s22;
    float b20 = s13;      float b21 = s23;      float b22 = s33 * s33;
    float a00 = s11; float oneDivA00 = 1.0f / a00;
    float a10 = b10 * oneDivA00;
    float a11 = sqrtf(b11 - a10 * a10);
    float a20 = b20 * oneDivA00;
    float a21 = (b21 - a20 * a10) / a11;
    float a22 = sqrtf(b22 - a20 * a20 - a21 * a21);
    float z0 = rng.gaussian(1.0f);
    float z1 = rng.gaussian(1.0f);
    float z2 = rng.gaussian(1.0f);
    y[0] += a00 * z0;
    y[1] += a10 * z0 + a11 * z1;
    y[2] += a20 * z0 + a21 * z1 + a22 * z2;
}

__device__ __forceinline__ void draw_moments(float v[3], float R2, float Z, const gf_vmoments &mo, bool disk, gfr::Mwc &rng)
{
    for (int i = 0; i < 3; i++) v[i] = modfun(R2, Z, mo.m[i]);
    if (disk && v[1] > 0.f) v[1] = 0.f;
    float sg[6];
    for (int i = 0; i < 6; i++) sg[i] = modfun(R2, Z, mo.ss[i]);
    trivar_gauss(v, sg, rng);
}

/* rows [begin + 256 th, min(begin + 256 (th + 1), end)) with stream th (Bond2010_gpu.cu.h:179, 217) */
__device__ __forceinline__ void bond2010_chunk(const gf_bond2010_config &par, uint32_t *rng, int32_t NS, gf_table &t,
                                               int64_t begin, int64_t end, int64_t th)
{
    const int64_t P = t.capacity;
    gfr::Mwc r;
    r.a = rng[th]; r.c = rng[NS + th]; r.x = rng[2 * NS + th];
    int64_t rb = begin + 256 * th, re = begin + 256 * (th + 1);
    if (re > end) re = end;
    for (int64_t row = rb; row < re; row++) {
        if (t.hidden[row]) continue;
        const int cmp = t.comp[row];
        float vx = t.XYZ[row] + par.T[0], vy = t.XYZ[P + row] + par.T[1], vz = t.XYZ[2 * P + row] + par.T[2];
        float wx = par.M[0] * vx + par.M[1] * vy + par.M[2] * vz;
        float wy = par.M[3] * vx + par.M[4] * vy + par.M[5] * vz;
        float wz = par.M[6] * vx + par.M[7] * vy + par.M[8] * vz;
        const float R2 = (float)(1e-6 * (double)(wx * wx + wy * wy));
        const float Z = (float)(1e-3 * (double)wz);
        float v[3];
        if (((par.comp_thin | par.comp_thick) >> cmp) & 1u) {
            float pu = r.uniform();
            const gf_vmoments &disk = pu < par.fk ? par.disk_1 : par.disk_2;
            draw_moments(v, R2, Z, disk, true, r);
        } else if ((par.comp_halo >> cmp) & 1u) {
            draw_moments(v, R2, Z, par.halo, false, r);
            float invR = 1.f / sqrtf(R2 + Z * Z);
            float cosa = sqrtf(R2) * invR;
            float sina = Z * invR;
            float vR = cosa * v[0] - sina * v[1];
            float vZ = sina * v[0] + cosa * v[1];
            v[0] = vR;
            v[1] = v[2];
            v[2] = vZ;
        } else {
            continue;
        }
        t.vcyl[row] = v[0];
        t.vcyl[P + row] = v[1];
        t.vcyl[2 * P + row] = v[2];
    }
    rng[NS + th] = r.c;
    rng[2 * NS + th] = r.x;
}

__global__ void __launch_bounds__(128) bond2010_kernel(const gf_bond2010_config par, uint32_t *rng, int32_t NS, gf_table t,
                                                        int64_t begin, int64_t end, int64_t nchunks)
{
    int64_t th = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (th >= nchunks) return;
    bond2010_chunk(par, rng, NS, t, begin, end, th);
}

/* the 256-row chunks of every request, each drawing from its request's streams */
__global__ void __launch_bounds__(128) bond2010_multi_kernel(const gf_bond2010_config par, uint32_t *rng_all, int32_t NS,
                                                              MultiRows R, const int64_t *slot_chunk_begin, int32_t nslots,
                                                              int64_t nchunks, const int64_t *slot_rows, gf_table t)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    int lo = 0, hi = nslots - 1;          /* last slot whose first chunk is <= c */
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (slot_chunk_begin[mid] <= c) lo = mid; else hi = mid - 1;
    }
    const int64_t b = R.slot_row_begin[lo];
    bond2010_chunk(par, rng_all + (size_t)R.slot_job[lo] * 3 * NS, NS, t, b, b + slot_rows[lo], c - slot_chunk_begin[lo]);
}

cudaError_t launch_bond2010_multi(const gf_bond2010_config &c, uint32_t *rng_all, int32_t NS, MultiRows R,
                                  const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks,
                                  const int64_t *slot_rows, gf_table t, cudaStream_t s)
{
    if (nchunks <= 0) return cudaSuccess;
    bond2010_multi_kernel<<<(unsigned)((nchunks + 127) / 128), 128, 0, s>>>(c, rng_all, NS, R, slot_chunk_begin, nslots,
                                                                          nchunks, slot_rows, t);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_bond2010(const gf_bond2010_config &c, uint32_t *rng, int32_t NS, gf_table t, int64_t begin, int64_t end,
                            cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    int64_t n = end - begin;
    int64_t nchunks = n / 256 + (n % 256 ? 1 : 0);
    if (nchunks > NS) return cudaErrorInvalidValue;
    bond2010_kernel<<<(int)((nchunks + 127) / 128), 128, 0, s>>>(c, rng, NS, t, begin, end, nchunks);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- FeH (Ivezic et al. 2008) and GaussianFeH ---------------- */

/* os_FeH_kernel (FeH_gpu.cu.h:43-87) on rows [begin + 256 th, ...) with stream th */
__device__ __forceinline__ void feh_chunk(const gf_feh_config &par, uint32_t *rng, int32_t NS, gf_table &t, int64_t begin,
                                          int64_t end, int64_t th)
{
    const int64_t P = t.capacity;
    gfr::Mwc r;
    r.a = rng[th]; r.c = rng[NS + th]; r.x = rng[2 * NS + th]; r.used = 0;
    int64_t rb = begin + 256 * th, re = begin + 256 * (th + 1);
    if (re > end) re = end;
    for (int64_t row = rb; row < re; row++) {
        if (t.hidden[row]) continue;
        const int cmp = t.comp[row];
        if (((par.comp_thin | par.comp_thick) >> cmp) & 1u) {
            /* the Gaussian to draw from */
            const float p = r.uniform() * (par.A[0] + par.A[1]);
            const int i = p < par.A[0] ? 0 : 1;
            /* the star's place in the disk */
            const float vx = t.XYZ[row] + par.T[0], vy = t.XYZ[P + row] + par.T[1], vz = t.XYZ[2 * P + row] + par.T[2];
            const float wz = par.M[6] * vx + par.M[7] * vy + par.M[8] * vz;
            /* Bond et al. A2; exp in single precision through the portable expf */
            const float muD = par.muInf + par.DeltaMu * gfm::expf_(-fabsf(wz) / par.Hmu);
            const float aZ = muD - 0.067f;
            const float feh = r.gaussian(par.sigma[i]) + aZ + par.offs[i];
            t.FeH[row] = feh;
        } else if ((par.comp_halo >> cmp) & 1u) {
            const float feh = par.offs[2] + r.gaussian(par.sigma[2]);
            t.FeH[row] = feh;
        }
    }
    rng[NS + th] = r.c;
    rng[2 * NS + th] = r.x;
}

/* os_GaussianFeH_kernel (GaussianFeH_gpu.cu.h:42-73) on rows [begin + 256 th, ...) with stream th */
__device__ __forceinline__ void gaussfeh_chunk(const gf_gaussfeh_config &par, uint32_t *rng, int32_t NS, gf_table &t,
                                               int64_t begin, int64_t end, int64_t th)
{
    gfr::Mwc r;
    r.a = rng[th]; r.c = rng[NS + th]; r.x = rng[2 * NS + th]; r.used = 0;
    int64_t rb = begin + 256 * th, re = begin + 256 * (th + 1);
    if (re > end) re = end;
    for (int64_t row = rb; row < re; row++) {
        if (t.hidden[row]) continue;
        const int cmp = t.comp[row];
        if (!((par.comp_mask >> cmp) & 1u)) continue;
        int at = 0;
        if (par.ncomp != 1) {
            const float u = r.uniform();
            while (par.pcum[at] < u) ++at;
        }
        t.FeH[row] = par.mean[at] + r.gaussian(par.sigma[at]);
        t.FeH_comp[row] = at;
    }
    rng[NS + th] = r.c;
    rng[2 * NS + th] = r.x;
}

template <int KIND>
__global__ void __launch_bounds__(128) feh_kernel(const gf_feh_config fp, const gf_gaussfeh_config gp, uint32_t *rng,
                                                  int32_t NS, gf_table t, int64_t begin, int64_t end, int64_t nchunks)
{
    const int64_t th = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (th >= nchunks) return;
    if (KIND == 0) feh_chunk(fp, rng, NS, t, begin, end, th);
    else gaussfeh_chunk(gp, rng, NS, t, begin, end, th);
}

/* the 256-row chunks of every request of a multi-request pass, each with its request's streams */
template <int KIND>
__global__ void __launch_bounds__(128) feh_multi_kernel(const gf_feh_config fp, const gf_gaussfeh_config gp,
                                                        uint32_t *rng_all, int32_t NS, MultiRows R,
                                                        const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks,
                                                        const int64_t *slot_rows, gf_table t)
{
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    int lo = 0, hi = nslots - 1;          /* last slot whose first chunk is <= c */
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (slot_chunk_begin[mid] <= c) lo = mid; else hi = mid - 1;
    }
    const int64_t b = R.slot_row_begin[lo];
    uint32_t *rng = rng_all + (size_t)R.slot_job[lo] * 3 * NS;
    if (KIND == 0) feh_chunk(fp, rng, NS, t, b, b + slot_rows[lo], c - slot_chunk_begin[lo]);
    else gaussfeh_chunk(gp, rng, NS, t, b, b + slot_rows[lo], c - slot_chunk_begin[lo]);
}

cudaError_t launch_feh(const gf_feh_config *fp, const gf_gaussfeh_config *gp, uint32_t *rng, int32_t NS, gf_table t,
                       int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    const int64_t n = end - begin, nchunks = n / 256 + (n % 256 ? 1 : 0);
    if (nchunks > NS) return cudaErrorInvalidValue;
    gf_feh_config f = {};
    gf_gaussfeh_config g = {};
    if (fp) f = *fp;
    if (gp) g = *gp;
    if (fp) feh_kernel<0><<<(int)((nchunks + 127) / 128), 128, 0, s>>>(f, g, rng, NS, t, begin, end, nchunks);
    else feh_kernel<1><<<(int)((nchunks + 127) / 128), 128, 0, s>>>(f, g, rng, NS, t, begin, end, nchunks);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_feh_multi(const gf_feh_config *fp, const gf_gaussfeh_config *gp, uint32_t *rng_all, int32_t NS,
                             MultiRows R, const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks,
                             const int64_t *slot_rows, gf_table t, cudaStream_t s)
{
    if (nchunks <= 0) return cudaSuccess;
    gf_feh_config f = {};
    gf_gaussfeh_config g = {};
    if (fp) f = *fp;
    if (gp) g = *gp;
    const unsigned blocks = (unsigned)((nchunks + 127) / 128);
    if (fp) feh_multi_kernel<0><<<blocks, 128, 0, s>>>(f, g, rng_all, NS, R, slot_chunk_begin, nslots, nchunks, slot_rows, t);
    else feh_multi_kernel<1><<<blocks, 128, 0, s>>>(f, g, rng_all, NS, R, slot_chunk_begin, nslots, nchunks, slot_rows, t);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- unresolved multiple systems ---------------- */

/* nearest-texel lookup of a 1-D table (cux.h:786-792, 849-855) */
__device__ __forceinline__ float mult_tex(const float *tab, int n, float x0, float inv_dx, float x)
{
    float xi = (x - x0) * inv_dx + 0.5f;
    if (xi < 0.f) xi = 0.f;
    else if (xi >= (float)n) xi = (float)n - 1;
    return tab[(uint32_t)xi];
}

/* draw_companion (unresolvedMultiples_gpu.cu.h:46-77) */
__device__ __forceinline__ bool mult_companion(const gf_multiples_config &c, float M1, gfr::Mwc &r, float &M2)
{
    const float psec = mult_tex(c.secprob, c.nsec, c.sec_x0, c.sec_inv_dx, M1);
    float u = r.uniform();
    if (u > psec) return false;
    if (c.algo == GF_MULT_EQUAL_MASS) { M2 = M1; return true; }
    const float pprim = mult_tex(c.cumlf, c.ncum, c.cum_x0, c.cum_inv_dx, M1);
    u = r.uniform();
    /* fainter than the primary: u rescaled into [pprim, 1] in double, as written */
    if (c.algo == GF_MULT_LF_M2_GT_M1) u = (float)((double)pprim + (double)u * (1. - (double)pprim));
    M2 = mult_tex(c.invcumlf, c.ninv, c.inv_x0, c.inv_inv_dx, u);
    if (c.algo == GF_MULT_LF_M2_GT_M1 && M2 < M1) M2 = M1;
    return true;
}

/* os_unresolvedMultiples_kernel (unresolvedMultiples_gpu.cu.h:80-123) on rows
 * [begin + 256 th, ...) with stream th; two system components (absmagSys[2]) */
__device__ __forceinline__ void multiples_chunk(const gf_multiples_config &c, uint32_t *rng, int32_t NS, gf_table &t,
                                                int64_t begin, int64_t end, int64_t th)
{
    const int64_t P = t.capacity;
    gfr::Mwc r;
    r.a = rng[th]; r.c = rng[NS + th]; r.x = rng[2 * NS + th]; r.used = 0;
    int64_t rb = begin + 256 * th, re = begin + 256 * (th + 1);
    if (re > end) re = end;
    for (int64_t row = rb; row < re; row++) {
        const float M1 = t.absmag[row];
        if (t.hidden[row] || !((c.comp_mask >> t.comp[row]) & 1u)) {
            /* a single star */
            t.absmagSys[row] = M1;
            t.absmagSys[P + row] = 99.999f;
            t.absmagSysNcomp[row] = 1;
            continue;
        }
        t.absmagSys[row] = M1;
        float Ltot = gfm::exp10f_(-0.4f * M1);
        int ncomps = 1;
        float M2 = 0.f;
        if (mult_companion(c, M1, r, M2)) {
            t.absmagSys[P + row] = M2;
            Ltot += gfm::exp10f_(-0.4f * M2);
            ncomps++;
        } else {
            t.absmagSys[P + row] = 99.999f;
        }
        /* -2.5 is a double: the product is formed in double and stored as float */
        t.absmag[row] = (float)(-2.5 * (double)gfm::log10f_(Ltot));
        t.absmagSysNcomp[row] = ncomps;
    }
    rng[NS + th] = r.c;
    rng[2 * NS + th] = r.x;
}

__global__ void __launch_bounds__(128) multiples_kernel(const gf_multiples_config c, uint32_t *rng, int32_t NS, gf_table t,
                                                        int64_t begin, int64_t end, int64_t nchunks)
{
    const int64_t th = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (th >= nchunks) return;
    multiples_chunk(c, rng, NS, t, begin, end, th);
}

__global__ void __launch_bounds__(128) multiples_multi_kernel(const gf_multiples_config c, uint32_t *rng_all, int32_t NS,
                                                              MultiRows R, const int64_t *slot_chunk_begin, int32_t nslots,
                                                              int64_t nchunks, const int64_t *slot_rows, gf_table t)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nchunks) return;
    int lo = 0, hi = nslots - 1;          /* last slot whose first chunk is <= k */
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (slot_chunk_begin[mid] <= k) lo = mid; else hi = mid - 1;
    }
    const int64_t b = R.slot_row_begin[lo];
    uint32_t *rng = rng_all + (size_t)R.slot_job[lo] * 3 * NS;
    multiples_chunk(c, rng, NS, t, b, b + slot_rows[lo], k - slot_chunk_begin[lo]);
}

cudaError_t launch_multiples(const gf_multiples_config &c, uint32_t *rng, int32_t NS, gf_table t, int64_t begin, int64_t end,
                             cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    const int64_t n = end - begin, nchunks = n / 256 + (n % 256 ? 1 : 0);
    if (nchunks > NS) return cudaErrorInvalidValue;
    multiples_kernel<<<(int)((nchunks + 127) / 128), 128, 0, s>>>(c, rng, NS, t, begin, end, nchunks);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_multiples_multi(const gf_multiples_config &c, uint32_t *rng_all, int32_t NS, MultiRows R,
                                   const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks, const int64_t *slot_rows,
                                   gf_table t, cudaStream_t s)
{
    if (nchunks <= 0) return cudaSuccess;
    multiples_multi_kernel<<<(unsigned)((nchunks + 127) / 128), 128, 0, s>>>(c, rng_all, NS, R, slot_chunk_begin, nslots,
                                                                             nchunks, slot_rows, t);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- photometry ---------------- */
__device__ __forceinline__ uint32_t brev(uint32_t a) { return __brev(a); }

__global__ void __launch_bounds__(256) photometry_kernel(PhotTables lt, gf_table t, int64_t begin, int64_t end)
{
    const int64_t P = t.capacity;
    const int ncolors = lt.nbands - 1;
    const bool sys = t.systems && t.absmagSys;
    const float *Mr = sys ? t.absmagSys : t.absmag;
    const int nabsmag = sys ? 2 : 1;
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        if (t.hidden[row]) continue;
        int cmp = t.comp[row];
        if (!((lt.comp_mask >> cmp) & 1u)) continue;
        float fFeH = t.FeH[row];
        uint32_t flag = 0;
        float c[GF_MAX_BANDS];
        /* the system's components (absmagSys when unresolved multiples ran, else the
         * single absmag): their luminosities are summed band by band */
        for (int syscomp = 0; syscomp < nabsmag; syscomp++) {
            const float fMr = Mr[(size_t)syscomp * P + row];
            if (fMr >= 99.999f) break;
            float xi = (fFeH - lt.tcFeH[0]) * lt.tcFeH[1] + 0.5f;
            float yi = (fMr - lt.tcMr[0]) * lt.tcMr[1] + 0.5f;
            if (xi < 0.f) xi = 0.f; else if (xi >= (float)lt.nFeH) xi = (float)lt.nFeH - 1;
            if (yi < 0.f) yi = 0.f; else if (yi >= (float)lt.nMr) yi = (float)lt.nMr - 1;
            uint32_t i = (uint32_t)xi, j = (uint32_t)yi;
            for (int ic = 0; ic < ncolors; ic++) {
                size_t off = ((size_t)ic * lt.nMr + j) * lt.nFeH + i;
                c[ic] = lt.colors[off];
                flag |= ((uint32_t)(lt.eflags[off] != 0)) << ic;
            }
            for (int b = 0; b <= ncolors; b++) {
                float M = fMr;
                if (b < lt.bidx) { for (int q = b; q != lt.bidx; q++) M += c[q]; }
                if (b > lt.bidx) { for (int q = lt.bidx; q != b; q++) M -= c[q]; }
                float L = gfm::exp10f_(-0.4f * M);
                if (syscomp) L += t.mags[b * P + row];
                t.mags[b * P + row] = L;
            }
        }
        bool fl = false;
        for (int q = lt.bidx - 1; q >= 0; q--) {
            fl = fl || (flag & (1u << q));
            flag |= ((uint32_t)fl) << q;
        }
        fl = false;
        for (int q = lt.bidx; q < ncolors; q++) {
            fl = fl || (flag & (1u << q));
            flag |= ((uint32_t)fl) << q << 1;
        }
        flag &= ~(1u << lt.bidx);
        flag = brev(flag);
        flag >>= (8 * sizeof(flag) - ncolors - 1);
        t.photoflags[row] = (int32_t)flag;
        float dm = t.DM[row];
        float Am0 = t.Am[row];
        for (int b = 0; b <= ncolors; b++) {
            float Msys = -2.5f * gfm::log10f_(t.mags[b * P + row]);
            float msys = dm + Msys;
            float Am = Am0 * lt.reddening[b];
            t.mags[b * P + row] = msys + Am;
        }
    }
}

cudaError_t launch_photometry(const PhotTables &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    photometry_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(c, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- photometric errors ---------------- */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw 2011) */
__device__ __forceinline__ void philox(uint32_t ctr[4], uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0 = __umulhi(0xD2511F53u, ctr[0]), lo0 = 0xD2511F53u * ctr[0];
        uint32_t hi1 = __umulhi(0xCD9E8D57u, ctr[2]), lo1 = 0xCD9E8D57u * ctr[2];
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0; ctr[1] = lo1; ctr[2] = n2; ctr[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

__device__ __forceinline__ double error_normal(uint64_t seed, uint64_t row, uint32_t band)
{
    uint32_t ctr[4] = {(uint32_t)row, (uint32_t)(row >> 32), band, 0x67616c66u};
    philox(ctr, (uint32_t)seed, (uint32_t)(seed >> 32));
    uint64_t a = ((uint64_t)ctr[0] << 21) ^ (ctr[1] >> 11);
    uint64_t b = ((uint64_t)ctr[2] << 21) ^ (ctr[3] >> 11);
    double u1 = ((double)(a & ((1ull << 53) - 1)) + 1.0) * 0x1p-53;
    double u2 = (double)(b & ((1ull << 53) - 1)) * 0x1p-53;
    double r = sqrt(-2.0 * gfm::log_d(u1));
    return r * gfm::cos_d(6.283185307179586 * u2);
}

/* gsl_interp_linear at x: the bisection's bracket (the last knot <= x, within
 * [0, n-2]), found from the guide cell when the knots are strictly increasing --
 * the same bracket, since the guide never starts past it -- and by bisection
 * otherwise (NaN takes the bisection's answer, n - 2). */
__device__ __forceinline__ double linear_eval(const double *xa, const double *ya, int n, double x, const int32_t *guide,
                                              int nguide, double gx0, double ginv)
{
    int ilo = 0;
    if (guide && x == x) {
        ilo = guide[perr_cell(x, gx0, ginv, nguide)];
        while (ilo < n - 2 && xa[ilo + 1] <= x) ilo++;
    } else {
        int ihi = n - 1;
        while (ihi > ilo + 1) {
            int i = (ihi + ilo) / 2;
            if (xa[i] > x) ihi = i; else ilo = i;
        }
    }
    double x_lo = xa[ilo], x_hi = xa[ilo + 1];
    double y_lo = ya[ilo], y_hi = ya[ilo + 1];
    double dx = x_hi - x_lo;
    if (dx > 0.0) return y_lo + (x - x_lo) / dx * (y_hi - y_lo);
    return 0.0;
}

/* observed magnitudes of one row; catalog_row numbers the row within its request's catalog */
__device__ __forceinline__ void photoerr_row(const PerrTables &c, uint64_t seed, int64_t catalog_row, gf_table &t, int64_t row)
{
    const int64_t P = t.capacity;
    if (t.hidden[row]) return;
    for (int b = 0; b < c.nbands; b++) {
        float mag = t.mags[b * P + row];
        float sigma = (float)linear_eval(c.mag + (size_t)b * c.nknots, c.sigma + (size_t)b * c.nknots, c.nknots, mag,
                                         c.guide ? c.guide + (size_t)b * c.nguide : nullptr, c.nguide, c.gx0[b], c.ginv[b]);
        double z = error_normal(seed, (uint64_t)catalog_row, (uint32_t)b);
        t.obsmags[b * P + row] = mag + (float)((double)sigma * z);
    }
}

__global__ void __launch_bounds__(256) photoerr_kernel(PerrTables c, int64_t row_offset, gf_table t, int64_t begin, int64_t end)
{
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x)
        photoerr_row(c, c.seed, row_offset + row, t, row);
}

__global__ void __launch_bounds__(256) photoerr_multi_kernel(PerrTables c, const uint64_t *seed_by_job,
                                                              const int64_t *catalog_offset_by_job, MultiRows R, gf_table t,
                                                              int64_t begin, int64_t end)
{
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        const int sl = R.row_slot[row];
        const int job = R.slot_job[sl];
        photoerr_row(c, seed_by_job[job], catalog_offset_by_job[job] + (row - R.slot_row_begin[sl]), t, row);
    }
}

cudaError_t launch_photoerrors_multi(const PerrTables &c, const uint64_t *seed_by_job, const int64_t *catalog_offset_by_job,
                                     MultiRows R, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    photoerr_multi_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(c, seed_by_job, catalog_offset_by_job, R, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_photoerrors(const PerrTables &c, int64_t row_offset, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    photoerr_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(c, row_offset, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- vel2pm ---------------- */
__device__ __forceinline__ void vel_xyz2lbr(float &vl, float &vb, float &vr, const float vx, const float vy, const float vz,
                                            const float l, const float b)
{
    float cl = gfm::cosf_(l), sl = gfm::sinf_(l), cb = gfm::cosf_(b), sb = gfm::sinf_(b);
    float tmp;
    vl = -vx * sl + vy * cl;
    tmp = vx * cl + vy * sl;
    vr = cb * tmp + vz * sb;
    vb = -sb * tmp + vz * cb;
}

__device__ __forceinline__ void transform_pm(float &vlout, float &vbout, float l, float b, float vl, float vb,
                                             const double ce, const double se, const double l0)
{
    double cb = gfm::cos_d((double)b);
    double sb = gfm::sin_d((double)b);
    double cl = gfm::cos_d((double)l - l0);
    double sl = gfm::sin_d((double)l - l0);
    double tmp1 = cb * se - ce * sb * sl;
    double tmp2 = ce * sb - cb * se * sl;
    double tmp4 = cb * cl;
    double tmp3 = sb * se + cb * ce * sl;
    if (fabs(tmp3) > 0.9999999) {
        vlout = vbout = 999.99f;
    } else {
        double denom1 = 1. / (tmp4 * tmp4 + tmp2 * tmp2);
        double cd = sqrt(1. - tmp3 * tmp3);
        vl = (float)((double)vl / cb);
        vlout = (float)((-ce * cl * (double)vb + cb * tmp1 * (double)vl) * denom1);
        vbout = (float)((tmp1 * (double)vb + cb * ce * cl * (double)vl) / cd);
        vlout = (float)((double)vlout * cd);
    }
}

__global__ void __launch_bounds__(256) vel2pm_kernel(gf_vel2pm_config par, gf_table t, int64_t begin, int64_t end)
{
    const int64_t P = t.capacity;
    const double ce = 0.88998740217659689, se = 0.45598511375586859, l0 = D2R * 32.932;
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        if (t.hidden[row]) continue;
        float l = 0.017453292519943295769f * (float)t.lb[row];
        float b = 0.017453292519943295769f * (float)t.lb[P + row];
        float X = par.Rg - t.XYZ[row];
        float Y = -t.XYZ[P + row];
        float Z = t.XYZ[2 * P + row];
        float vx = t.vcyl[row], vy = t.vcyl[P + row], vz = t.vcyl[2 * P + row];
        /* vel_cyl2xyz */
        float rho = sqrtf(X * X + Y * Y);
        float cphi = X / rho;
        float sphi = Y / rho;
        float px = -sphi * vy + cphi * vx;
        float py = cphi * vy + sphi * vx;
        float pz = vz;
        px -= par.u0;
        py -= par.v0 + par.vLSR;
        pz -= par.w0;
        float ix = -px, iy = -py, iz = pz;
        vel_xyz2lbr(px, py, pz, ix, iy, iz, l, b);
        float D = sqrtf((8000.f - X) * (8000.f - X) + Y * Y + Z * Z);
        px = (float)((double)px / (4.74 * (double)D * 1e-3));
        py = (float)((double)py / (4.74 * (double)D * 1e-3));
        if (par.coordsys == 1) {
            float ivl = px, ivb = py;
            transform_pm(px, py, l, b, ivl, ivb, ce, se, l0);
        } else if (par.coordsys != 0) {
            px = py = pz = -9.99f;
        }
        t.pm[row] = px;
        t.pm[P + row] = py;
        t.pm[2 * P + row] = pz;
    }
}

cudaError_t launch_vel2pm(const gf_vel2pm_config &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    vel2pm_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(c, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

/* ---------------- gal2other ---------------- */
__global__ void __launch_bounds__(256) gal2other_kernel(int32_t coordsys, gf_table t, int64_t begin, int64_t end)
{
    const int64_t P = t.capacity;
    const double angp = D2R * 192.859508333, l0 = D2R * 32.932;
    const double ce = 0.88998740217659689, se = 0.45598511375586859;
    const double pi2 = 2 * 3.14159265358979323846264338;
    for (int64_t row = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < end; row += (int64_t)gridDim.x * blockDim.x) {
        if (t.hidden[row]) continue;
        double lx = t.lb[row] * D2R, ly = t.lb[P + row] * D2R;
        double rx, ry;
        if (coordsys == 1) {
            const double cb = gfm::cos_d(ly), sb = gfm::sin_d(ly);
            const double cl = gfm::cos_d(lx - l0), sl = gfm::sin_d(lx - l0);
            rx = gfm::atan2_d(cb * cl, sb * ce - cb * se * sl) + angp;
            ry = gfm::asin_d(cb * ce * sl + sb * se);
            while (rx < 0.) rx += pi2;
            while (rx >= pi2) rx -= pi2;
        } else {
            rx = ry = -9999.;
        }
        t.radec[row] = rx / D2R;
        t.radec[P + row] = ry / D2R;
    }
}

cudaError_t launch_gal2other(int32_t coordsys, gf_table t, int64_t begin, int64_t end, cudaStream_t s)
{
    if (end <= begin) return cudaSuccess;
    gal2other_kernel<<<grid_for(end - begin, 256), 256, 0, s>>>(coordsys, t, begin, end);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace gfk
