/*
 * gf_oracle.cpp -- sequential CPU restatement of mjuric/galfast's catalog hot
 * path.  TEST INFRASTRUCTURE: loaded only by the test suite, smoke() and the
 * CPU-baseline leg of bench.py, as the checker or as the timed CPU baseline.
 *
 * It follows the reference's CPU build: the skygen kernel's emulated threads
 * run one after another (src/skygen/skygen.cu.h:119-151), atomicAdd is a plain
 * add (skygen.cu.h:153), textures are sampled at the nearest texel
 * (src/common/cux.h:778-810, 849-874), and every expression keeps the types
 * and evaluation order of the reference source (x86 SSE arithmetic, no FMA
 * contraction).  With -DOR_PORTABLE the elementary functions come from
 * galfast_b200/csrc/gf_math.h (bit-comparable with the GPU); otherwise from the
 * host libm, as in the reference's own build.
 */
#include "../include/galfast_b200.h"
#include "../galfast_b200/csrc/gf_math.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <thread>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>

#ifdef OR_PORTABLE
#define OR_EXPF gfm::expf_
#define OR_LOGF gfm::logf_
#define OR_LOG10F gfm::log10f_
#define OR_EXP10F gfm::exp10f_
#define OR_POWF gfm::powf_
#define OR_TANF gfm::tanf_
#define OR_SINF gfm::sinf_
#define OR_COSF gfm::cosf_
#define OR_SIN gfm::sin_d
#define OR_COS gfm::cos_d
#define OR_ASIN gfm::asin_d
#define OR_ATAN2 gfm::atan2_d
#define OR_EXP gfm::exp_d
#define OR_LOG gfm::log_d
#else
#define OR_EXPF ::expf
#define OR_LOGF ::logf
#define OR_LOG10F ::log10f
#define OR_EXP10F ::exp10f
#define OR_POWF ::powf
#define OR_TANF ::tanf
#define OR_SINF ::sinf
#define OR_COSF ::cosf
#define OR_SIN ::sin
#define OR_COS ::cos
#define OR_ASIN ::asin
#define OR_ATAN2 ::atan2
#define OR_EXP ::exp
#define OR_LOG ::log
#endif

namespace {

const double dbl_pi = 3.14159265358979323846264338;
const double dbl_d2r = 0.01745329251994329576923691;   /* module_lib.h:41-43 */
const double dbl_r2d = 57.2957795130823208767981548;
const float POGSON = 0.4605170185988091f;              /* skygen.cu.h:466 */
const int BLOCK = 10;                                   /* skygen.cu.h:467 */

/* ------------------------------------------------------------------ */
/* Multiply-with-carry stream and samplers: src/common/cuda_rng.h      */
/* ------------------------------------------------------------------ */
struct Rng {
    uint32_t a, c, xn;
    /* cuda_rng.h:439-463 */
    float uniform()
    {
        uint64_t xnew = (uint64_t)a * xn + c;
        c = (uint32_t)(xnew >> 32);
        xn = (uint32_t)((xnew << 32) >> 32);
        return 2.32830643708e-10f * xn;
    }
    /* cuda_rng.h:158-163 */
    float uniform_pos()
    {
        float x;
        do { x = uniform(); } while (x == 0.f);
        return x;
    }
    /* cuda_rng.h:165-182 (float square root, as the device build evaluates it) */
    float gaussian(const float sigma)
    {
        float x, y, r2;
        do {
            x = -1.f + 2.f * uniform();
            y = -1.f + 2.f * uniform();
            r2 = x * x + y * y;
        } while (r2 > 1.0f || r2 == 0.f || r2 == 4.f);
        return sigma * y * sqrtf(-2.0f * OR_LOGF(r2) / r2);
    }
    /* cuda_rng.h:185-208 */
    float gamma_large(const float aa)
    {
        float sqa, x, y, v;
        sqa = sqrtf(2 * aa - 1);
        do {
            do {
                y = OR_TANF((float)(M_PI * uniform()));
                x = sqa * y + aa - 1;
            } while (x <= 0);
            v = uniform();
        } while (v > (1 + y * y) * OR_EXPF((aa - 1) * OR_LOGF(x / (aa - 1)) - sqa * y));
        return x;
    }
    /* cuda_rng.h:211-235 */
    float gamma_int(const unsigned int aa)
    {
        if (aa < 3) {
            unsigned int i;
            float prod = 1;
            for (i = 0; i < aa; i++) prod *= uniform_pos();
            return -OR_LOGF(prod);
        }
        return gamma_large((float)aa);
    }
    /* cuda_rng.h:238-264 */
    float gamma_frac(const float aa)
    {
        float p, q, x, u, v;
        p = (float)(M_E / (aa + M_E));
        do {
            u = uniform();
            v = uniform_pos();
            if (u < p) {
                x = (float)OR_EXP((1 / aa) * OR_LOG(v));
                q = (float)OR_EXP(-x);
            } else {
                x = (float)(1 - OR_LOG(v));
                q = (float)OR_EXP((aa - 1) * OR_LOG(x));
            }
        } while (uniform() >= q);
        return x;
    }
    /* cuda_rng.h:276-297 */
    float gamma(const float aa, const float b)
    {
        unsigned int na = (unsigned int)floorf(aa);
        if (aa >= 4294967295.f) return b * (gamma_large(floorf(aa)) + gamma_frac(aa - floorf(aa)));
        else if (aa == (float)na) return b * gamma_int(na);
        else if (na == 0) return b * gamma_frac(aa);
        else return b * (gamma_int(na) + gamma_frac(aa - na));
    }
    /* cuda_rng.h:299-305 */
    float beta(const float aa, const float b)
    {
        float x1 = gamma(aa, 1.0);
        float x2 = gamma(b, 1.0);
        return x1 / (x1 + x2);
    }
    /* cuda_rng.h:308-340 */
    unsigned int binomial(float p, unsigned int n)
    {
        unsigned int i, aa, b, k = 0;
        while (n > 10) {
            float X;
            aa = 1 + (n / 2);
            b = 1 + n - aa;
            X = beta((float)aa, (float)b);
            if (X >= p) {
                n = aa - 1;
                p /= X;
            } else {
                k += aa;
                n = b - 1;
                p = (p - X) / (1 - X);
            }
        }
        for (i = 0; i < n; i++) {
            float u = uniform();
            if (u < p) k++;
        }
        return k;
    }
    /* cuda_rng.h:344-376 */
    unsigned int poisson(float mu)
    {
        float emu;
        float prod = 1.0;
        unsigned int k = 0;
        while (mu > 10) {
            unsigned int m = (unsigned int)(mu * (7.0 / 8.0));
            float X = gamma_int(m);
            if (X >= mu) return k + binomial(mu / X, m - 1);
            k += m;
            mu -= X;
        }
        emu = OR_EXPF(-mu);
        do {
            prod *= uniform();
            k++;
        } while (prod > emu);
        return k - 1;
    }
};

/* rng_base::load/store: gstate[i*nstreams + tid] (cuda_rng.h:45-69) */
struct RngState {
    uint32_t *g;
    int nstreams;
    Rng load(int tid) const { Rng r; r.a = g[tid]; r.c = g[nstreams + tid]; r.xn = g[2 * nstreams + tid]; return r; }
    void store(int tid, const Rng &r) const { g[tid] = r.a; g[nstreams + tid] = r.c; g[2 * nstreams + tid] = r.xn; }
};

/* ------------------------------------------------------------------ */
/* GSL linear interpolation (spline.cpp:59-65, gsl_interp_linear)     */
/* evaluated with the index search of gsl_interp_bsearch and linear    */
/* extrapolation beyond the end knots.                                 */
/* ------------------------------------------------------------------ */
double linear_eval(const double *xa, const double *ya, int n, double x)
{
    int ilo = 0, ihi = n - 1;
    while (ihi > ilo + 1) {
        int i = (ihi + ilo) / 2;
        if (xa[i] > x) ihi = i; else ilo = i;
    }
    double x_lo = xa[ilo], x_hi = xa[ilo + 1];
    double y_lo = ya[ilo], y_hi = ya[ilo + 1];
    double dx = x_hi - x_lo;
    if (dx > 0.0) return y_lo + (x - x_lo) / dx * (y_hi - y_lo);
    return 0.0;
}

/* direction (module_lib.h:87-114): cos/sin evaluated in double, stored as float */
struct Dir { float cl, cb, sl, sb; };
Dir make_dir(double l, double b)
{
    Dir d;
    d.cl = (float)OR_COS(l); d.cb = (float)OR_COS(b);
    d.sl = (float)OR_SIN(l); d.sb = (float)OR_SIN(b);
    return d;
}

struct F3 { float x, y, z; };

/* ------------------------------------------------------------------ */
/* Density models (model_expDisk.h:71-121, model_powerLawEllipsoid.h:60-105) */
/* ------------------------------------------------------------------ */
struct Model {
    int type, comp;
    float f, l, h, r_cut2;
    float n, ba, ca, rminSq, rmaxSq;
    int nbreaks;                       /* brokenPowerLaw (model_brokenPowerLaw.h:41-45) */
    float nArr[10], fArr[10], rbreakSq[9];
    float Rg;                          /* densityCube (model_densityCube.h:40-44) */
    const float *cube;
    int cube_n[3];
    float cube_tc[3][2];
    float T[3];
    float M[3][3];
    std::vector<float> lf;
    float lf_x0, lf_inv_dx;
    /* skygenParams of this model after init() (skyconfig_impl.h:244-297) */
    float m0, m1, dm, M0, M1, dM, dmin, dmax;
    int npixels, nm, nM, nthreads;
    float norm;
    double nstarsExpectedToGenerate, nstarsExpected;

    float rho(float x, float y, float z) const
    {
        /* transform(v, T, M) (module_lib.h:133-146) */
        float vx = x + T[0], vy = y + T[1], vz = z + T[2];
        float wx = M[0][0] * vx + M[0][1] * vy + M[0][2] * vz;
        float wy = M[1][0] * vx + M[1][1] * vy + M[1][2] * vz;
        float wz = M[2][0] * vx + M[2][1] * vy + M[2][2] * vz;
        if (type == GF_MODEL_DENSITY_CUBE) {
            /* densityCube::setpos (model_densityCube.h:60-66): galactocentric, nearest texel */
            float gx = Rg - x, gy = y * -1, gz = z;
            const float c3[3] = {gx, gy, gz};
            size_t ix[3];
            for (int a = 0; a < 3; a++) {
                float t = (c3[a] - cube_tc[a][0]) * cube_tc[a][1] + 0.5f;
                if (t < 0.f) t = 0.f;
                else if (t >= cube_n[a]) t = cube_n[a] - 1;
                ix[a] = (uint32_t)t;
            }
            return f * cube[(ix[2] * cube_n[1] + ix[1]) * cube_n[0] + ix[0]];
        }
        if (type == GF_MODEL_EXP_DISK) {
            float r2 = wx * wx + wy * wy;
            if (r_cut2 && r2 + wz * wz > r_cut2) return 0.f;
            float r = sqrtf(r2);
            float rho = f * OR_EXPF(-r / l - fabsf(wz) / h);
            return rho;
        } else if (type == GF_MODEL_BROKEN_POWER_LAW) {
            /* brokenPowerLaw::rho (model_brokenPowerLaw.h:55-82) */
            float DSq = wx * wx + wy * wy + wz * wz;
            if (rmaxSq && (DSq < rminSq || DSq >= rmaxSq)) return 0.f;
            int k = 0;
            float rSq = wx * wx + (wy / ba) * (wy / ba) + (wz / ca) * (wz / ca);
            while (k != nbreaks && rSq > rbreakSq[k]) k++;
            float rho = f * fArr[k] * OR_POWF(rSq, 0.5f * nArr[k]);
            return rho;
        } else if (type == GF_MODEL_LCBULGE) {
            /* LCBulge::rho (model_LCBulge.h:79-92) */
            float t = OR_POWF(OR_POWF(wx, n) + OR_POWF(wy / ba, n) + OR_POWF(wz / ca, n), (float)(1. / n));
            float rho = OR_EXPF(-t / l);
            return rho;
        } else {
            /* powerLawEllipsoid::rho (model_powerLawEllipsoid.h:60-92) */
            float DSq = wx * wx + wy * wy + wz * wz;
            if (rmaxSq && (DSq < rminSq || DSq >= rmaxSq)) return 0.f;
            float ty = wy / ba, tz = wz / ca;
            float rSq = wx * wx + ty * ty + tz * tz;
            float rho = f * OR_POWF(rSq, 0.5f * n);
            return rho;
        }
    }
    /* TEX1D on the CPU: nearest texel with clamping (cux.h:778-792, 849-855) */
    float lf_sample(float Mabs) const
    {
        float xi = (Mabs - lf_x0) * lf_inv_dx + 0.5f;
        float i = xi;
        if (i < 0.f) i = 0.f;
        else if (i >= (float)lf.size()) i = (float)lf.size() - 1;
        return lf[(uint32_t)i];
    }
};

/* reset_absmag (os_skygen.cpp:401-407) */
void reset_absmag(Model &m, float M0, float M1, float dM)
{
    m.M0 = M0; m.M1 = M1; m.dM = dM;
    m.nM = (int)round((m.M1 - m.M0) / m.dM);
    m.M1 -= 0.5 * m.dM;
}

/* galplane frame: xxx2galxyz + get_gal2xxx_matrix (transform.cpp:100-135, 194-213, 345-388) */
void load_transform(const gf_model_config &c, float T[3], float M[3][3])
{
    if (c.frame == GF_FRAME_EXPLICIT) {
        for (int i = 0; i < 3; i++) T[i] = (float)c.T[i];
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) M[i][j] = (float)c.M[3 * i + j];
        return;
    }
    double Rg = c.Rg, z0 = c.z0;
    double v[3] = {0., 0., 0.};
    double sina = -z0 / Rg, cosa = sqrt(1 - sina * sina);
    double x = cosa * v[0] - sina * v[2];
    double z = sina * v[0] + cosa * v[2];
    v[0] = Rg - x;
    v[1] = -v[1];
    v[2] = z;
    T[0] = (float)-v[0]; T[1] = (float)-v[1]; T[2] = (float)-v[2];
    double go[3][3];
    go[0][0] = -cosa; go[0][1] = 0; go[0][2] = sina;
    go[1][0] = 0;     go[1][1] = -1; go[1][2] = 0;
    go[2][0] = sina;  go[2][1] = 0; go[2][2] = cosa;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) M[i][j] = (float)go[i][j];
}

/* load_resample_and_clip_texture_1D + construct_texture_by_resampling_1D (cux.cpp:336-384),
 * or load_constant_texture_1D(1, -100, 100) (cux.cpp:310-318) without a LF table. */
void load_lf(Model &m, const gf_model_config &c)
{
    if (c.lf_n <= 0 || !c.lf_M) {
        m.lf.assign(2, 1.f);
        m.lf_x0 = -100.f;
        m.lf_inv_dx = (float)(1. / (100. - -100.));
        return;
    }
    std::vector<double> X, Y;
    X.push_back(-123); Y.push_back(0.f);
    for (int i = 0; i < c.lf_n; i++) { X.push_back(c.lf_M[i]); Y.push_back(c.lf_phi[i]); }
    double xrange = X.back() - X[1];
    X[0] = X[1] - 1e-5 * xrange;
    X.push_back(X.back() + 1e-5 * xrange);
    Y.push_back(0.f);
    int ndata = (int)X.size(), nsamp = 1024;
    m.lf.resize(nsamp);
    double X0 = X[0], X1 = X[ndata - 1], dX = (X1 - X0) / (nsamp - 1);
    for (int i = 0; i != nsamp; i++) {
        m.lf[i] = (float)linear_eval(X.data(), Y.data(), ndata, X0 + i * dX);
    }
    m.lf_x0 = (float)X0;
    m.lf_inv_dx = (float)(1. / dX);
}

/* ------------------------------------------------------------------ */
/* skygen                                                              */
/* ------------------------------------------------------------------ */
struct Pixel : gf_pencil_beam {};

/* runtime_state<Model> (skygen.h:184-257) */
struct KState {
    std::vector<int> cont, ilb, im, iM, k, bc, ndraw;
    std::vector<F3> pos;
    std::vector<float> D, Am, ms;
    std::vector<gf_pencil_beam> pix;
    void alloc(int n)
    {
        cont.assign(n, 0); ilb.assign(n, 0); im.assign(n, 0); iM.assign(n, 0); k.assign(n, 0);
        bc.assign(n, 0); ndraw.assign(n, 0); pos.assign(n, F3{0, 0, 0});
        D.assign(n, 0); Am.assign(n, 0); ms.assign(n, 0); pix.assign(n, gf_pencil_beam());
    }
};

struct Sky {
    gf_skygen_config cfg;
    std::vector<gf_pencil_beam> pixels;
    std::vector<float> ammin;
    gf_extinction ext;
    int ext_nz = 1;                    /* GF_EXT_MAPS: DM texels of the per-beam rows */
    float ext_tcz[2] = {0.f, 1.f};
    std::vector<Model> models;
    std::vector<KState> ks;            /* per model draw state */
    std::vector<char> ks_alloc;
};

/* One star row of the skygen columns (os_skygen.cpp:838-858), as draw_stars
 * fills it; rows hidden by the projection edge carry only hidden = 1. */
struct StarRow {
    double l, b;
    float x, y, absmag, DM, X, Y, Z, Am, AmInf;
    int32_t projIdx, comp, hidden;
};

/* The constant part of one kernel launch (skygenGPU<T> in __constant__ memory). */
struct Launch {
    const Sky *sky;
    const Model *m;
    int npixels;
    const gf_pencil_beam *pixels;
    int stopstars;
    /* draw */
    int *nstars;
    gf_table *out;                 /* rows at their atomicAdd index ... */
    std::vector<StarRow> *rows;    /* ... or appended here (the parallel draw's private runs) */
    KState *ks;
    RngState rng;
    /* integrate */
    double *counts, *countsCovered;
    float *countsCoveredPerBeam;   /* [nthreads][npixels] */
    float *maxCount;
    int64_t *nabove;               /* diagnostics (nullable): bins with rho > above, per thread */
    float above;
};

/* skygen.cu.h:257-300 */
void diagIndexToIJ(int &ilb, int &i, int &j, int &k, const int x, const int y)
{
    int kmax = x * y;
    if (k >= kmax) {
        ilb += k / kmax;
        k %= kmax;
    }
    int l = x < y ? x : y;
    int m = x < y ? y : x;
    int d;
    if (2 * k < l * (l - 1)) {
        d = int(0.5 * (sqrtf(1 + 8 * k) - 1));
        i = k - d * (d + 1) / 2;
    } else if (2 * k < l * (2 * m + 1 - l)) {
        if (x >= y) {
            int ka = k - y * (y - 1) / 2;
            d = int(ka / y) + (y - 1);
            i = (ka % y) + d - (y - 1);
        } else {
            int ka = k - x * (x - 1) / 2;
            d = int(ka / x) + (x - 1);
            i = ka % x;
        }
    } else {
        int ka = x * y - k - 1;
        int dd = int(0.5 * (sqrtf(1 + 8 * ka) - 1));
        d = (x + y - 2) - dd;
        i = (x - 1) - (ka - dd * (dd + 1) / 2);
    }
    j = d - i;
}

/* skygen.cu.h:307-358 */
bool advance(const Launch &L, int &ilb, int &i, int &j, gf_pencil_beam &dir, const int x, const int y)
{
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
        if (i == x) {
            ilb++;
            if (ilb != L.npixels) dir = L.pixels[ilb];
        }
    } else {
        return false;
    }
    return true;
}

/* nearest-texel index of the host build's texture sampling (cux.h:778-809, 860-874) */
static uint32_t texel(float v, const float tc[2], int n)
{
    float t = (v - tc[0]) * tc[1] + 0.5f;
    if (t < 0.f) t = 0.f;
    else if (t >= n) t = n - 1;
    return (uint32_t)t;
}

/* The minimum extinction along a beam (ext_beam texture, os_skygen.cpp:742-797):
 * with 3-D maps the beam's row at the nearest DM texel (TEX3D(ext_beam, xidx, yidx, DM)). */
float beam_extinction(const Launch &L, const gf_pencil_beam &pix, float DM)
{
    const Sky &s = *L.sky;
    if (s.ext.kind == GF_EXT_NONE || s.ammin.empty()) return 0.f;
    if (s.ext.kind == GF_EXT_MAPS) {
        const uint32_t k = texel(DM, s.ext_tcz, s.ext_nz);
        return s.ammin[(size_t)pix.extIdx * s.ext_nz + k];
    }
    return s.ammin[pix.extIdx];
}

/* Extinction towards a star (sampleExtinction, skygen.cu.h:199-208): the screen,
 * or the map of the star's hemisphere at its projected position and DM. */
float star_extinction(const Launch &L, const Dir &d, int projIdx, float x, float y, float DM)
{
    const Sky &s = *L.sky;
    if (s.ext.kind == GF_EXT_SCREEN_CSCB) return s.ext.A0 / fabsf(d.sb);
    if (s.ext.kind == GF_EXT_MAPS) {
        const gf_ext_map *e = projIdx == 0 ? s.ext.north : s.ext.south;
        if (!e) return 0.f;
        const uint32_t i = texel(x, e->tc[0], e->n[0]), j = texel(y, e->tc[1], e->n[1]), k = texel(DM, e->tc[2], e->n[2]);
        return e->A[((size_t)k * e->n[1] + j) * e->n[0] + i];
    }
    return 0.f;
}

/* skygen.cu.h:216-229 */
F3 compute_pos(const Launch &L, float &D, float &Am, float M, const int im, const gf_pencil_beam &pix)
{
    const Model &m = *L.m;
    float mm = m.m0 + im * m.dm;
    float DM = mm - M;
    D = OR_POWF(10.f, 0.2f * DM + 1.f);
    Am = beam_extinction(L, pix, DM);
    F3 p;
    p.x = D * pix.cl * pix.cb;
    p.y = D * pix.sl * pix.cb;
    p.z = D * pix.sb;
    return p;
}

/* lambert::deproject (skygen.h:131-146) */
void deproject(const gf_lambert &p, double &l, double &b, const float x, const float y)
{
    double r2 = x * x + y * y;
    if (r2 == 0.) { b = p.b0; l = 0.; return; }
    double ir = 1. / sqrt(r2);
    double sc = 1. / ir * sqrt(1. - 0.25 * r2);
    double cc = 1. - 0.5 * r2;
    b = OR_ASIN(cc * p.sb + y * sc * p.cb * ir);
    l = p.l0 + OR_ATAN2(x * sc, p.cb * cc / ir - y * p.sb * sc);
}

/* Store one row at index idx of the launch's output. */
void put_row(const Launch &L, int idx, const StarRow &r)
{
    if (L.rows) { L.rows->push_back(r); return; }
    gf_table &s = *L.out;
    const int64_t P = s.capacity;
    s.hidden[idx] = r.hidden;
    if (r.hidden && r.projIdx < 0) return;          /* beyond the projection edge: only the flag */
    s.projIdx[idx] = r.projIdx;
    s.projXY[idx] = r.x;
    s.projXY[P + idx] = r.y;
    s.lb[idx] = r.l;
    s.lb[P + idx] = r.b;
    s.absmag[idx] = r.absmag;
    s.DM[idx] = r.DM;
    s.XYZ[idx] = r.X;
    s.XYZ[P + idx] = r.Y;
    s.XYZ[2 * P + idx] = r.Z;
    s.comp[idx] = r.comp;
    s.Am[idx] = r.Am;
    s.AmInf[idx] = r.AmInf;
}

/* skygen.cu.h:366-457 */
void draw_stars(const Launch &L, Rng &rng, int &ndraw, const float &M, const int &im, const gf_pencil_beam &pix, float AmMin)
{
    if (!ndraw) return;
    const Model &m = *L.m;
    int idx = *L.nstars; *L.nstars += ndraw;          /* CPU atomicAdd, skygen.cu.h:153 */
    for (; ndraw && idx < L.stopstars; idx++, ndraw--) {
        StarRow r = StarRow();
        float x = pix.X, y = pix.Y;
        x += pix.dx * (rng.uniform() - 0.5f);
        y += pix.dx * (rng.uniform() - 0.5f);
        if (x * x + y * y > 2.f) {
            r.hidden = 1;
            r.projIdx = -1;
            put_row(L, idx, r);
            continue;
        }
        r.projIdx = pix.projIdx;
        r.x = x;
        r.y = y;
        double l, b;
        deproject(L.sky->cfg.proj[pix.projIdx], l, b, x, y);
        Dir dir2 = make_dir(l, b);
        l *= dbl_r2d;
        if (l < 0.) l += 360.;
        if (l > 360.) l -= 360.;
        b *= dbl_r2d;
        r.l = l;
        r.b = b;
        float Mtmp, mtmp, DM;
        r.absmag = Mtmp = M + m.dM * (rng.uniform() - 0.5f);
        mtmp = m.m0 + m.dm * (im + rng.uniform() - 0.5f);
        DM = mtmp - Mtmp;
        r.DM = DM;
        float D = OR_POWF(10, 0.2f * DM + 1.f);
        r.X = D * dir2.cl * dir2.cb;
        r.Y = D * dir2.sl * dir2.cb;
        r.Z = D * dir2.sb;
        r.comp = m.comp;
        float Am0, Am1;
        r.Am = Am0 = star_extinction(L, dir2, pix.projIdx, x, y, DM);
        Am1 = star_extinction(L, dir2, pix.projIdx, x, y, 100);
        r.AmInf = Am1 > Am0 ? Am1 : Am0;
        r.hidden = (mtmp + Am0 > m.m1) ? 1 : 0;
        if (AmMin > Am0) r.AmInf = -AmMin;
        put_row(L, idx, r);
    }
}

/* skygenGPU<T>::kernel<draw> (skygen.cu.h:469-618) for one emulated thread */
void kernel(const Launch &L, int draw, int tid)
{
    const Model &mdl = *L.m;
    const int nthreads = mdl.nthreads, nm = mdl.nm, nM = mdl.nM;
    int ilb, im = 0, iM = 0, k, ndraw = 0;
    F3 pos = {0, 0, 0};
    gf_pencil_beam pix = gf_pencil_beam();
    float Am = 0;
    double count = 0.f, countCovered = 0.f;
    float maxCount1 = 0.;
    int bc = 0;
    float D = 0;
    float ms = 0;
    Rng rng = {0, 0, 0};

    ilb = 0;
    k = BLOCK * (tid - nthreads);
    if (draw) {
        KState &ks = *L.ks;
        if (ks.cont[tid]) {
            ilb = ks.ilb[tid]; im = ks.im[tid]; iM = ks.iM[tid]; k = ks.k[tid]; bc = ks.bc[tid];
            pos = ks.pos[tid]; pix = ks.pix[tid]; D = ks.D[tid]; Am = ks.Am[tid]; ms = ks.ms[tid];
            ndraw = ks.ndraw[tid];
        }
        if (ilb >= L.npixels) return;
        rng = L.rng.load(tid);
        if (ndraw) {
            float M = mdl.M1 - iM * mdl.dM;
            draw_stars(L, rng, ndraw, M, im, pix, Am);
        }
    }

    double rhoBeam = 0.f;
    int ilbPrev = 0;
    while (ndraw == 0) {
        bool moved;
        if (bc == 0) {
            bc = BLOCK;
            k += BLOCK * nthreads;
            diagIndexToIJ(ilb, im, iM, k, nm, nM);
            if (ilb >= L.npixels) break;
            pix = L.pixels[ilb];
            moved = true;
        } else {
            moved = advance(L, ilb, im, iM, pix, nm, nM);
        }
        bc--;

        float M = mdl.M1 - iM * mdl.dM;
        if (moved) {
            if (ilb >= L.npixels) break;
            pos = compute_pos(L, D, Am, M, im, pix);
            ms = mdl.rho(pos.x, pos.y, pos.z);
        }

        if ((mdl.dmin || mdl.dmax) && (mdl.dmin > D || mdl.dmax <= D)) continue;

        float m = mdl.m0 + mdl.dm * im + Am;
        if (m > mdl.m1) continue;

        float rho = mdl.lf_sample(M) * ms;
        rho *= mdl.norm;
        rho *= D * D * D;
        rho *= pix.dA * POGSON * mdl.dm * mdl.dM;

        if (draw) {
            if (ndraw == 0) ndraw = rng.poisson(rho);
            draw_stars(L, rng, ndraw, M, im, pix, Am);
        } else {
            if (ilbPrev != ilb) {
                L.countsCoveredPerBeam[(size_t)tid * L.npixels + ilbPrev] = (float)rhoBeam;
                rhoBeam = 0.f;
                ilbPrev = ilb;
            }
            count += rho;
            countCovered += rho * pix.coveredFraction;
            rhoBeam += rho * pix.coveredFraction;
            if (maxCount1 < rho) maxCount1 = rho;
            if (L.nabove && rho > L.above) L.nabove[tid]++;
        }
    }

    if (!draw) {
        L.countsCoveredPerBeam[(size_t)tid * L.npixels + ilbPrev] = (float)rhoBeam;
        L.counts[tid] = count;
        L.countsCovered[tid] = countCovered;
        L.maxCount[tid] = maxCount1;
    } else {
        KState &ks = *L.ks;
        ks.ilb[tid] = ilb; ks.im[tid] = im; ks.iM[tid] = iM; ks.k[tid] = k; ks.bc[tid] = bc;
        ks.pos[tid] = pos; ks.pix[tid] = pix; ks.D[tid] = D; ks.Am[tid] = Am; ks.ms[tid] = ms;
        ks.ndraw[tid] = ndraw;
        ks.cont[tid] = 1;
        L.rng.store(tid, rng);
    }
}

thread_local std::string g_err;

int g_nthreads_cpu = 1;     /* host threads used by the parallel loops (or_set_threads) */

/* A persistent pool of host threads for the loops over independent streams,
 * rows and columns.  run(n, f) calls f(i) for every i in [0, n) once, handing
 * out indices in small chunks from a counter of that run; the calling thread
 * takes part and returns when every index is done, without waiting for workers
 * that woke too late to find work.  Idle workers spin briefly before they sleep,
 * since loops follow one another closely.  Results never depend on which thread
 * ran an index. */
class Pool {
public:
    ~Pool() { resize(0); }
    void resize(int nworkers)
    {
        {
            std::unique_lock<std::mutex> lk(mu_);
            stop_ = true;
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
        th_.clear();
        stop_ = false;
        const uint64_t g0 = gen_.load();      /* workers wait for the first run after this generation */
        for (int i = 0; i < nworkers; i++) th_.emplace_back([this, g0]() { worker(g0); });
    }
    int workers() const { return (int)th_.size(); }
    void run(int n, int chunk, const std::function<void(int)> &f)
    {
        if (th_.empty() || n <= chunk) { for (int i = 0; i < n; i++) f(i); return; }
        auto job = std::make_shared<Job>();
        job->f = &f; job->n = n; job->chunk = chunk;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cur_ = job;
            gen_.fetch_add(1);
        }
        cv_.notify_all();
        work(*job);
        while (job->done.load() < n) std::this_thread::yield();
    }

private:
    struct Job {
        const std::function<void(int)> *f = nullptr;
        int n = 0, chunk = 1;
        std::atomic<int> next{0}, done{0};
    };
    static void work(Job &j)
    {
        for (;;) {
            int b = j.next.fetch_add(j.chunk);
            if (b >= j.n) break;
            int e = std::min(b + j.chunk, j.n);
            for (int i = b; i < e; i++) (*j.f)(i);
            j.done.fetch_add(e - b);
        }
    }
    void worker(uint64_t seen)
    {
        for (;;) {
            for (int spin = 0; spin < 20000 && gen_.load() == seen; spin++) std::this_thread::yield();
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&]() { return gen_.load() != seen; });
                seen = gen_.load();
                if (stop_) return;
                job = cur_;
            }
            if (job) work(*job);
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::shared_ptr<Job> cur_;
    std::atomic<uint64_t> gen_{0};
    bool stop_ = false;
};

Pool &pool()
{
    static Pool p;
    if (p.workers() != g_nthreads_cpu - 1) p.resize(g_nthreads_cpu - 1);
    return p;
}

/* Run f(i) for i in [0, n) on g_nthreads_cpu host threads. */
template <typename F>
void parallel_for(int n, F f, int chunk = 16)
{
    if (g_nthreads_cpu <= 1 || n <= 1) { for (int i = 0; i < n; i++) f(i); return; }
    std::function<void(int)> fn = f;
    pool().run(n, chunk, fn);
}

/* f(begin, end) over [0, n) in contiguous pieces of at least `grain` rows. */
template <typename F>
void parallel_rows(int64_t n, F f, int64_t grain = 128)
{
    if (g_nthreads_cpu <= 1 || n <= grain) { if (n > 0) f((int64_t)0, n); return; }
    int64_t pieces = std::min<int64_t>((n + grain - 1) / grain, 64 * (int64_t)g_nthreads_cpu);
    int64_t step = (n + pieces - 1) / pieces;
    parallel_for((int)pieces, [&](int i) {
        int64_t b = i * step, e = std::min(n, b + step);
        if (b < e) f(b, e);
    }, 1);
}

/* Copy stream tid's crawl state from one runtime_state to another. */
void copy_state(KState &d, const KState &s, int tid)
{
    d.cont[tid] = s.cont[tid]; d.ilb[tid] = s.ilb[tid]; d.im[tid] = s.im[tid]; d.iM[tid] = s.iM[tid];
    d.k[tid] = s.k[tid]; d.bc[tid] = s.bc[tid]; d.ndraw[tid] = s.ndraw[tid]; d.pos[tid] = s.pos[tid];
    d.D[tid] = s.D[tid]; d.Am[tid] = s.Am[tid]; d.ms[tid] = s.ms[tid]; d.pix[tid] = s.pix[tid];
}

/* One draw batch with the emulated threads run on several host threads, with
 * the result of running them one after another (skygen.cu.h:119-151; batch
 * rules skyconfig_impl.h:445-534).  First every stream runs alone from its
 * state, on a private counter and with the whole capacity as its room.  The
 * streams' counts, summed in stream order, give each stream's first output
 * index in the sequential run (its atomicAdd base).  Streams whose stars all fit
 * keep that run.  The stream whose stars cross the capacity and every later one
 * run again from their saved state with the room the sequential run leaves them:
 * what remains of the capacity for the crossing stream, none for the later ones
 * (they stop at their first bin with stars).  *nstars receives the sequential
 * run's final counter, or any value >= stopstars when a stream crossed. */
void draw_parallel(const Sky *s, const Model &m, KState &ks, RngState rs, gf_table *t, int stopstars, int64_t *nstars)
{
    const int N = m.nthreads;
    KState snap = ks;
    std::vector<Rng> rng0(N);
    for (int tid = 0; tid < N; tid++) rng0[tid] = rs.load(tid);
    std::vector<std::vector<StarRow>> rows(N);
    std::vector<int64_t> cnt(N, 0);
    auto run = [&](int tid, int room) {
        int c = 0;
        Launch L = {};
        L.sky = s; L.m = &m; L.npixels = m.npixels; L.pixels = s->pixels.data();
        L.stopstars = room; L.nstars = &c; L.rows = &rows[tid]; L.ks = &ks; L.rng = rs;
        rows[tid].clear();
        kernel(L, 1, tid);
        cnt[tid] = c;
    };
    parallel_for(N, [&](int tid) { run(tid, stopstars); }, 64);
    std::vector<int64_t> base(N, 0);
    int64_t G = 0;
    int T = -1;
    for (int tid = 0; tid < N; tid++) {
        base[tid] = G;
        if (G + cnt[tid] > stopstars) { T = tid; break; }
        G += cnt[tid];
    }
    int placed = N;
    if (T >= 0) {
        for (int tid = T; tid < N; tid++) { copy_state(ks, snap, tid); rs.store(tid, rng0[tid]); }
        parallel_for(N - T, [&](int i) {
            const int tid = T + i;
            run(tid, tid == T ? (int)(stopstars - base[T]) : 0);
        }, 64);
        placed = T + 1;
    }
    Launch P = {};
    P.out = t;
    parallel_for(placed, [&](int tid) {
        for (size_t k = 0; k < rows[tid].size(); k++) put_row(P, (int)(base[tid] + (int64_t)k), rows[tid][k]);
    }, 16);
    *nstars = T >= 0 ? (int64_t)stopstars + 1 : G;
}

/* star_comp (skyconfig_impl.h:34-68) */
struct StarComp {
    const gf_table *t;
    bool operator()(const size_t a, const size_t b) const
    {
        const int64_t P = t->capacity;
        const double *lb = t->lb;
        int ha = t->hidden[a], hb = t->hidden[b];
        if (ha != hb) return ha < hb;
        if (lb[a] != lb[b]) return lb[a] < lb[b];
        if (lb[P + a] != lb[P + b]) return lb[P + a] < lb[P + b];
        if (t->DM[a] != t->DM[b]) return t->DM[a] < t->DM[b];
        if (t->absmag[a] != t->absmag[b]) return t->absmag[a] < t->absmag[b];
        return t->Am[a] < t->Am[b];
    }
};

/* The order of star_comp over row indices: std::sort on one thread; on several,
 * sorted pieces merged pairwise.  star_comp orders rows by (hidden, l, b, DM, M,
 * Am); rows equal in all six never occur in practice, so both give one order. */
void sort_rows(std::vector<size_t> &idx, const StarComp &sc)
{
    const size_t n = idx.size();
    if (g_nthreads_cpu <= 1 || n < 65536) { std::sort(idx.begin(), idx.end(), sc); return; }
    int pieces = 1;
    while (pieces < 2 * g_nthreads_cpu && pieces < 64) pieces *= 2;
    std::vector<size_t> bnd(pieces + 1);
    for (int i = 0; i <= pieces; i++) bnd[i] = n * i / pieces;
    parallel_for(pieces, [&](int i) { std::sort(idx.begin() + bnd[i], idx.begin() + bnd[i + 1], sc); }, 1);
    std::vector<size_t> tmp(n);
    for (int w = 1; w < pieces; w *= 2) {
        const int pairs = pieces / (2 * w);
        parallel_for(pairs, [&](int p) {
            size_t a = bnd[2 * w * p], b = bnd[2 * w * p + w], e = bnd[2 * w * (p + 1)];
            std::merge(idx.begin() + a, idx.begin() + b, idx.begin() + b, idx.begin() + e, tmp.begin() + a, sc);
        }, 1);
        idx.swap(tmp);
    }
}

template <typename T>
void permute(T *col, const std::vector<size_t> &s, int64_t n)
{
    std::vector<T> tmp(col, col + n);
    for (int64_t i = 0; i < n; i++) col[i] = tmp[s[i]];
}

/* ------------------------------------------------------------------ */
/* Modules                                                              */
/* ------------------------------------------------------------------ */

/* sampleColors with nearest-texel 2-D lookup (photometry_gpu.cu.h:40-70) */
struct Phot {
    const gf_photometry_config *c;
    float tex(int color, float FeH, float Mr, bool &flag) const
    {
        float xi = (FeH - c->tcFeH[0]) * c->tcFeH[1] + 0.5f;
        float yi = (Mr - c->tcMr[0]) * c->tcMr[1] + 0.5f;
        if (xi < 0.f) xi = 0.f; else if (xi >= (float)c->nFeH) xi = (float)c->nFeH - 1;
        if (yi < 0.f) yi = 0.f; else if (yi >= (float)c->nMr) yi = (float)c->nMr - 1;
        uint32_t i = (uint32_t)xi, j = (uint32_t)yi;
        size_t off = ((size_t)color * c->nMr + j) * c->nFeH + i;
        flag = c->eflags[off] != 0;
        return c->colors[off];
    }
};

uint32_t brev32(uint32_t a)     /* photometry_gpu.cu.h:76-84 */
{
    a = ((a >> 1) & 0x55555555) + ((a & 0x55555555) << 1);
    a = ((a >> 2) & 0x33333333) + ((a & 0x33333333) << 2);
    a = ((a >> 4) & 0x0F0F0F0F) + ((a & 0x0F0F0F0F) << 4);
    a = ((a >> 8) & 0x00FF00FF) + ((a & 0x00FF00FF) << 8);
    a = (a >> 16) + (a << 16);
    return a;
}

/* Philox4x32-10 (Salmon et al. 2011, "Parallel random numbers: as easy as 1, 2, 3") */
void philox4x32_10(uint32_t ctr[4], const uint32_t key_in[2])
{
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * ctr[0];
        uint64_t p1 = (uint64_t)0xCD9E8D57u * ctr[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        uint32_t n3 = lo0;
        ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

/* Standard normal deviate for (seed, row, band): Box-Muller on two 53-bit uniforms. */
double error_normal(uint64_t seed, uint64_t row, uint32_t band)
{
    uint32_t ctr[4] = {(uint32_t)row, (uint32_t)(row >> 32), band, 0x67616c66u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    philox4x32_10(ctr, key);
    uint64_t a = ((uint64_t)ctr[0] << 21) ^ (ctr[1] >> 11);
    uint64_t b = ((uint64_t)ctr[2] << 21) ^ (ctr[3] >> 11);
    double u1 = ((double)(a & ((1ull << 53) - 1)) + 1.0) * 0x1p-53;   /* (0, 1] */
    double u2 = (double)(b & ((1ull << 53) - 1)) * 0x1p-53;           /* [0, 1) */
    double r = sqrt(-2.0 * OR_LOG(u1));
    return r * OR_COS(6.283185307179586 * u2);
}

/* vel2pm_gpu.cu.h:52-61 */
void vel_xyz2lbr(float &vl, float &vb, float &vr, const float vx, const float vy, const float vz, const float l, const float b)
{
    float cl, sl, cb, sb;
    cl = OR_COSF(l); sl = OR_SINF(l); cb = OR_COSF(b); sb = OR_SINF(b);
    float tmp;
    vl = -vx * sl + vy * cl;
    tmp = vx * cl + vy * sl;
    vr = cb * tmp + vz * sb;
    vb = -sb * tmp + vz * cb;
}

/* vel2pm_gpu.cu.h:89-97 */
void vel_cyl2xyz(float &vx, float &vy, float &vz, const float vr, const float vphi, const float vz0, const float X, const float Y)
{
    float rho = sqrtf(X * X + Y * Y);
    float cphi = X / rho;
    float sphi = Y / rho;
    vx = -sphi * vphi + cphi * vr;
    vy = cphi * vphi + sphi * vr;
    vz = vz0;
}

/* galequ constants (module_lib.h:60-71) */
const double GE_angp = dbl_d2r * 192.859508333;
const double GE_l0 = dbl_d2r * 32.932;
const double GE_ce = 0.88998740217659689;
const double GE_se = 0.45598511375586859;

/* vel2pm_gpu.cu.h:109-137 */
void transform_pm(float &vlout, float &vbout, float l, float b, float vl, float vb, const double ce, const double se, const double l0)
{
    double cb = OR_COS(b);
    double sb = OR_SIN(b);
    double cl = OR_COS(l - l0);
    double sl = OR_SIN(l - l0);
    double tmp1 = cb * se - ce * sb * sl;
    double tmp2 = ce * sb - cb * se * sl;
    double tmp4 = cb * cl;
    double tmp3 = sb * se + cb * ce * sl;
    if (fabs(tmp3) > 0.9999999) {
        vlout = vbout = 999.99;
    } else {
        double denom1 = 1. / (tmp4 * tmp4 + tmp2 * tmp2);
        double cd = sqrt(1. - tmp3 * tmp3);
        vl /= cb;
        vlout = (-ce * cl * vb + cb * tmp1 * vl) * denom1;
        vbout = (tmp1 * vb + cb * ce * cl * vl) / cd;
        vlout *= cd;
    }
}

}  // namespace

/* ================================================================== */
/* C API                                                               */
/* ================================================================== */
extern "C" {

const char *or_last_error(void) { return g_err.c_str(); }

/* Number of host threads for the loops over independent streams (default 1). */
void or_set_threads(int n) { g_nthreads_cpu = n < 1 ? 1 : n; }

int or_math_portable(void)
{
#ifdef OR_PORTABLE
    return 1;
#else
    return 0;
#endif
}

/* Seeding of the persistent streams (cux.cpp:404-414, cuda_rng.h:466-497) with
 * glibc's srand48/drand48/lrand48 (on several host threads: the same recurrence
 * with jump-ahead).  `primes` holds the stream multipliers.
 * (int)(drand48()*prime) uses the x86 conversion: out-of-range values become INT_MIN. */
int or_rng_seed(uint32_t seed, int32_t nstreams, const uint32_t *primes, uint32_t *state)
{
    if (nstreams % 64) nstreams += 64 - nstreams % 64;
    if (g_nthreads_cpu > 1) {
        /* the same draws from the drand48 recurrence x' = (0x5DEECE66D x + 11) mod 2^48
         * (POSIX), with each block of streams jumping ahead to its first draw */
        const uint64_t A = 0x5DEECE66DULL, Cc = 0xB, M48 = (1ULL << 48) - 1;
        const uint64_t x0 = (((uint64_t)seed << 16) | 0x330E) & M48;
        const int per = 256;
        parallel_for((nstreams + per - 1) / per, [&](int blk) {
            /* x after 2 * blk * per steps: x_n = A^n x0 + C (A^n - 1) / (A - 1), by squaring */
            uint64_t n = 2ULL * blk * per, ma = 1, mc = 0, pa = A, pc = Cc;
            while (n) {
                if (n & 1) { ma = (ma * pa) & M48; mc = (mc * pa + pc) & M48; }
                pc = (pc * (pa + 1)) & M48;
                pa = (pa * pa) & M48;
                n >>= 1;
            }
            uint64_t x = (ma * x0 + mc) & M48;
            const int i1 = std::min(nstreams, (blk + 1) * per);
            for (int i = blk * per; i < i1; i++) {
                uint32_t prime = primes[i];
                state[i] = prime;
                x = (A * x + Cc) & M48;
                double t = ldexp((double)x, -48) * prime;
                int32_t cv = (t >= 2147483648.0) ? INT32_MIN : (int32_t)t;
                state[nstreams + i] = (uint32_t)cv;
                x = (A * x + Cc) & M48;
                state[2 * nstreams + i] = (uint32_t)(x >> 17);
            }
        }, 1);
        return nstreams;
    }
    srand48(seed);
    for (int i = 0; i != nstreams; i++) {
        uint32_t prime = primes[i];
        state[i] = prime;
        double t = drand48() * prime;
        int32_t cv = (t >= 2147483648.0) ? INT32_MIN : (int32_t)t;
        state[nstreams + i] = (uint32_t)cv;
        state[2 * nstreams + i] = (uint32_t)lrand48();
    }
    return nstreams;
}

/* n uniforms of one stream (for the known-answer tests) */
void or_mwc_uniforms(uint32_t *a, uint32_t *c, uint32_t *x, int n, float *out)
{
    Rng r = {*a, *c, *x};
    for (int i = 0; i < n; i++) out[i] = r.uniform();
    *a = r.a; *c = r.c; *x = r.xn;
}

/* n Poisson / Gaussian draws of one stream */
void or_mwc_poisson(uint32_t *a, uint32_t *c, uint32_t *x, const float *mu, int n, uint32_t *out)
{
    Rng r = {*a, *c, *x};
    for (int i = 0; i < n; i++) out[i] = r.poisson(mu[i]);
    *a = r.a; *c = r.c; *x = r.xn;
}
void or_mwc_gaussian(uint32_t *a, uint32_t *c, uint32_t *x, float sigma, int n, float *out)
{
    Rng r = {*a, *c, *x};
    for (int i = 0; i < n; i++) out[i] = r.gaussian(sigma);
    *a = r.a; *c = r.c; *x = r.xn;
}

void *or_skygen_create(const gf_skygen_config *cfg, const gf_pencil_beam *pixels, int32_t npixels,
                       const float *beam_ammin, const gf_extinction *ext,
                       const gf_model_config *mc, int32_t nmodels)
{
    Sky *s = new Sky();
    s->cfg = *cfg;
    s->pixels.assign(pixels, pixels + npixels);
    s->ext = ext ? *ext : gf_extinction{GF_EXT_NONE, 0.f, nullptr, nullptr};
    if (s->ext.kind == GF_EXT_MAPS) {
        const gf_ext_map *e = s->ext.north ? s->ext.north : s->ext.south;
        if (e) {
            s->ext_nz = e->n[2];
            s->ext_tcz[0] = e->tc[2][0];
            s->ext_tcz[1] = e->tc[2][1];
        }
    }
    if (beam_ammin) s->ammin.assign(beam_ammin, beam_ammin + (size_t)npixels * s->ext_nz);

    /* load_skyPixelizationConfig (os_skygen.cpp:409-430) */
    float M0 = cfg->M0, M1 = cfg->M1, m0 = cfg->m0, m1 = cfg->m1, dm = cfg->dm, dM = dm;
    Model base = Model();
    base.dmin = cfg->dmin; base.dmax = cfg->dmax;
    base.m1 = m1; base.dm = dm;
    reset_absmag(base, M0, M1, dM);
    base.nm = (int)round((m1 - m0) / dm);
    base.m0 = m0 + 0.5 * dm;
    base.npixels = npixels;
    base.nthreads = cfg->nthreads;

    for (int i = 0; i < nmodels; i++) {
        const gf_model_config &c = mc[i];
        Model m = base;
        m.type = c.type;
        m.comp = c.comp;
        m.norm = 1.f;
        load_transform(c, m.T, m.M);
        m.l = (float)c.l; m.h = (float)c.h; m.r_cut2 = 0.f;
        m.n = (float)c.n; m.ba = (float)c.ba; m.ca = (float)c.ca;
        m.rminSq = m.rmaxSq = 0.f;
        m.nbreaks = 0;
        if (c.type == GF_MODEL_BROKEN_POWER_LAW) {
            /* brokenPowerLaw::load (model_brokenPowerLaw.cpp:31-62) */
            m.nbreaks = c.nbreaks;
            for (int k = 0; k <= c.nbreaks; k++) m.nArr[k] = (float)c.n_brk[k];
            for (int k = 0; k < c.nbreaks; k++) { float rb = (float)c.rbreak[k]; m.rbreakSq[k] = rb * rb; }
            m.fArr[0] = m.f = 1.f;
            for (int k = 0; k < m.nbreaks; k++)
                m.fArr[k + 1] = m.fArr[k] * OR_POWF(m.rbreakSq[k], 0.5f * (m.nArr[k] - m.nArr[k + 1]));
        }
        /* load_lf (model_lib.h:68-95); the LC bulge: load_lf_raw times f (model_LCBulge.cpp:50-56) */
        load_lf(m, c);
        if (c.type == GF_MODEL_DENSITY_CUBE) {
            /* densityCube::load (model_densityCube.cpp:250-300): f, Rg, the grid; the LF by
             * load_and_resample_texture_1D (no clipping), no normalisation */
            m.f = (float)c.f;
            m.Rg = (float)c.Rg;
            m.cube = c.cube;
            for (int k = 0; k < 3; k++) {
                m.cube_n[k] = c.cube_n[k];
                m.cube_tc[k][0] = c.cube_tc[k][0];
                m.cube_tc[k][1] = c.cube_tc[k][1];
            }
            if (c.lf_n > 0 && c.lf_M) {
                std::vector<double> X(c.lf_M, c.lf_M + c.lf_n), Y(c.lf_phi, c.lf_phi + c.lf_n);
                int ndata = (int)X.size(), nsamp = 1024;
                m.lf.resize(nsamp);
                double X0 = X[0], X1 = X[ndata - 1], dX = (X1 - X0) / (nsamp - 1);
                for (int i = 0; i != nsamp; i++) m.lf[i] = (float)linear_eval(X.data(), Y.data(), ndata, X0 + i * dX);
                m.lf_x0 = (float)X0;
                m.lf_inv_dx = (float)(1. / dX);
            }
        } else if (c.type == GF_MODEL_LCBULGE) {
            float f0 = (float)c.f;
            for (auto &v : m.lf) v *= f0;
            m.f = 1.f;
        } else {
            float lfx = (float)c.lf_l, lfy = (float)c.lf_b, lfz = (float)c.lf_D;
            Dir d = make_dir(lfx * dbl_d2r, lfy * dbl_d2r);
            F3 lfc = {lfz * d.cl * d.cb, lfz * d.sl * d.cb, lfz * d.sb};
            m.f = 1.f;
            float norm = m.rho(lfc.x, lfc.y, lfc.z);
            if (!(norm != 0.f && std::isnormal(norm))) {
                g_err = "LF normalisation point has zero density";
                delete s;
                return nullptr;
            }
            float f0 = (float)c.f;
            m.f = f0 / norm;
        }
        if (c.type == GF_MODEL_EXP_DISK) {
            float rc = (float)c.rcut;
            m.r_cut2 = rc * rc;
        } else if (c.type != GF_MODEL_LCBULGE && c.type != GF_MODEL_DENSITY_CUBE) {
            float rmin = (float)c.rmin, rmax = (float)c.rmax;
            m.rminSq = rmin * rmin;
            m.rmaxSq = rmax * rmax;
        }
        /* skygenHost<T>::init (skyconfig_impl.h:257-263): LF hint */
        float hM0 = m.M0, hM1 = m.M1 + 0.5 * m.dM;
        float X0 = m.lf_x0;
        float X1 = double(m.lf.size() - 1) / m.lf_inv_dx + X0;
        bool ret = false;
        if (X0 > hM0) { ret = true; hM0 = X0; }
        if (X1 < hM1) { ret = true; hM1 = X1; }
        if (ret) reset_absmag(m, hM0, hM1, m.dM);
        m.nstarsExpected = m.nstarsExpectedToGenerate = 0;
        s->models.push_back(m);
    }
    s->ks.resize(nmodels);
    s->ks_alloc.assign(nmodels, 0);
    return s;
}

void or_skygen_destroy(void *h) { delete (Sky *)h; }

int or_skygen_model_info(void *h, int32_t mi, gf_skygen_model_info *info)
{
    Sky *s = (Sky *)h;
    const Model &m = s->models[mi];
    info->m0 = m.m0; info->m1 = m.m1; info->dm = m.dm; info->M0 = m.M0; info->M1 = m.M1; info->dM = m.dM;
    info->nm = m.nm; info->nM = m.nM; info->npixels = m.npixels; info->nthreads = m.nthreads;
    info->f = m.f; info->lf_x0 = m.lf_x0; info->lf_inv_dx = m.lf_inv_dx; info->lf_n = (int)m.lf.size();
    info->norm = m.norm;
    return 0;
}

int or_skygen_model_lf(void *h, int32_t mi, float *lf)
{
    Sky *s = (Sky *)h;
    std::copy(s->models[mi].lf.begin(), s->models[mi].lf.end(), lf);
    return 0;
}

/* integrateCounts (skyconfig_impl.h:323-429), pixel blocks of PIXBLOCK */
int or_skygen_integrate(void *h, int32_t mi, double *expected, double *expected_covered, double *per_pixel)
{
    Sky *s = (Sky *)h;
    Model &m = s->models[mi];
    const int N = m.nthreads;
    const int lastpix = m.npixels;
    const int PIXBLOCK = 1024 * 1024 * 2 / N;
    std::vector<double> counts(N), countsCovered(N);
    std::vector<float> maxCount(N);
    double nE = 0, nEC = 0;
    int startpix = 0;
    while (startpix < lastpix) {
        int endpix = std::min(startpix + PIXBLOCK, lastpix);
        int npix = endpix - startpix;
        std::vector<float> ccpb((size_t)N * npix, 0.f);
        Launch L = {};
        L.sky = s; L.m = &m; L.npixels = npix; L.pixels = s->pixels.data() + startpix;
        L.counts = counts.data(); L.countsCovered = countsCovered.data();
        L.countsCoveredPerBeam = ccpb.data(); L.maxCount = maxCount.data();
        std::fill(counts.begin(), counts.end(), 0.);
        std::fill(countsCovered.begin(), countsCovered.end(), 0.);
        parallel_for(N, [&](int tid) { kernel(L, 0, tid); }, 64);
        for (int i = 0; i != N; i++) { nE += counts[i]; nEC += countsCovered[i]; }
        if (per_pixel) {
            for (int px = 0; px < npix; px++) {
                double rho = 0;
                for (int th = 0; th != N; th++) rho += ccpb[(size_t)th * npix + px];
                per_pixel[startpix + px] = rho;
            }
        }
        startpix = endpix;
    }
    m.nstarsExpectedToGenerate = nE;
    m.nstarsExpected = nEC;
    if (expected) *expected = nE;
    if (expected_covered) *expected_covered = nEC;
    return 0;
}

/* Diagnostics for the tests: the number of bins of one model whose expected
 * count exceeds `above` (e.g. 10, where rng::poisson switches to the gamma /
 * binomial reduction, cuda_rng.h:344-376), by the integrate crawl of
 * or_skygen_integrate. */
int or_count_bins_above(void *h, int32_t mi, float above, int64_t *count)
{
    Sky *s = (Sky *)h;
    Model &m = s->models[mi];
    const int N = m.nthreads;
    const int lastpix = m.npixels;
    const int PIXBLOCK = 1024 * 1024 * 2 / N;
    std::vector<double> counts(N), countsCovered(N);
    std::vector<float> maxCount(N);
    std::vector<int64_t> nab(N, 0);
    for (int startpix = 0; startpix < lastpix; startpix += PIXBLOCK) {
        int npix = std::min(startpix + PIXBLOCK, lastpix) - startpix;
        std::vector<float> ccpb((size_t)N * npix, 0.f);
        Launch L = {};
        L.sky = s; L.m = &m; L.npixels = npix; L.pixels = s->pixels.data() + startpix;
        L.counts = counts.data(); L.countsCovered = countsCovered.data();
        L.countsCoveredPerBeam = ccpb.data(); L.maxCount = maxCount.data();
        L.nabove = nab.data(); L.above = above;
        parallel_for(N, [&](int tid) { kernel(L, 0, tid); }, 64);
    }
    int64_t t = 0;
    for (int i = 0; i < N; i++) t += nab[i];
    *count = t;
    return 0;
}

/* The precision form's FP64 oracle for one pixel: every bin in the crawl's order
 * with its anchor at the block starts (every 10th bin, nm*nM a multiple of 10)
 * and the diagonal starts, the reference's float expected count (skygen.cu.h:
 * 541-565, summed in double) and the same bin evaluated in double throughout
 * (D = 10^(0.2 DM + 1), model density, D^3 dA POGSON dm dM; the LF texel and the
 * float model parameters as given). */
int or_expected_fp64(void *h, int32_t mi, int32_t px, double *sum32, double *sum64)
{
    Sky *s = (Sky *)h;
    const Model &m = s->models[mi];
    const int nm = m.nm, nM = m.nM, kmax = nm * nM;
    if (px < 0 || px >= (int)s->pixels.size() || kmax % BLOCK) return 1;
    Launch L = {};
    L.sky = s; L.m = &m; L.npixels = (int)s->pixels.size(); L.pixels = s->pixels.data();
    const gf_pencil_beam pix = s->pixels[px];
    double a32 = 0, a64 = 0;
    float D = 0, Am = 0, ms = 0;
    double ms64 = 0, D364 = 0, K64 = 0;
    for (int k = 0; k < kmax; k++) {
        int ilb = 0, im, iM, kk = k;
        diagIndexToIJ(ilb, im, iM, kk, nm, nM);
        const bool anchor = (k % BLOCK == 0) || im == 0 || iM == nM - 1;
        const float M = m.M1 - iM * m.dM;
        if (anchor) {
            F3 pos = compute_pos(L, D, Am, M, im, pix);
            ms = m.rho(pos.x, pos.y, pos.z);
            const double Md = (double)m.M1 - (double)iM * (double)m.dM;
            const double mm = (double)m.m0 + (double)im * (double)m.dm;
            const double Dd = pow(10.0, 0.2 * (mm - Md) + 1.0);
            const double x = Dd * (double)pix.cl * (double)pix.cb, y = Dd * (double)pix.sl * (double)pix.cb, z = Dd * (double)pix.sb;
            const double vx = x + m.T[0], vy = y + m.T[1], vz = z + m.T[2];
            const double wx = m.M[0][0] * vx + m.M[0][1] * vy + m.M[0][2] * vz;
            const double wy = m.M[1][0] * vx + m.M[1][1] * vy + m.M[1][2] * vz;
            const double wz = m.M[2][0] * vx + m.M[2][1] * vy + m.M[2][2] * vz;
            if (m.type == GF_MODEL_EXP_DISK) {
                const double r2 = wx * wx + wy * wy;
                ms64 = (m.r_cut2 && r2 + wz * wz > m.r_cut2) ? 0.0 : m.f * exp(-sqrt(r2) / m.l - fabs(wz) / m.h);
            } else if (m.type == GF_MODEL_LCBULGE) {
                const double t = pow(pow(wx, (double)m.n) + pow(wy / m.ba, (double)m.n) + pow(wz / m.ca, (double)m.n), 1.0 / m.n);
                ms64 = exp(-t / m.l);
            } else {
                const double DSq = wx * wx + wy * wy + wz * wz;
                const double ty = wy / m.ba, tz = wz / m.ca;
                const double rSq = wx * wx + ty * ty + tz * tz;
                int k = 0;
                while (k != m.nbreaks && rSq > m.rbreakSq[k]) k++;
                const double nk = m.type == GF_MODEL_BROKEN_POWER_LAW ? m.nArr[k] : m.n;
                const double fk = m.type == GF_MODEL_BROKEN_POWER_LAW ? m.fArr[k] : 1.0;
                ms64 = (m.rmaxSq && (DSq < m.rminSq || DSq >= m.rmaxSq)) ? 0.0 : m.f * fk * pow(rSq, 0.5 * nk);
            }
            D364 = Dd * Dd * Dd;
            K64 = (double)pix.dA * 0.46051701859880913680 * (double)m.dm * (double)m.dM;
        }
        if ((m.dmin || m.dmax) && (m.dmin > D || m.dmax <= D)) continue;
        if (m.m0 + m.dm * im + Am > m.m1) continue;
        const float lfv = m.lf_sample(M);
        float rho = lfv * ms;
        rho *= m.norm;
        rho *= D * D * D;
        rho *= pix.dA * POGSON * m.dm * m.dM;
        a32 += rho;
        a64 += (double)lfv * ms64 * (double)m.norm * D364 * K64;
    }
    *sum32 = a32;
    *sum64 = a64;
    return 0;
}

/* setDensityNorm (skyconfig_impl.h:308-320) */
int or_skygen_set_norm(void *h, int32_t mi, float norm)
{
    Sky *s = (Sky *)h;
    Model &m = s->models[mi];
    m.norm = norm;
    m.nstarsExpected *= norm;
    m.nstarsExpectedToGenerate *= norm;
    return 0;
}

/* One iteration of drawSources' batch loop (skyconfig_impl.h:445-515):
 * draw into the host table t (capacity rows), sort, truncate.  rng_state is
 * the persistent [3][nstreams] stream state, updated in place. */
int or_skygen_draw(void *h, int32_t mi, uint32_t *rng_state, int32_t nstreams, gf_table *t,
                   int64_t *n_generated, int32_t *done)
{
    Sky *s = (Sky *)h;
    Model &m = s->models[mi];
    if (!s->ks_alloc[mi]) { s->ks[mi].alloc(m.nthreads); s->ks_alloc[mi] = 1; }
    const int stopstars = (int)t->capacity;
    RngState rs = {rng_state, nstreams};
    int64_t nstars = 0;
    if (g_nthreads_cpu <= 1) {
        /* the reference CPU build: emulated threads one after another */
        int n = 0;
        Launch L = {};
        L.sky = s; L.m = &m; L.npixels = m.npixels; L.pixels = s->pixels.data();
        L.stopstars = stopstars;
        L.nstars = &n;
        L.out = t;
        L.ks = &s->ks[mi];
        L.rng = rs;
        for (int tid = 0; tid < m.nthreads; tid++) kernel(L, 1, tid);
        nstars = n;
    } else {
        draw_parallel(s, m, s->ks[mi], rs, t, stopstars, &nstars);
    }
    int stars_generated = (int)std::min<int64_t>(nstars, stopstars);
    int generated_all = stars_generated < stopstars;

    /* sort by (hidden, l, b, DM, M, Am) and truncate at the first hidden row */
    std::vector<size_t> idx(stars_generated);
    for (int i = 0; i < stars_generated; i++) idx[i] = i;
    t->size = stars_generated;
    StarComp sc = {t};
    sort_rows(idx, sc);
    const int64_t P = t->capacity;
    const int n = stars_generated;
    parallel_for(14, [&](int c) {
        switch (c) {
        case 0: permute(t->lb, idx, n); break;
        case 1: permute(t->lb + P, idx, n); break;
        case 2: permute(t->projIdx, idx, n); break;
        case 3: permute(t->projXY, idx, n); break;
        case 4: permute(t->projXY + P, idx, n); break;
        case 5: permute(t->Am, idx, n); break;
        case 6: permute(t->AmInf, idx, n); break;
        case 7: permute(t->XYZ, idx, n); break;
        case 8: permute(t->XYZ + P, idx, n); break;
        case 9: permute(t->XYZ + 2 * P, idx, n); break;
        case 10: permute(t->comp, idx, n); break;
        case 11: permute(t->absmag, idx, n); break;
        case 12: permute(t->DM, idx, n); break;
        case 13: permute(t->hidden, idx, n); break;
        }
    }, 1);
    int32_t *h0 = std::upper_bound(t->hidden, t->hidden + stars_generated, 0);
    t->size = h0 - t->hidden;
    *n_generated = stars_generated;
    *done = generated_all;
    return 0;
}

/* Per-stream star counts of a full single-batch draw, without writing rows
 * (diagnostics for the batch tests): out[tid] = stars drawn by thread tid. */

/* ---- modules on a host table, rows [begin, end) ---- */

/* os_clipper::process (os_skygen.cpp:999-1044) with an analytic footprint */
/* The footprint regions (footprint.cpp: load_footprint_beam :675-704, load_footprint_rect
 * :486-589, clip_zone_of_avoidance :706-727, the union of load_footprints :746-758), tested
 * exactly on the sphere: equatorial coordinates through the Hipparcos (J2000) rotation. */
static bool or_region_inside(const gf_region &r, double l, double b)
{
    if (r.bmin > 0.0 && fabs(b) < r.bmin) return false;
    double lon = l * dbl_d2r, lat = b * dbl_d2r;
    if (r.coordsys == GF_COORD_EQU) {
        static const double A[3][3] = {{-0.0548755604162154, -0.8734370902348850, -0.4838350155487132},
                                       {+0.4941094278755837, -0.4448296299600112, +0.7469822444972189},
                                       {-0.8676661490190047, -0.1980763734312015, +0.4559837761750669}};
        const double g[3] = {OR_COS(lat) * OR_COS(lon), OR_COS(lat) * OR_SIN(lon), OR_SIN(lat)};
        double e[3];
        for (int i = 0; i < 3; i++) e[i] = A[0][i] * g[0] + A[1][i] * g[1] + A[2][i] * g[2];
        lon = OR_ATAN2(e[1], e[0]);
        lat = OR_ASIN(std::max(-1.0, std::min(1.0, e[2])));
    }
    if (r.type == GF_REGION_BEAM) {
        const double l0 = r.a * dbl_d2r, b0 = r.b * dbl_d2r;
        const double cosd = OR_SIN(lat) * OR_SIN(b0) + OR_COS(lat) * OR_COS(b0) * OR_COS(lon - l0);
        if (r.c < 180.0 && !(cosd >= OR_COS(r.c * dbl_d2r))) return false;
        if (r.d > 0.0 && cosd > OR_COS(r.d * dbl_d2r)) return false;
        return true;
    }
    if (r.type == GF_REGION_RECT) {
        const double latd = lat / dbl_d2r;
        if (!(latd >= r.c && latd < r.d)) return false;
        if (r.a == r.b) return true;
        double lond = fmod(lon / dbl_d2r, 360.0);
        if (lond < 0) lond += 360.0;
        double a = fmod(r.a, 360.0), e = fmod(r.b, 360.0);
        if (a < 0) a += 360.0;
        if (e < 0) e += 360.0;
        return (a <= e) ? (lond >= a && lond < e) : (lond >= a || lond < e);
    }
    return false;
}

int or_module_clipper(const gf_footprint *foot, const gf_lambert *proj, gf_table *t, int64_t begin, int64_t end)
{
    (void)proj;
    const int64_t P = t->capacity;
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int64_t row = begin + rb_; row < begin + re_; row++) {
            if (t->hidden[row]) continue;
            bool in = true;
            if (foot->kind == GF_FOOT_LAMBERT_RECT) {
                float x = t->projXY[row], y = t->projXY[P + row];
                in = t->projIdx[row] == foot->proj && x >= foot->a && x < foot->b && y >= foot->c && y < foot->d;
            } else if (foot->kind == GF_FOOT_CAP) {
                double l = t->lb[row] * dbl_d2r, b = t->lb[P + row] * dbl_d2r;
                double l0 = foot->a * dbl_d2r, b0 = foot->b * dbl_d2r;
                double cosd = OR_SIN(b) * OR_SIN(b0) + OR_COS(b) * OR_COS(b0) * OR_COS(l - l0);
                in = cosd >= OR_COS(foot->c * dbl_d2r);
            } else if (foot->kind == GF_FOOT_LATCUT) {
                in = fabs(t->lb[P + row]) > foot->a;
            } else if (foot->kind == GF_FOOT_LB_RECT) {
                const double l = t->lb[row], b = t->lb[P + row];
                in = b >= foot->c && b < foot->d &&
                     ((foot->a <= foot->b) ? (l >= foot->a && l < foot->b) : (l >= foot->a || l < foot->b));
            } else if (foot->kind == GF_FOOT_REGIONS) {
                in = false;
                for (int q = 0; q < foot->nregions && q < GF_MAX_REGIONS && !in; q++)
                    in = or_region_inside(foot->regions[q], t->lb[row], t->lb[P + row]);
            }
            if (!in) t->hidden[row] = 1;
        }
    });
    return 0;
}

/* os_fixedFeH_kernel (fixedFeH_gpu.cu.h:34-50) */
int or_module_fixedfeh(const gf_fixedfeh_config *c, gf_table *t, int64_t begin, int64_t end)
{
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int64_t row = begin + rb_; row < begin + re_; row++) {
            if (t->hidden[row]) continue;
            int cmp = t->comp[row];
            if (!((c->comp_mask >> cmp) & 1u)) continue;
            t->FeH[row] = c->FeH;
        }
    });
    return 0;
}

/* os_Bond2010_kernel (Bond2010_gpu.cu.h:81-218): thread t owns rows
 * [begin + 256 t, begin + 256 (t+1)) and stream t of the persistent state. */
static float modfun(float Rsquared, float Z, const float val[5])
{
    return val[0] + val[1] * OR_POWF(fabsf(Z), val[2]) + val[3] * OR_POWF(Rsquared, (float)(0.5 * val[4]));
}

static void trivar_gaussK_draw(float y[3], float s11, float s12, float s13, float s22, float s23, float s33, Rng &rng)
{
    float b10 = s12;      float b11 = s22 * s22;
    float b20 = s13;      float b21 = s23;      float b22 = s33 * s33;
    float a00 = s11; float oneDivA00 = 1.0f / a00;
    float a10 = (b10) * oneDivA00;
    float a11 = sqrtf(b11 - a10 * a10);
    float a20 = (b20) * oneDivA00;
    float a21 = (b21 - a20 * a10) / a11;
    float a22 = sqrtf(b22 - a20 * a20 - a21 * a21);
    float z0 = rng.gaussian(1.0f);
    float z1 = rng.gaussian(1.0f);
    float z2 = rng.gaussian(1.0f);
    y[0] += a00 * z0;
    y[1] += a10 * z0 + a11 * z1;
    y[2] += a20 * z0 + a21 * z1 + a22 * z2;
}

static void add_dispersion(float v[3], float Rsquared, float Z, const float ellip[6][5], Rng &rng)
{
    float sigma[6];
    for (int i = 0; i < 6; i++) sigma[i] = modfun(Rsquared, Z, ellip[i]);
    trivar_gaussK_draw(v, sigma[0], sigma[1], sigma[2], sigma[3], sigma[4], sigma[5], rng);
}

static void compute_means(float v[3], float Rsquared, float Z, const float means[3][5])
{
    for (int i = 0; i < 3; i++) v[i] = modfun(Rsquared, Z, means[i]);
}

int or_module_bond2010(const gf_bond2010_config *par, uint32_t *rng_state, int32_t nstreams,
                       gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    RngState rs = {rng_state, nstreams};
    int64_t n = end - begin;
    int64_t nth = n / 256 + (n % 256 ? 1 : 0);
    if (nth > nstreams) { g_err = "Bond2010: more than 256*nstreams rows"; return -1; }
    parallel_for((int)nth, [&](int th) {
        Rng rng = rs.load((int)th);
        int64_t rb = begin + 256 * th, re = std::min(begin + 256 * (th + 1), end);
        for (int64_t row = rb; row < re; row++) {
            if (t->hidden[row]) continue;
            const int cmp = t->comp[row];
            float vx = t->XYZ[row] + par->T[0], vy = t->XYZ[P + row] + par->T[1], vz = t->XYZ[2 * P + row] + par->T[2];
            float wx = par->M[0] * vx + par->M[1] * vy + par->M[2] * vz;
            float wy = par->M[3] * vx + par->M[4] * vy + par->M[5] * vz;
            float wz = par->M[6] * vx + par->M[7] * vy + par->M[8] * vz;
            const float Rsquared = (float)(1e-6 * (wx * wx + wy * wy));
            const float Z = (float)(1e-3 * wz);
            float tmp[3];
            if (((par->comp_thin | par->comp_thick) >> cmp) & 1u) {
                float p = rng.uniform();
                const gf_vmoments &disk = p < par->fk ? par->disk_1 : par->disk_2;
                compute_means(tmp, Rsquared, Z, disk.m);
                if (tmp[1] > 0.) tmp[1] = 0.;
                add_dispersion(tmp, Rsquared, Z, disk.ss, rng);
            } else if ((par->comp_halo >> cmp) & 1u) {
                compute_means(tmp, Rsquared, Z, par->halo.m);
                add_dispersion(tmp, Rsquared, Z, par->halo.ss, rng);
                float invR = 1.f / sqrtf(Rsquared + Z * Z);
                float cosa = sqrtf(Rsquared) * invR;
                float sina = Z * invR;
                float vR = cosa * tmp[0] - sina * tmp[1];
                float vZ = sina * tmp[0] + cosa * tmp[1];
                tmp[0] = vR;
                tmp[1] = tmp[2];
                tmp[2] = vZ;
            } else {
                continue;
            }
            t->vcyl[row] = tmp[0];
            t->vcyl[P + row] = tmp[1];
            t->vcyl[2 * P + row] = tmp[2];
        }
        rs.store((int)th, rng);
    }, 16);
    return 0;
}

/* os_FeH_kernel (FeH_gpu.cu.h:43-87) and os_GaussianFeH_kernel
 * (GaussianFeH_gpu.cu.h:42-73): thread t owns rows [begin + 256 t, ...) and
 * stream t.  exp(-|Z|/Hmu) is evaluated in single precision (the GPU build's
 * float overload) with this flavour's expf. */
int or_module_feh(const gf_feh_config *par, uint32_t *rng_state, int32_t nstreams, gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    RngState rs = {rng_state, nstreams};
    const int64_t n = end - begin, nth = n / 256 + (n % 256 ? 1 : 0);
    if (nth > nstreams) { g_err = "FeH: more than 256*nstreams rows"; return -1; }
    parallel_for((int)nth, [&](int th) {
        Rng rng = rs.load(th);
        const int64_t rb = begin + 256 * (int64_t)th, re = std::min(begin + 256 * ((int64_t)th + 1), end);
        for (int64_t row = rb; row < re; row++) {
            if (t->hidden[row]) continue;
            const int cmp = t->comp[row];
            if (((par->comp_thin | par->comp_thick) >> cmp) & 1u) {
                float p = rng.uniform() * (par->A[0] + par->A[1]);
                int i = p < par->A[0] ? 0 : 1;
                float vx = t->XYZ[row] + par->T[0], vy = t->XYZ[P + row] + par->T[1], vz = t->XYZ[2 * P + row] + par->T[2];
                float z = par->M[6] * vx + par->M[7] * vy + par->M[8] * vz;
                float muD = par->muInf + par->DeltaMu * OR_EXPF(-fabsf(z) / par->Hmu);
                float aZ = muD - 0.067f;
                float feh = rng.gaussian(par->sigma[i]) + aZ + par->offs[i];
                t->FeH[row] = feh;
            } else if ((par->comp_halo >> cmp) & 1u) {
                float feh = par->offs[2] + rng.gaussian(par->sigma[2]);
                t->FeH[row] = feh;
            }
        }
        rs.store(th, rng);
    }, 4);
    return 0;
}

int or_module_gaussfeh(const gf_gaussfeh_config *par, uint32_t *rng_state, int32_t nstreams, gf_table *t, int64_t begin,
                       int64_t end)
{
    RngState rs = {rng_state, nstreams};
    const int64_t n = end - begin, nth = n / 256 + (n % 256 ? 1 : 0);
    if (nth > nstreams) { g_err = "GaussianFeH: more than 256*nstreams rows"; return -1; }
    parallel_for((int)nth, [&](int th) {
        Rng rng = rs.load(th);
        const int64_t rb = begin + 256 * (int64_t)th, re = std::min(begin + 256 * ((int64_t)th + 1), end);
        for (int64_t row = rb; row < re; row++) {
            if (t->hidden[row]) continue;
            int cmp = t->comp[row];
            if (!((par->comp_mask >> cmp) & 1u)) continue;
            int at = 0;
            if (par->ncomp != 1) {
                float u = rng.uniform();
                while (par->pcum[at] < u) ++at;
            }
            t->FeH[row] = par->mean[at] + rng.gaussian(par->sigma[at]);
            t->FeH_comp[row] = at;
        }
        rs.store(th, rng);
    }, 4);
    return 0;
}

/* nearest-texel 1-D table lookup of the host build (cux.h:786-792, 849-855) */
static float tex1(const float *tab, int n, float x0, float inv_dx, float x)
{
    float xi = (x - x0) * inv_dx + 0.5f;
    if (xi < 0.f) xi = 0.f;
    else if (xi >= (float)n) xi = (float)(n - 1);
    return tab[(uint32_t)xi];
}

/* os_unresolvedMultiples_kernel (unresolvedMultiples_gpu.cu.h:46-123): two system
 * components; rows the module skips hold a single-star system */
int or_module_multiples(const gf_multiples_config *c, uint32_t *rng_state, int32_t nstreams, gf_table *t, int64_t begin,
                        int64_t end)
{
    const int64_t P = t->capacity;
    RngState rs = {rng_state, nstreams};
    const int64_t n = end - begin, nth = n / 256 + (n % 256 ? 1 : 0);
    if (nth > nstreams) { g_err = "unresolvedMultiples: more than 256*nstreams rows"; return -1; }
    parallel_for((int)nth, [&](int th) {
        Rng rng = rs.load(th);
        const int64_t rb = begin + 256 * (int64_t)th, re = std::min(begin + 256 * ((int64_t)th + 1), end);
        for (int64_t row = rb; row < re; row++) {
            const float M1 = t->absmag[row];
            t->absmagSys[row] = M1;
            if (t->hidden[row] || !((c->comp_mask >> t->comp[row]) & 1u)) {
                t->absmagSys[P + row] = 99.999f;
                t->absmagSysNcomp[row] = 1;
                continue;
            }
            float Ltot = OR_EXP10F(-0.4f * M1);
            int ncomps = 1;
            /* draw_companion */
            bool has = false;
            float M2 = 0.f;
            const float psec = tex1(c->secprob, c->nsec, c->sec_x0, c->sec_inv_dx, M1);
            float u = rng.uniform();
            if (!(u > psec)) {
                has = true;
                if (c->algo == GF_MULT_EQUAL_MASS) {
                    M2 = M1;
                } else {
                    const float pprim = tex1(c->cumlf, c->ncum, c->cum_x0, c->cum_inv_dx, M1);
                    u = rng.uniform();
                    if (c->algo == GF_MULT_LF_M2_GT_M1) u = pprim + u * (1. - pprim);
                    M2 = tex1(c->invcumlf, c->ninv, c->inv_x0, c->inv_inv_dx, u);
                    if (c->algo == GF_MULT_LF_M2_GT_M1 && M2 < M1) M2 = M1;
                }
            }
            if (has) {
                t->absmagSys[P + row] = M2;
                Ltot += OR_EXP10F(-0.4f * M2);
                ncomps++;
            } else {
                t->absmagSys[P + row] = 99.999f;
            }
            float Mtot = -2.5 * OR_LOG10F(Ltot);
            t->absmag[row] = Mtot;
            t->absmagSysNcomp[row] = ncomps;
        }
        rs.store(th, rng);
    }, 4);
    t->systems = 1;
    return 0;
}

/* os_photometry_kernel (photometry_gpu.cu.h:87-174); the system's components come
 * from absmagSys when unresolved multiples ran (photometry_host.cpp:373-376) */
int or_module_photometry(const gf_photometry_config *lt, gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    const int ncolors = lt->nbands - 1;
    const bool sys = t->systems && t->absmagSys;
    const float *Mr = sys ? t->absmagSys : t->absmag;
    const int nabsmag = sys ? 2 : 1;
    Phot ph = {lt};
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int64_t row = begin + rb_; row < begin + re_; row++) {
            float c[GF_MAX_BANDS];
            if (t->hidden[row]) continue;
            int cmp = t->comp[row];
            if (!((lt->comp_mask >> cmp) & 1u)) continue;
            float fFeH = t->FeH[row];
            uint32_t flag = 0;
            for (int syscomp = 0; syscomp < nabsmag; syscomp++) {
                float fMr = Mr[syscomp * P + row];
                if (fMr >= 99.999f) break;
                for (int ic = 0; ic < ncolors; ic++) {
                    bool fl;
                    c[ic] = ph.tex(ic, fFeH, fMr, fl);
                    flag |= ((uint32_t)fl) << ic;
                }
                for (int b = 0; b <= ncolors; b++) {
                    float M = fMr;
                    if (b < lt->bidx) { for (int i = b; i != lt->bidx; i++) M += c[i]; }
                    if (b > lt->bidx) { for (int i = lt->bidx; i != b; i++) M -= c[i]; }
                    float L = OR_EXP10F(-0.4f * M);
                    if (syscomp) L += t->mags[b * P + row];
                    t->mags[b * P + row] = L;
                }
            }
            bool fl = false;
            for (int i = lt->bidx - 1; i >= 0; i--) {
                uint32_t mask = 1u << i;
                fl = fl || (flag & mask);
                flag |= ((uint32_t)fl) << i;
            }
            fl = false;
            for (int i = lt->bidx; i < ncolors; i++) {
                uint32_t mask = 1u << i;
                fl = fl || (flag & mask);
                flag |= ((uint32_t)fl) << i << 1;
            }
            flag &= ~(1u << lt->bidx);
            flag = brev32(flag);
            flag >>= (8 * sizeof(flag) - ncolors - 1);
            t->photoflags[row] = (int32_t)flag;
            float dm = t->DM[row];
            float Am0 = t->Am[row];
            for (int b = 0; b <= ncolors; b++) {
                float Msys = -2.5f * OR_LOG10F(t->mags[b * P + row]);
                float msys = dm + Msys;
                float Am = Am0 * lt->reddening[b];
                t->mags[b * P + row] = msys + Am;
            }
        }
    });
    return 0;
}

/* os_photometricErrors::process (photometricErrors_host.cpp:112-131) with
 * counter-based Gaussian deviates keyed by (seed, row_offset + row, band). */
int or_module_photoerrors(const gf_photoerr_config *c, int64_t row_offset, gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int b = 0; b < c->nbands; b++) {
            const double *mk = c->mag + (size_t)b * c->nknots, *sk = c->sigma + (size_t)b * c->nknots;
            for (int64_t row = begin + rb_; row < begin + re_; row++) {
                if (t->hidden[row]) continue;
                float mag = t->mags[b * P + row];
                float sigma = (float)linear_eval(mk, sk, c->nknots, mag);
                double z = error_normal(c->seed, (uint64_t)(row_offset + row), (uint32_t)b);
                t->obsmags[b * P + row] = mag + (float)(sigma * z);
            }
        }
    });
    return 0;
}

/* os_vel2pm_kernel (vel2pm_gpu.cu.h:221-301) */
int or_module_vel2pm(const gf_vel2pm_config *par, gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int64_t row = begin + rb_; row < begin + re_; row++) {
            if (t->hidden[row]) continue;
            float l = 0.017453292519943295769f * (float)t->lb[row];
            float b = 0.017453292519943295769f * (float)t->lb[P + row];
            float X = par->Rg - t->XYZ[row];
            float Y = -t->XYZ[P + row];
            float Z = t->XYZ[2 * P + row];
            float vx = t->vcyl[row], vy = t->vcyl[P + row], vz = t->vcyl[2 * P + row];
            float px, py, pz;
            vel_cyl2xyz(px, py, pz, vx, vy, vz, X, Y);
            px -= par->u0;
            py -= par->v0 + par->vLSR;
            pz -= par->w0;
            vel_xyz2lbr(px, py, pz, -px, -py, pz, l, b);
            float D = sqrtf((8000.f - X) * (8000.f - X) + Y * Y + Z * Z);
            px = (float)(px / (4.74 * D * 1e-3));
            py = (float)(py / (4.74 * D * 1e-3));
            if (par->coordsys == 1) {
                transform_pm(px, py, l, b, px, py, GE_ce, GE_se, GE_l0);
            } else if (par->coordsys != 0) {
                px = py = pz = -9.99f;
            }
            t->pm[row] = px;
            t->pm[P + row] = py;
            t->pm[2 * P + row] = pz;
        }
    });
    return 0;
}

/* os_gal2other_kernel (gal2other_gpu.cu.h:39-96) */
int or_module_gal2other(int32_t coordsys, gf_table *t, int64_t begin, int64_t end)
{
    const int64_t P = t->capacity;
    const double pi2 = 2 * dbl_pi;
    parallel_rows(end - begin, [&](int64_t rb_, int64_t re_) {
        for (int64_t row = begin + rb_; row < begin + re_; row++) {
            if (t->hidden[row]) continue;
            double lx = t->lb[row] * dbl_d2r, ly = t->lb[P + row] * dbl_d2r;
            double rx, ry;
            if (coordsys == 1) {
                const double cb = OR_COS(ly);
                const double sb = OR_SIN(ly);
                const double cl = OR_COS(lx - GE_l0);
                const double sl = OR_SIN(lx - GE_l0);
                rx = OR_ATAN2(cb * cl, sb * GE_ce - cb * GE_se * sl) + GE_angp;
                ry = OR_ASIN(cb * GE_ce * sl + sb * GE_se);
                while (rx < 0.) rx += pi2;
                while (rx >= pi2) rx -= pi2;
            } else {
                rx = ry = -9999.;
            }
            t->radec[row] = rx / dbl_d2r;
            t->radec[P + row] = ry / dbl_d2r;
        }
    });
    return 0;
}

/* vcyl2pm on explicit inputs (for the golden-file and known-answer tests) */
void or_vcyl2pm(const gf_vel2pm_config *par, int n, const double *l_deg, const double *b_deg,
                const float *X, const float *Y, const float *Z, const float *vx, const float *vy, const float *vz,
                float *out /* [n][3] */)
{
    for (int i = 0; i < n; i++) {
        float l = 0.017453292519943295769f * (float)l_deg[i];
        float b = 0.017453292519943295769f * (float)b_deg[i];
        float px, py, pz;
        vel_cyl2xyz(px, py, pz, vx[i], vy[i], vz[i], X[i], Y[i]);
        px -= par->u0;
        py -= par->v0 + par->vLSR;
        pz -= par->w0;
        vel_xyz2lbr(px, py, pz, -px, -py, pz, l, b);
        float D = sqrtf((8000.f - X[i]) * (8000.f - X[i]) + Y[i] * Y[i] + Z[i] * Z[i]);
        px = (float)(px / (4.74 * D * 1e-3));
        py = (float)(py / (4.74 * D * 1e-3));
        if (par->coordsys == 1) transform_pm(px, py, l, b, px, py, GE_ce, GE_se, GE_l0);
        out[3 * i] = px; out[3 * i + 1] = py; out[3 * i + 2] = pz;
    }
}

double or_error_normal(uint64_t seed, uint64_t row, uint32_t band) { return error_normal(seed, row, band); }

/* elementary functions of this flavour on arrays (for the accuracy tests):
 * kind 0 expf, 1 logf, 2 log10f, 3 exp10f, 4 sinf, 5 cosf, 6 tanf, 7 powf(x, y) */
void or_math_f(int kind, int n, const float *x, const float *y, float *out)
{
    for (int i = 0; i < n; i++) {
        switch (kind) {
        case 0: out[i] = OR_EXPF(x[i]); break;
        case 1: out[i] = OR_LOGF(x[i]); break;
        case 2: out[i] = OR_LOG10F(x[i]); break;
        case 3: out[i] = OR_EXP10F(x[i]); break;
        case 4: out[i] = OR_SINF(x[i]); break;
        case 5: out[i] = OR_COSF(x[i]); break;
        case 6: out[i] = OR_TANF(x[i]); break;
        case 7: out[i] = OR_POWF(x[i], y[i]); break;
        }
    }
}
/* kind 0 exp, 1 log, 2 sin, 3 cos, 4 asin, 5 atan2(x, y) */
void or_math_d(int kind, int n, const double *x, const double *y, double *out)
{
    for (int i = 0; i < n; i++) {
        switch (kind) {
        case 0: out[i] = OR_EXP(x[i]); break;
        case 1: out[i] = OR_LOG(x[i]); break;
        case 2: out[i] = OR_SIN(x[i]); break;
        case 3: out[i] = OR_COS(x[i]); break;
        case 4: out[i] = OR_ASIN(x[i]); break;
        case 5: out[i] = OR_ATAN2(x[i], y[i]); break;
        }
    }
}

/* the crawl's bin order: diagIndexToIJ of k and advance() from it (skygen.cu.h:257-358) */
void or_diag(int k, int x, int y, int *i, int *j)
{
    int ilb = 0, kk = k;
    diagIndexToIJ(ilb, *i, *j, kk, x, y);
}
int or_advance(int *i, int *j, int x, int y)
{
    Launch L = {};
    gf_pencil_beam pix;
    int ilb = 0;
    L.npixels = 1 << 30;
    std::vector<gf_pencil_beam> dummy(2);
    L.pixels = dummy.data();
    L.npixels = 2;
    bool mv = advance(L, ilb, *i, *j, pix, x, y);
    return (mv ? 1 : 0) | (ilb ? 2 : 0);
}

}  /* extern "C" */
