/*
 * gf_host.cpp -- host setup of the catalog generator: binning, luminosity
 * functions, model frames and normalisation, stream seeding, footprint
 * pixelisation and photometric-system tables.
 */
#include "gf_host.h"
#include "gf_footprint.h"
#include "gf_math.h"
#include "gf_safeprimes.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <dlfcn.h>
#include <map>
#include <mutex>
#include <thread>
#include <limits>

namespace gfh {

/* ---------------- random number seeding ---------------- */

void MT19937::seed(uint32_t s)
{
    mt[0] = s;
    for (int i = 1; i < 624; i++) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
    mti = 624;
}

uint32_t MT19937::next()
{
    static const uint32_t mag01[2] = {0u, 0x9908b0dfu};
    if (mti >= 624) {
        int k;
        for (k = 0; k < 624 - 397; k++) {
            uint32_t y = (mt[k] & 0x80000000u) | (mt[k + 1] & 0x7fffffffu);
            mt[k] = mt[k + 397] ^ (y >> 1) ^ mag01[y & 1u];
        }
        for (; k < 623; k++) {
            uint32_t y = (mt[k] & 0x80000000u) | (mt[k + 1] & 0x7fffffffu);
            mt[k] = mt[k + (397 - 624)] ^ (y >> 1) ^ mag01[y & 1u];
        }
        uint32_t y = (mt[623] & 0x80000000u) | (mt[0] & 0x7fffffffu);
        mt[623] = mt[396] ^ (y >> 1) ^ mag01[y & 1u];
        mti = 0;
    }
    uint32_t y = mt[mti++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

void seed_streams(uint32_t seed48, int nstreams, const uint32_t *mult, uint32_t *state)
{
    Rand48 r;
    r.srand(seed48);
    for (int i = 0; i < nstreams; i++) {
        uint32_t prime = mult[i];
        state[i] = prime;
        /* (int)(drand48() * prime): x86 cvttsd2si gives INT_MIN out of range */
        double t = r.drand() * prime;
        int32_t c = (t >= 2147483648.0) ? INT32_MIN : (int32_t)t;
        state[nstreams + i] = (uint32_t)c;
        state[2 * nstreams + i] = r.lrand();
    }
}

static std::string library_dir()
{
    Dl_info info;
    if (dladdr((void *)&library_dir, &info) && info.dli_fname) {
        std::string p(info.dli_fname);
        size_t s = p.rfind('/');
        if (s != std::string::npos) return p.substr(0, s);
    }
    return ".";
}

const std::vector<uint32_t> &multipliers()
{
    static std::vector<uint32_t> tab;
    static std::once_flag once;
    std::call_once(once, [] {
        tab.resize(GF_MAX_STREAMS);
        std::string fn = library_dir() + "/safeprimes_65536.bin";
        FILE *f = fopen(fn.c_str(), "rb");
        bool ok = false;
        if (f) {
            ok = fread(tab.data(), 4, GF_MAX_STREAMS, f) == GF_MAX_STREAMS;
            fclose(f);
        }
        if (!ok) gf_safeprimes_generate(tab.data(), GF_MAX_STREAMS);
    });
    return tab;
}

/* ---------------- model setup ---------------- */

/* gsl_interp_linear evaluation with linear extrapolation (spline.cpp:59-65) */
double interp_linear(const std::vector<double> &xa, const std::vector<double> &ya, double x)
{
    int n = (int)xa.size();
    int lo = 0, hi = n - 1;
    while (hi > lo + 1) {
        int mid = (hi + lo) / 2;
        if (xa[mid] > x) hi = mid; else lo = mid;
    }
    double dx = xa[lo + 1] - xa[lo];
    if (dx > 0.0) return ya[lo] + (x - xa[lo]) / dx * (ya[lo + 1] - ya[lo]);
    return 0.0;
}

namespace {

void reset_absmag(SkyModel &m, float M0, float M1, float dM)
{
    /* os_skygen.cpp:401-407 */
    m.M0 = M0; m.M1 = M1; m.dM = dM;
    m.nM = (int)round((m.M1 - m.M0) / m.dM);
    m.M1 -= 0.5 * m.dM;
}

float rho_host(const SkyModel &m, float x, float y, float z)
{
    float vx = x + m.T[0], vy = y + m.T[1], vz = z + m.T[2];
    float wx = m.M[0] * vx + m.M[1] * vy + m.M[2] * vz;
    float wy = m.M[3] * vx + m.M[4] * vy + m.M[5] * vz;
    float wz = m.M[6] * vx + m.M[7] * vy + m.M[8] * vz;
    if (m.type == GF_MODEL_EXP_DISK) {
        float r2 = wx * wx + wy * wy;
        if (m.r_cut2 != 0.f && r2 + wz * wz > m.r_cut2) return 0.f;
        return m.f * gfm::expf_(-sqrtf(r2) / m.l - fabsf(wz) / m.h);
    }
    if (m.type == GF_MODEL_LCBULGE) {
        const float t = gfm::powf_(gfm::powf_(wx, m.n) + gfm::powf_(wy / m.ba, m.n) + gfm::powf_(wz / m.ca, m.n),
                                   (float)(1. / m.n));
        return gfm::expf_(-t / m.l);
    }
    float DSq = wx * wx + wy * wy + wz * wz;
    if (m.rmaxSq != 0.f && (DSq < m.rminSq || DSq >= m.rmaxSq)) return 0.f;
    float ty = wy / m.ba, tz = wz / m.ca;
    float rSq = wx * wx + ty * ty + tz * tz;
    int k = 0;
    while (k != m.nbreaks && rSq > m.rbreakSq[k]) k++;
    return m.f * m.fArr[k] * gfm::powf_(rSq, 0.5f * m.nArr[k]);
}

}  // namespace

bool setup_models(const gf_skygen_config &cfg, int npixels, const gf_model_config *mc, int nmodels,
                  std::vector<HostModel> &out, std::string &err)
{
    if (cfg.dm <= 0.f || !(cfg.m1 > cfg.m0) || !(cfg.M1 > cfg.M0)) { err = "invalid magnitude binning"; return false; }
    if (cfg.nthreads <= 0 || cfg.nthreads > 65536) { err = "nthreads must be in [1, 65536]"; return false; }
    SkyModel base;
    memset(&base, 0, sizeof(base));
    /* load_skyPixelizationConfig (os_skygen.cpp:409-430) */
    base.dmin = cfg.dmin;
    base.dmax = cfg.dmax;
    base.dm = cfg.dm;
    base.m1 = cfg.m1;
    reset_absmag(base, cfg.M0, cfg.M1, cfg.dm);
    base.nm = (int)round((cfg.m1 - cfg.m0) / cfg.dm);
    base.m0 = cfg.m0 + 0.5 * cfg.dm;
    base.npixels = npixels;
    base.nthreads = cfg.nthreads;
    base.norm = 1.f;

    out.clear();
    for (int i = 0; i < nmodels; i++) {
        const gf_model_config &c = mc[i];
        HostModel hm;
        SkyModel &m = hm.m;
        m = base;
        if (c.type < GF_MODEL_EXP_DISK || c.type > GF_MODEL_DENSITY_CUBE) { err = "unknown model type"; return false; }
        const bool cube = c.type == GF_MODEL_DENSITY_CUBE;
        if (c.comp < 0 || c.comp > 31) { err = "component id must be in [0, 31]"; return false; }
        m.type = c.type;
        m.comp = c.comp;
        /* frame: load_transform (transform.cpp:345-388) */
        if (c.frame == GF_FRAME_EXPLICIT) {
            for (int k = 0; k < 3; k++) m.T[k] = (float)c.T[k];
            for (int k = 0; k < 9; k++) m.M[k] = (float)c.M[k];
        } else {
            double Rg = c.Rg, z0 = c.z0;
            double sina = -z0 / Rg, cosa = sqrt(1 - sina * sina);
            /* centre of the galplane frame in galactic cartesian coordinates (transform.cpp:194-213) */
            double cx = cosa * 0.0 - sina * 0.0, cz = sina * 0.0 + cosa * 0.0;
            double ctr[3] = {Rg - cx, -0.0, cz};
            for (int k = 0; k < 3; k++) m.T[k] = (float)-ctr[k];
            double R[9] = {-cosa, 0, sina, 0, -1, 0, sina, 0, cosa};
            for (int k = 0; k < 9; k++) m.M[k] = (float)R[k];
        }
        if (cube) {
            /* densityCube::setpos: (Rg - x, -y, z) as a frame: T = (-Rg, 0, 0), M = diag(-1, -1, 1) */
            const float Rg = (float)c.Rg;
            const float T[3] = {-Rg, 0.f, 0.f}, M[9] = {-1.f, 0.f, 0.f, 0.f, -1.f, 0.f, 0.f, 0.f, 1.f};
            for (int k = 0; k < 3; k++) m.T[k] = T[k];
            for (int k = 0; k < 9; k++) m.M[k] = M[k];
            if (!c.cube) { err = "density cube without a grid"; return false; }
            size_t n = 1;
            for (int k = 0; k < 3; k++) {
                if (c.cube_n[k] < 1 || c.cube_n[k] > 65536) { err = "density cube dimensions must be in [1, 65536]"; return false; }
                n *= (size_t)c.cube_n[k];
                m.cube_n[k] = c.cube_n[k];
                m.cube_tc[k][0] = c.cube_tc[k][0];
                m.cube_tc[k][1] = c.cube_tc[k][1];
            }
            if (n > ((size_t)1 << 31)) { err = "density cube above 2^31 texels"; return false; }
            hm.cube = c.cube;
            hm.cube_size = n;
            m.nbreaks = 0;
            m.nArr[0] = 0.f;
            m.fArr[0] = 1.f;
        } else if (c.type == GF_MODEL_EXP_DISK) {
            if (!(c.l > 0) || !(c.h > 0)) { err = "exponential disk needs l > 0 and h > 0"; return false; }
            m.l = (float)c.l;
            m.h = (float)c.h;
        } else {
            m.n = (float)c.n;
            m.ba = (float)c.ba;
            m.ca = (float)c.ca;
            m.nbreaks = 0;
            m.nArr[0] = m.n;
            m.fArr[0] = 1.f;
            if (c.type == GF_MODEL_LCBULGE) {
                if (!(c.l > 0) || !(c.n != 0)) { err = "LC bulge needs l > 0 and n != 0"; return false; }
                m.l = (float)c.l;
            }
            if (c.type == GF_MODEL_BROKEN_POWER_LAW) {
                /* brokenPowerLaw::load (model_brokenPowerLaw.cpp:31-62): indices, squared break
                 * radii, and the piece-wise factors that keep the profile continuous */
                if (c.nbreaks < 0 || c.nbreaks > 9) { err = "a broken power law has 0 to 9 breaks"; return false; }
                m.nbreaks = c.nbreaks;
                for (int k = 0; k <= c.nbreaks; k++) m.nArr[k] = (float)c.n_brk[k];
                for (int k = 0; k < c.nbreaks; k++) {
                    const float rb = (float)c.rbreak[k];
                    m.rbreakSq[k] = rb * rb;
                }
                m.fArr[0] = 1.f;
                for (int k = 0; k < c.nbreaks; k++)
                    m.fArr[k + 1] = m.fArr[k] * gfm::powf_(m.rbreakSq[k], 0.5f * (m.nArr[k] - m.nArr[k + 1]));
                m.n = m.nArr[0];
            }
        }
        m.r_cut2 = 0.f;
        m.rminSq = m.rmaxSq = 0.f;
        /* luminosity function (cux.cpp:336-384) */
        if (cube && c.lf_n > 0 && c.lf_M && c.lf_phi) {
            /* load_and_resample_texture_1D: the knots' range, 1024 texels, no clipping */
            if (c.lf_n < 2) { err = "LF needs at least 2 knots"; return false; }
            const std::vector<double> X(c.lf_M, c.lf_M + c.lf_n), Y(c.lf_phi, c.lf_phi + c.lf_n);
            const int nsamp = 1024;
            const double X0 = X[0], X1 = X.back(), dX = (X1 - X0) / (nsamp - 1);
            hm.lf.resize(nsamp);
            for (int k = 0; k < nsamp; k++) hm.lf[k] = (float)interp_linear(X, Y, X0 + k * dX);
            m.lf_x0 = (float)X0;
            m.lf_inv_dx = (float)(1. / dX);
        } else if (c.lf_n <= 0 || !c.lf_M || !c.lf_phi) {
            hm.lf.assign(2, 1.f);
            m.lf_x0 = -100.f;
            m.lf_inv_dx = (float)(1. / (100. - -100.));
        } else {
            if (c.lf_n < 2) { err = "LF needs at least 2 knots"; return false; }
            std::vector<double> X, Y;
            X.push_back(-123);
            Y.push_back(0.f);
            for (int k = 0; k < c.lf_n; k++) { X.push_back(c.lf_M[k]); Y.push_back(c.lf_phi[k]); }
            double xrange = X.back() - X[1];
            X[0] = X[1] - 1e-5 * xrange;
            X.push_back(X.back() + 1e-5 * xrange);
            Y.push_back(0.f);
            const int nsamp = 1024;
            double X0 = X[0], X1 = X.back(), dX = (X1 - X0) / (nsamp - 1);
            hm.lf.resize(nsamp);
            for (int k = 0; k < nsamp; k++) hm.lf[k] = (float)interp_linear(X, Y, X0 + k * dX);
            m.lf_x0 = (float)X0;
            m.lf_inv_dx = (float)(1. / dX);
        }
        m.lf_n = (int)hm.lf.size();
        if (c.type == GF_MODEL_LCBULGE) {
            /* the LF scaled by f, no normalisation at a point (model_LCBulge.cpp:50-56) */
            const float f0 = (float)c.f;
            for (auto &v : hm.lf) v *= f0;
            m.f = 1.f;
        }
        /* normalisation at the LF sampling point (model_lib.h:68-95) */
        const double d2r = 0.01745329251994329576923691;
        float lfl = (float)c.lf_l, lfb = (float)c.lf_b, lfD = (float)c.lf_D;
        double rl = lfl * d2r, rb = lfb * d2r;
        float cl = (float)gfm::cos_d(rl), cb = (float)gfm::cos_d(rb), sl = (float)gfm::sin_d(rl), sb = (float)gfm::sin_d(rb);
        float px = lfD * cl * cb, py = lfD * sl * cb, pz = lfD * sb;
        if (cube) {
            m.f = (float)c.f;                /* a plain scale factor (densityCube::load) */
        } else if (c.type != GF_MODEL_LCBULGE) {
            m.f = 1.f;
            float norm = rho_host(m, px, py, pz);
            if (!(norm != 0.f && std::isnormal(norm))) { err = "density is zero at the LF sampling point"; return false; }
            float f0 = (float)c.f;
            m.f = f0 / norm;
        }
        if (c.type == GF_MODEL_EXP_DISK) {
            float rc = (float)c.rcut;
            m.r_cut2 = rc * rc;
        } else if (c.type != GF_MODEL_LCBULGE && !cube) {
            float rmin = (float)c.rmin, rmax = (float)c.rmax;
            m.rminSq = rmin * rmin;
            m.rmaxSq = rmax * rmax;
        }
        /* absolute magnitude hint from the LF range (skyconfig_impl.h:257-263, model_lib.h:97-112) */
        float hM0 = m.M0, hM1 = m.M1 + 0.5 * m.dM;
        float X0 = m.lf_x0;
        float X1 = double(m.lf_n - 1) / m.lf_inv_dx + X0;
        bool hint = false;
        if (X0 > hM0) { hint = true; hM0 = X0; }
        if (X1 < hM1) { hint = true; hM1 = X1; }
        if (hint) reset_absmag(m, hM0, hM1, m.dM);
        if (m.nm <= 0 || m.nM <= 0) { err = "empty magnitude grid"; return false; }
        if ((long long)m.nm * m.nM > 0x3fffffff) { err = "magnitude grid too large"; return false; }
        if (m.nm > 32767 || m.nM > 32767) { err = "magnitude grid dimension above 32767"; return false; }
        m.lf = nullptr;
        m.cube = nullptr;                  /* the device copy is attached by the caller */
        out.push_back(hm);
    }
    return true;
}

}  // namespace gfh

/* ------------------------------------------------------------------ */
/* Host-only C entry points                                            */
/* ------------------------------------------------------------------ */
extern "C" {

uint32_t gf_rng_seed48_from_cli_seed(uint64_t seed)
{
    /* rng_gsl_t(seed) with gsl_rng_default = mt19937 (gpu.h:362-382), then
     * (uint32_t)(seeder.uniform() * (1 << 24)) (cux.cpp:409) */
    gfh::MT19937 mt;
    uint32_t s = (uint32_t)seed;
    if (s == 0) s = 4357;       /* GSL's mt19937 treats seed 0 as 4357 */
    mt.seed(s);
    double u = mt.next() / 4294967296.0;
    float fu = (float)u;
    return (uint32_t)(fu * (float)(1 << 24));
}

void gf_mt19937_outputs(uint32_t seed, int n, uint32_t *out)
{
    gfh::MT19937 mt;
    mt.seed(seed);
    for (int i = 0; i < n; i++) out[i] = mt.next();
}

void gf_rng_seed_host(uint32_t seed48, int32_t nstreams, uint32_t *state)
{
    gfh::seed_streams(seed48, nstreams, gfh::multipliers().data(), state);
}

/* Host-only model setup (binning, LF resampling, frames, normalisation): the
 * derived parameters and LF of each model, as gf_skygen_create computes them. */
gf_status gf_skygen_setup_host(const gf_skygen_config *cfg, int32_t npixels, const gf_model_config *models, int32_t nmodels,
                               gf_skygen_model_info *info, float *lf /* [nmodels][1024] or NULL */)
{
    std::vector<gfh::HostModel> hms;
    std::string err;
    if (!cfg || !models || nmodels <= 0 || !info) return GF_E_INVALID;
    if (!gfh::setup_models(*cfg, npixels, models, nmodels, hms, err)) return GF_E_INVALID;
    for (int i = 0; i < nmodels; i++) {
        const SkyModel &m = hms[i].m;
        gf_skygen_model_info &o = info[i];
        o.m0 = m.m0; o.m1 = m.m1; o.dm = m.dm; o.M0 = m.M0; o.M1 = m.M1; o.dM = m.dM;
        o.nm = m.nm; o.nM = m.nM; o.npixels = m.npixels; o.nthreads = m.nthreads;
        o.f = m.f; o.lf_x0 = m.lf_x0; o.lf_inv_dx = m.lf_inv_dx; o.lf_n = m.lf_n; o.norm = m.norm;
        if (lf) std::copy(hms[i].lf.begin(), hms[i].lf.end(), lf + (size_t)i * 1024);
    }
    return GF_OK;
}

int gf_multipliers(uint32_t *out, int32_t n)
{
    if (n < 0 || n > GF_MAX_STREAMS) return GF_E_INVALID;
    const std::vector<uint32_t> &m = gfh::multipliers();
    std::copy(m.begin(), m.begin() + n, out);
    return GF_OK;
}

}  /* extern "C" */

/* ------------------------------------------------------------------ */
/* Footprint pixelisation (host setup; the reference builds its pixel  */
/* list from GPC polygons, os_skygen.cpp:130-283 -- here footprints    */
/* are analytic and coverage is measured by supersampling).            */
/* ------------------------------------------------------------------ */
namespace {

const double kD2R = 0.01745329251994329576923691;

/* lambert deprojection in double precision (skygen.h:131-146 with double x, y) */
void deproject_d(const gf_lambert &p, double x, double y, double &l, double &b)
{
    double r2 = x * x + y * y;
    if (r2 == 0.) { b = p.b0; l = 0.; return; }
    double ir = 1. / sqrt(r2);
    double sc = 1. / ir * sqrt(1. - 0.25 * r2);
    double cc = 1. - 0.5 * r2;
    b = gfm::asin_d(cc * (double)p.sb + y * sc * (double)p.cb * ir);
    l = p.l0 + gfm::atan2_d(x * sc, (double)p.cb * cc / ir - y * (double)p.sb * sc);
}

/* galactic longitude/latitude rectangle, degrees; l in any turn */
static bool lb_rect_inside(const gf_footprint &f, double l, double b)
{
    if (!(b >= f.c && b < f.d)) return false;
    l = fmod(l, 360.0);
    if (l < 0) l += 360.0;
    return (f.a <= f.b) ? (l >= f.a && l < f.b) : (l >= f.a || l < f.b);
}

struct FootTest {
    gf_footprint f;
    double cb0, sb0, l0, cosr;
    explicit FootTest(const gf_footprint &ff) : f(ff)
    {
        l0 = f.a * kD2R;
        cb0 = gfm::cos_d(f.b * kD2R);
        sb0 = gfm::sin_d(f.b * kD2R);
        cosr = gfm::cos_d(f.c * kD2R);
    }
    /* is the point (l, b) (radians), seen in projection `proj` at (x, y), inside? */
    bool inside(int proj, double x, double y, double l, double b) const
    {
        switch (f.kind) {
        case GF_FOOT_ALL: return true;
        case GF_FOOT_LAMBERT_RECT: return proj == f.proj && x >= f.a && x < f.b && y >= f.c && y < f.d;
        case GF_FOOT_CAP: return gfm::sin_d(b) * sb0 + gfm::cos_d(b) * cb0 * gfm::cos_d(l - l0) >= cosr;
        case GF_FOOT_LATCUT: return fabs(b) > f.a * kD2R;
        case GF_FOOT_LB_RECT: return lb_rect_inside(f, l / kD2R, b / kD2R);
        case GF_FOOT_REGIONS: return gff::regions_inside(f, l / kD2R, b / kD2R);
        }
        return false;
    }
};

/* galactic samples (radians) of the boundaries of a region set, for its bounding boxes */
template <class F>
static void region_boundaries(const gf_footprint &f, F &&add)
{
    auto put = [&](const gf_region &r, double lon, double lat) {
        if (r.coordsys == GF_COORD_EQU) gff::equ_to_gal(lon, lat, lon, lat);
        add(lon, lat);
    };
    for (int q = 0; q < f.nregions && q < GF_MAX_REGIONS; q++) {
        const gf_region &r = f.regions[q];
        if (r.type == GF_REGION_BEAM) {
            /* small circles about the centre c: cos(r) c + sin(r) (cos(az) u + sin(az) v)
             * with u, v orthonormal tangents (well defined at the poles too) */
            const double lc = r.a * kD2R, bc = r.b * kD2R;
            const double c[3] = {gfm::cos_d(bc) * gfm::cos_d(lc), gfm::cos_d(bc) * gfm::sin_d(lc), gfm::sin_d(bc)};
            const double u[3] = {-gfm::sin_d(lc), gfm::cos_d(lc), 0.0};
            const double v[3] = {c[1] * u[2] - c[2] * u[1], c[2] * u[0] - c[0] * u[2], c[0] * u[1] - c[1] * u[0]};
            const double radii[2] = {std::min(r.c, 180.0) * kD2R, r.d * kD2R};
            for (int h = 0; h < 2; h++) {
                const double rr = radii[h];
                if (h == 1 && !(r.d > 0)) break;
                for (int k = 0; k <= 4096; k++) {
                    const double az = 2 * M_PI * k / 4096.0, r0 = (k == 4096) ? 0.0 : rr;
                    double p[3];
                    for (int i = 0; i < 3; i++)
                        p[i] = gfm::cos_d(r0) * c[i] + gfm::sin_d(r0) * (gfm::cos_d(az) * u[i] + gfm::sin_d(az) * v[i]);
                    const double b = gfm::asin_d(std::max(-1.0, std::min(1.0, p[2])));
                    const double l = gfm::atan2_d(p[1], p[0]);
                    put(r, l, b);
                }
            }
        } else if (r.type == GF_REGION_RECT) {
            double l0 = r.a, l1 = r.b;
            if (l1 <= l0) l1 += 360.0;
            const double b0 = std::max(r.c, -90.0), b1 = std::min(r.d, 90.0);
            for (int k = 0; k <= 2048; k++) {
                const double t = k / 2048.0;
                const double l = (l0 + t * (l1 - l0)) * kD2R, b = (b0 + t * (b1 - b0)) * kD2R;
                put(r, l, b0 * kD2R);
                put(r, l, b1 * kD2R);
                put(r, l0 * kD2R, b);
                put(r, l1 * kD2R, b);
                put(r, 0.5 * (l0 + l1) * kD2R, b);
            }
        }
    }
}

/* does the region set hold a region smaller than s degrees across? */
static bool regions_small(const gf_footprint &f, double s)
{
    for (int q = 0; q < f.nregions && q < GF_MAX_REGIONS; q++) {
        const gf_region &r = f.regions[q];
        if (r.type == GF_REGION_BEAM && (r.c < s || (r.d > 0 && r.c - r.d < s))) return true;
        if (r.type == GF_REGION_RECT && (r.d - r.c < s || (r.a != r.b && fabs(fmod(r.b - r.a + 360.0, 360.0)) < s))) return true;
    }
    return false;
}

}  // namespace

extern "C" {

gf_status gf_lambert_init(double l0_deg, double b0_deg, gf_lambert *p)
{
    /* lambert::init (skygen.h:115-120) */
    p->l0 = l0_deg * kD2R;
    p->b0 = b0_deg * kD2R;
    p->cl = (float)gfm::cos_d(p->l0);
    p->cb = (float)gfm::cos_d(p->b0);
    p->sl = (float)gfm::sin_d(p->l0);
    p->sb = (float)gfm::sin_d(p->b0);
    return GF_OK;
}

/* Pixelise a footprint on the Lambert grids of the two hemispheres (cell side
 * dx_deg in degrees of Lambert coordinate, grid anchored at the pole).  A point
 * belongs to the north grid when b >= 0 and to the south grid otherwise.
 * beam_ammin (nullable) receives the minimum screen extinction over each cell.
 * Call with pixels == NULL to count. */
gf_status gf_footprint_pixelize(const gf_footprint *foot, double dx_deg, const gf_lambert proj[2],
                                const gf_extinction *ext, gf_pencil_beam *pixels, float *beam_ammin,
                                int64_t max_pixels, int64_t *npixels)
{
    if (!foot || !npixels || !(dx_deg > 0)) return GF_E_INVALID;
    if (foot->kind == GF_FOOT_REGIONS) {
        if (foot->nregions < 1 || foot->nregions > GF_MAX_REGIONS) return GF_E_INVALID;
        for (int q = 0; q < foot->nregions; q++) {
            const gf_region &r = foot->regions[q];
            if ((r.type != GF_REGION_BEAM && r.type != GF_REGION_RECT) || (r.coordsys != GF_COORD_GAL && r.coordsys != GF_COORD_EQU))
                return GF_E_INVALID;
        }
    }
    const double dx = dx_deg * kD2R;
    const float dxf = (float)dx;
    FootTest ft(*foot);
    const int SS = 16;                       /* supersampling per axis at the boundary */
    int64_t n = 0;
    for (int h = 0; h < 2; h++) {
        /* bounding box of the footprint in this hemisphere's Lambert plane */
        double xmin = -M_SQRT2, xmax = M_SQRT2, ymin = -M_SQRT2, ymax = M_SQRT2;
        if (foot->kind == GF_FOOT_LAMBERT_RECT) {
            if (foot->proj != h) continue;
            xmin = foot->a; xmax = foot->b; ymin = foot->c; ymax = foot->d;
        } else if (foot->kind == GF_FOOT_LATCUT) {
            double R = 2 * gfm::sin_d(0.5 * (90. - foot->a) * kD2R);
            xmin = ymin = -R; xmax = ymax = R;
        } else if (foot->kind == GF_FOOT_CAP || foot->kind == GF_FOOT_LB_RECT || foot->kind == GF_FOOT_REGIONS) {
            /* project boundary samples of the footprint that fall in this hemisphere */
            double bx0 = 1e9, bx1 = -1e9, by0 = 1e9, by1 = -1e9;
            bool any = false;
            const gf_lambert &p = proj[h];
            auto add_point = [&](double l, double b) {
                if ((h == 0) != (b >= 0)) return;
                /* forward Lambert projection about the pole */
                double cll0 = gfm::cos_d(l - p.l0);
                double sll0 = gfm::sin_d(l - p.l0);
                double kp = 1.414213562373095 * sqrt(1. / (1. + (double)p.sb * gfm::sin_d(b) + (double)p.cb * gfm::cos_d(b) * cll0));
                double x = kp * gfm::cos_d(b) * sll0;
                double y = kp * ((double)p.cb * gfm::sin_d(b) - (double)p.sb * gfm::cos_d(b) * cll0);
                bx0 = std::min(bx0, x); bx1 = std::max(bx1, x); by0 = std::min(by0, y); by1 = std::max(by1, y);
                any = true;
            };
            if (foot->kind == GF_FOOT_REGIONS) {
                region_boundaries(*foot, add_point);
            } else if (foot->kind == GF_FOOT_CAP) {
                double lc = foot->a * kD2R, bc = foot->b * kD2R, r = foot->c * kD2R;
                for (int k = 0; k <= 4096; k++) {
                    double rr = (k == 4096) ? 0.0 : r;
                    double az = 2 * M_PI * k / 4096.0;
                    /* destination point at distance rr, azimuth az from (lc, bc) */
                    double sb = gfm::sin_d(bc) * gfm::cos_d(rr) + gfm::cos_d(bc) * gfm::sin_d(rr) * gfm::cos_d(az);
                    double b = gfm::asin_d(sb);
                    double l = lc + gfm::atan2_d(gfm::sin_d(az) * gfm::sin_d(rr) * gfm::cos_d(bc), gfm::cos_d(rr) - gfm::sin_d(bc) * sb);
                    add_point(l, b);
                }
            } else {
                double l0 = foot->a, l1 = foot->b < foot->a ? foot->b + 360.0 : foot->b;
                double b0 = std::max(foot->c, -90.0), b1 = std::min(foot->d, 90.0);
                for (int k = 0; k <= 2048; k++) {
                    double t = k / 2048.0;
                    double l = (l0 + t * (l1 - l0)) * kD2R, b = (b0 + t * (b1 - b0)) * kD2R;
                    add_point(l, b0 * kD2R);
                    add_point(l, b1 * kD2R);
                    add_point(l0 * kD2R, b);
                    add_point(l1 * kD2R, b);
                    add_point(0.5 * (l0 + l1) * kD2R, b);
                }
            }
            /* a footprint that reaches the equator is also bounded by the rim: its inside points at b = 0 */
            for (int k = 0; k < 8192; k++) {
                const double l = 2 * M_PI * k / 8192.0, b = (h == 0) ? 0.0 : -1e-12;
                if (ft.inside(h, 0.0, 0.0, l, b)) add_point(l, b);
            }
            if (!any) continue;
            double pad = 2 * dx;
            xmin = std::max(-M_SQRT2, bx0 - pad); xmax = std::min(M_SQRT2, bx1 + pad);
            ymin = std::max(-M_SQRT2, by0 - pad); ymax = std::min(M_SQRT2, by1 + pad);
            /* a footprint containing the pole covers the origin */
            bool pole = (foot->kind == GF_FOOT_REGIONS) ? ft.inside(h, 0.0, 0.0, 0.0, (h == 0 ? 0.5 : -0.5) * M_PI)
                        : (foot->kind == GF_FOOT_CAP) ? ((h == 0 ? 90. - foot->b : 90. + foot->b) <= foot->c)
                                                      : (h == 0 ? foot->d >= 90. : foot->c <= -90.);
            if (pole) { xmin = std::min(xmin, -dx); xmax = std::max(xmax, dx); ymin = std::min(ymin, -dx); ymax = std::max(ymax, dx); }
        }
        long long i0 = (long long)floor(xmin / dx), i1 = (long long)ceil(xmax / dx);
        long long j0 = (long long)floor(ymin / dx), j1 = (long long)ceil(ymax / dx);
        for (long long i = i0; i < i1; i++) {
            for (long long j = j0; j < j1; j++) {
                double cx0 = i * dx, cy0 = j * dx;
                /* reject cells entirely outside the Lambert disk of the hemisphere */
                double nx = std::max(cx0, std::min(0.0, cx0 + dx)), ny = std::max(cy0, std::min(0.0, cy0 + dx));
                double rmin2 = nx * nx + ny * ny;
                if (rmin2 > 2.0) continue;
                /* coverage: corners + centre decide interior and exterior cells; mixed
                 * cells (and cells that could hold a footprint smaller than a cell) are
                 * supersampled */
                auto in_point = [&](double px, double py) -> bool {
                    double r2 = px * px + py * py;
                    if (r2 > 2.0) return false;
                    if (foot->kind == GF_FOOT_LATCUT) {
                        /* pole projections: sin|b| = 1 - r^2/2 */
                        return 1.0 - 0.5 * r2 > gfm::sin_d(foot->a * kD2R);
                    }
                    if (foot->kind == GF_FOOT_LAMBERT_RECT) return ft.inside(h, px, py, 0, 0);
                    double l, b;
                    deproject_d(proj[h], px, py, l, b);
                    bool hemi = (h == 0) ? (b >= 0) : (b < 0);
                    return hemi && ft.inside(h, px, py, l, b);
                };
                int in_corners = 0;
                for (int c = 0; c < 5; c++) {
                    double px = (c == 4) ? cx0 + 0.5 * dx : cx0 + (c & 1) * dx;
                    double py = (c == 4) ? cy0 + 0.5 * dx : cy0 + ((c >> 1) & 1) * dx;
                    if (in_point(px, py)) in_corners++;
                }
                bool tiny = (foot->kind == GF_FOOT_CAP && foot->c * kD2R < 3 * dx) ||
                            (foot->kind == GF_FOOT_REGIONS && regions_small(*foot, 3 * dx / kD2R));
                double cov;
                if (foot->kind == GF_FOOT_LAMBERT_RECT) {
                    /* exact overlap of two rectangles */
                    double ox = std::max(0.0, std::min(cx0 + dx, foot->b) - std::max(cx0, foot->a));
                    double oy = std::max(0.0, std::min(cy0 + dx, foot->d) - std::max(cy0, foot->c));
                    cov = ox * oy / (dx * dx);
                    if (cx0 * cx0 + cy0 * cy0 > 2.0 && in_corners == 0) cov = 0.0;
                } else if (in_corners == 5 && !tiny) {
                    cov = 1.0;
                } else if (in_corners == 0 && !tiny) {
                    cov = 0.0;
                } else {
                    int cnt = 0;
                    for (int a = 0; a < SS; a++)
                        for (int bq = 0; bq < SS; bq++)
                            if (in_point(cx0 + (a + 0.5) * dx / SS, cy0 + (bq + 0.5) * dx / SS)) cnt++;
                    cov = (double)cnt / (SS * SS);
                }
                if (cov <= 0.0) continue;
                if (pixels && n < max_pixels) {
                    double X = cx0 + 0.5 * dx, Y = cy0 + 0.5 * dx;
                    double l, b;
                    deproject_d(proj[h], X, Y, l, b);
                    gf_pencil_beam &pb = pixels[n];
                    memset(&pb, 0, sizeof(pb));
                    pb.cl = (float)gfm::cos_d(l); pb.cb = (float)gfm::cos_d(b);
                    pb.sl = (float)gfm::sin_d(l); pb.sb = (float)gfm::sin_d(b);
                    pb.coveredFraction = (float)cov;
                    pb.dx = dxf;
                    pb.dA = dxf * dxf;
                    pb.projIdx = h;
                    pb.X = (float)X;
                    pb.Y = (float)Y;
                    pb.extIdx = (int32_t)n;
                    if (beam_ammin) {
                        float am = 0.f;
                        if (ext && ext->kind == GF_EXT_SCREEN_CSCB) {
                            double sbmax = 1.0 - 0.5 * rmin2;          /* sin|b| at the cell point nearest the pole */
                            am = (float)(ext->A0 / sbmax * (1.0 - 1e-6));
                        }
                        beam_ammin[n] = am;
                    }
                }
                n++;
            }
        }
    }
    *npixels = n;
    return (pixels && n > max_pixels) ? GF_E_INVALID : GF_OK;
}

/* Resample a photometric system table (rows Mr, FeH, c_1..c_ncolors) to the
 * colour/extrapolation-flag grids of os_photometry::construct
 * (photometry_host.cpp:233-344).  Call with colors == NULL to get the sizes. */
gf_status gf_photometry_build(const double *rows, int32_t nrows, int32_t ncolors, double dFeH, double dMr,
                              float *colors, uint8_t *eflags, int32_t *nFeH_out, int32_t *nMr_out,
                              float tcFeH[2], float tcMr[2])
{
    if (!rows || nrows < 1 || ncolors < 1 || ncolors >= GF_MAX_BANDS || !(dFeH > 0) || !(dMr > 0)) return GF_E_INVALID;
    const int w = 2 + ncolors;
    std::map<double, std::vector<const double *>> v;
    for (int r = 0; r < nrows; r++) v[rows[(size_t)r * w + 1]].push_back(rows + (size_t)r * w);
    double FeH0 = v.begin()->first, FeH1 = v.rbegin()->first;
    double Mr0 = rows[0], Mr1 = rows[0];
    for (int r = 0; r < nrows; r++) { Mr0 = std::min(Mr0, rows[(size_t)r * w]); Mr1 = std::max(Mr1, rows[(size_t)r * w]); }
    int nFeH = (int)((FeH1 - FeH0) / dFeH + 1);
    int nMr = (int)((Mr1 - Mr0) / dMr + 1);
    /* texcoord_from_range(0, n, x0, x0 + n*dx) in float (cux.cpp:389-397) */
    auto tc_range = [](float imgx, float imgy, float x, float y, float out[2]) {
        out[0] = (-imgy * x + imgx * y) / (imgx - imgy);
        out[1] = (imgx - imgy) / (x - y);
    };
    tc_range(0, (float)nFeH, (float)FeH0, (float)(FeH0 + nFeH * dFeH), tcFeH);
    tc_range(0, (float)nMr, (float)Mr0, (float)(Mr0 + nMr * dMr), tcMr);
    *nFeH_out = nFeH;
    *nMr_out = nMr;
    if (!colors) return GF_OK;
    /* per-FeH colour(Mr) knots, sorted by Mr */
    struct Line { double FeH; std::vector<double> Mr; std::vector<std::vector<double>> c; double Mrmin, Mrmax; };
    std::vector<Line> lines;
    std::vector<double> vFeH;
    for (auto &kv : v) {
        Line L;
        L.FeH = kv.first;
        std::vector<const double *> rs = kv.second;
        std::stable_sort(rs.begin(), rs.end(), [](const double *a, const double *b) { return a[0] < b[0]; });
        L.c.resize(ncolors);
        for (const double *r : rs) {
            L.Mr.push_back(r[0]);
            for (int ic = 0; ic < ncolors; ic++) L.c[ic].push_back(r[2 + ic]);
        }
        L.Mrmin = L.Mr.front();
        L.Mrmax = L.Mr.back();
        lines.push_back(L);
        vFeH.push_back(L.FeH);
    }
    std::vector<double> vcol(lines.size()), vecol(lines.size());
    for (int ic = 0; ic < ncolors; ic++) {
        for (int m = 0; m < nMr; m++) {
            double Mr = Mr0 + m * dMr;
            for (size_t k = 0; k < lines.size(); k++) {
                const Line &L = lines[k];
                vcol[k] = L.Mr.size() > 1 ? gfh::interp_linear(L.Mr, L.c[ic], Mr) : L.c[ic][0];
                vecol[k] = (L.Mrmin > Mr || Mr > L.Mrmax) ? 1.0 : 0.0;
            }
            for (int f = 0; f < nFeH; f++) {
                double FeH = FeH0 + f * dFeH;
                float color = (float)(lines.size() > 1 ? gfh::interp_linear(vFeH, vcol, FeH) : vcol[0]);
                double ef = lines.size() > 1 ? gfh::interp_linear(vFeH, vecol, FeH) : vecol[0];
                bool eflag = vFeH.front() > FeH || FeH > vFeH.back() || ef != 0.;
                size_t off = ((size_t)ic * nMr + m) * nFeH + f;
                colors[off] = color;
                eflags[off] = eflag ? 1 : 0;
            }
        }
    }
    return GF_OK;
}

/* os_unresolvedMultiples::construct (unresolvedMultiples_host.cpp:96-189): the
 * binary-fraction table (resampled to 64 texels, or the constant 1 over
 * [-100, 100]), and the cumulative luminosity function of the secondaries (the
 * trapezoid integral of the linearly interpolated LF at 256 points, normalised)
 * with its inverse, both resampled to 256 texels (cux.cpp:310-350). */
static void resample_1d(const std::vector<double> &X, const std::vector<double> &Y, int nsamp, float *tab, float *x0,
                        float *inv_dx)
{
    const double X0 = X[0], X1 = X.back(), dX = (X1 - X0) / (nsamp - 1);
    for (int i = 0; i != nsamp; i++) tab[i] = (float)gfh::interp_linear(X, Y, X0 + i * dX);
    *x0 = (float)X0;
    *inv_dx = (float)(1. / dX);
}

gf_status gf_multiples_build(const double *frac_M, const double *frac_p, int32_t nfrac, const double *lf_M,
                             const double *lf_phi, int32_t nlf, int32_t algo, uint32_t comp_mask, gf_multiples_config *out)
{
    if (!out || algo < GF_MULT_LF_M2_GT_M1 || algo > GF_MULT_EQUAL_MASS || nfrac < 0 || nlf < 0 || nfrac == 1 || nlf == 1 ||
        (nfrac && (!frac_M || !frac_p)) || (nlf && (!lf_M || !lf_phi)))
        return GF_E_INVALID;
    for (int i = 1; i < nfrac; i++)
        if (!(frac_M[i] > frac_M[i - 1])) return GF_E_INVALID;
    for (int i = 1; i < nlf; i++)
        if (!(lf_M[i] > lf_M[i - 1])) return GF_E_INVALID;
    memset(out, 0, sizeof(*out));
    out->algo = algo;
    out->comp_mask = comp_mask;
    if (nfrac) {
        const std::vector<double> X(frac_M, frac_M + nfrac), Y(frac_p, frac_p + nfrac);
        out->nsec = 64;
        resample_1d(X, Y, 64, out->secprob, &out->sec_x0, &out->sec_inv_dx);
    } else {
        /* load_constant_texture_1D(1, -100, 100) */
        out->nsec = 2;
        out->secprob[0] = out->secprob[1] = 1.f;
        out->sec_x0 = -100.f;
        out->sec_inv_dx = (float)(1. / (100. - -100.));
    }
    std::vector<double> x, y;
    if (nlf) {
        x.assign(lf_M, lf_M + nlf);
        y.assign(lf_phi, lf_phi + nlf);
    } else {
        x = {-100., 100.};
        y = {1., 1.};
    }
    const int NPIX = GF_MULT_TEX;
    const double dx = (x.back() - x.front()) / (NPIX - 1);
    std::vector<double> ycum(NPIX), xcum(NPIX);
    xcum[0] = x.front();
    ycum[0] = 0;
    double yprev = gfh::interp_linear(x, y, x.front());
    for (int i = 1; i < NPIX; i++) {
        const double xx = x.front() + i * dx;
        const double yy = gfh::interp_linear(x, y, xx);
        const double dy = yy - yprev;
        const double dA = (yprev + 0.5 * dy) * dx;
        xcum[i] = xx;
        ycum[i] = ycum[i - 1] + dA;
        yprev = yy;
    }
    const double norm = ycum.back();
    if (!(norm > 0)) return GF_E_INVALID;
    for (auto &v : ycum) v /= norm;
    for (int i = 1; i < NPIX; i++)
        if (!(ycum[i] > ycum[i - 1])) return GF_E_INVALID;     /* the inverse needs a strictly increasing integral */
    out->ncum = out->ninv = NPIX;
    resample_1d(xcum, ycum, NPIX, out->cumlf, &out->cum_x0, &out->cum_inv_dx);
    resample_1d(ycum, xcum, NPIX, out->invcumlf, &out->inv_x0, &out->inv_inv_dx);
    return GF_OK;
}

/* lambert::project (skygen.h:123-130): float direction and pole, double intermediates */
static void lambert_project(const gf_lambert &p, const gf_pencil_beam &d, float &x, float &y)
{
    const double cll0 = d.cl * p.cl + d.sl * p.sl;
    const double sll0 = p.cl * d.sl - d.cl * p.sl;
    const double kp = 1.414213562373095 * sqrt(1. / (1. + p.sb * d.sb + p.cb * d.cb * cll0));
    x = (float)(kp * d.cb * sll0);
    y = (float)(kp * (p.cb * d.sb - p.sb * d.cb * cll0));
}

gf_status gf_extinction_beam_minima(const gf_extinction *ext, const gf_lambert proj[2], const gf_pencil_beam *pixels,
                                    int32_t npixels, float *out, int32_t *nz_out)
{
    if (!ext || ext->kind != GF_EXT_MAPS || !proj || npixels < 0 || (npixels && !pixels)) return GF_E_INVALID;
    const gf_ext_map *mp[2] = {ext->north, ext->south};
    int nz = 0;
    for (int h = 0; h < 2; h++) {
        if (!mp[h]) continue;
        if (!mp[h]->A || mp[h]->n[0] < 1 || mp[h]->n[1] < 1 || mp[h]->n[2] < 1) return GF_E_INVALID;
        if (nz && mp[h]->n[2] != nz) return GF_E_INVALID;
        nz = mp[h]->n[2];
    }
    if (nz == 0) nz = 1;                                  /* no map: zero extinction */
    if (nz_out) *nz_out = nz;
    if (!out) return GF_OK;
    for (int32_t i = 0; i < npixels; i++)
        if (pixels[i].extIdx < 0 || pixels[i].extIdx >= npixels) return GF_E_INVALID;
    const bool any = mp[0] || mp[1];
    for (size_t q = 0; q < (size_t)npixels * nz; q++) out[q] = any ? std::numeric_limits<float>::infinity() : 0.f;
    /* find_extinction_minima (os_skygen.cpp:285-342) for every beam and given map */
    std::vector<std::thread> th;
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (int w = 0; w < nt; w++) {
        th.emplace_back([&, w] {
            for (int32_t i = w; i < npixels; i += nt) {
                const gf_pencil_beam &p = pixels[i];
                float *row = out + (size_t)p.extIdx * nz;
                for (int h = 0; h < 2; h++) {
                    if (!mp[h]) continue;
                    const gf_ext_map &e = *mp[h];
                    const int width = e.n[0], height = e.n[1], depth = e.n[2];
                    auto tex = [&](int x, int y, int z) { return e.A[((size_t)z * height + y) * width + x]; };
                    float x, y;
                    lambert_project(proj[h], p, x, y);
                    const float tcxx = e.tc[0][0], tcxy = e.tc[0][1], tcyx = e.tc[1][0], tcyy = e.tc[1][1];
                    const double dr = 1.0001 / 2. * sqrt(2) * (p.dx + std::max(1. / tcxy, 1. / tcyy));
                    int xi = (int)((x - dr - tcxx) * tcxy);  xi = std::max(0, std::min(xi - 1, width));
                    int yi = (int)((y - dr - tcyx) * tcyy);  yi = std::max(0, std::min(yi - 1, height));
                    int xie = (int)((x + dr - tcxx) * tcxy); xie = std::max(0, std::min(xie + 2, width));
                    int yie = (int)((y + dr - tcyx) * tcyy); yie = std::max(0, std::min(yie + 2, height));
                    for (int X = xi; X != xie; X++) {
                        if (X < 0 || X >= width) continue;
                        for (int Y = yi; Y != yie; Y++) {
                            if (Y < 0 || Y >= width) continue;       /* the reference compares y with the width */
                            if (Y >= height) continue;               /* (and never reads past the map) */
                            /* texels outside the hemisphere's disk hold zero: skip them */
                            const double Amax = tex(X, Y, depth - 1);
                            if (Amax == 0) {
                                const double xx = ((double)X) / tcxy + tcxx;
                                const double yy = ((double)Y) / tcyy + tcyx;
                                if (xx * xx + yy * yy > 2) continue;
                            }
                            for (int z = 0; z < depth; z++) {
                                const float Ar = z - 1 < 0 ? 0.f : tex(X, Y, z - 1);
                                row[z] = std::min(row[z], Ar);
                            }
                        }
                    }
                }
            }
        });
    }
    for (auto &t : th) t.join();
    return GF_OK;
}

}  /* extern "C" */
