/*
 * galfast_b200.h -- C ABI of the B200-native galfast catalog-generation hot path.
 *
 * The library replaces the compute behind galfast's skygen source module and
 * the postprocessing modules that follow it on the catalog path:
 *
 *   reference interface (mjuric/galfast)                      entry point here
 *   ------------------------------------------------------    ------------------------------
 *   skygenInterface::init / initRNG (src/skygen/skygen.h:47-60,
 *     src/skygen/skyconfig_impl.h:244-305, src/common/cux.cpp:404-435)
 *                                                             gf_rng_init, gf_skygen_create
 *   skygenInterface::integrateCounts (skyconfig_impl.h:323-429)
 *                                                             gf_skygen_integrate
 *   skygenInterface::setDensityNorm (skyconfig_impl.h:308-320) gf_skygen_set_norm
 *   skygenInterface::drawSources, one output batch per call
 *     (skyconfig_impl.h:435-545, kernel skygen.cu.h:469-618)  gf_skygen_draw
 *   osink::process of the modules (src/pipeline.h:98-110) and their kernels
 *     fixedFeH (src/modules/fixedFeH_host.cpp:49-70)          gf_module_fixedfeh
 *     Bond2010 (src/modules/Bond2010_host.cpp:70-90)          gf_module_bond2010
 *     photometry (src/modules/photometry_host.cpp:363-395)    gf_module_photometry
 *     photometricErrors (photometricErrors_host.cpp:112-131)  gf_module_photoerrors
 *     vel2pm (src/modules/vel2pm_host.cpp:58-74)              gf_module_vel2pm
 *     gal2other (src/modules/gal2other_host.cpp)              gf_module_gal2other
 *     clipper (src/skygen/os_skygen.cpp:999-1044)             gf_module_clipper
 *   os_skygen::run + drawSources + the module chain
 *     (os_skygen.cpp:866-932, pipeline.cpp:1143-1227)         gf_catalog_run
 *
 * All pointers are plain host or device pointers, all sizes are element
 * counts, and every entry point returns a gf_status; gf_last_error() returns
 * a description of the last failure on the calling thread.  A gf_ctx owns one
 * CUDA stream on one device and is used by one host thread at a time.
 */
#ifndef GALFAST_B200_H
#define GALFAST_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GF_ABI_VERSION 1

typedef enum {
    GF_OK = 0,
    GF_E_INVALID = -1,      /* bad argument or configuration */
    GF_E_OOM = -2,          /* device or host allocation failed */
    GF_E_CUDA = -3,         /* CUDA runtime error */
    GF_E_TIMEOUT = -4,      /* a bounded device wait gave up */
    GF_E_UNSUPPORTED = -5,  /* configuration outside what this build implements */
    GF_E_STATE = -6         /* call out of sequence */
} gf_status;

/* ------------------------------------------------------------------ */
/* Geometry (layouts mirror the reference's device structs)            */
/* ------------------------------------------------------------------ */

/* A pencil beam (sky pixel); mirrors struct pencilBeam, src/skygen/skygen.h:89-103. */
typedef struct gf_pencil_beam {
    float cl, cb, sl, sb;      /* cos/sin of the pixel centre (l, b) */
    float coveredFraction;     /* fraction of the pixel inside the footprint */
    float dx, dA;              /* side (radians, Lambert units) and area dx*dx */
    int32_t projIdx;           /* 0 = north, 1 = south Lambert projection */
    float X, Y;                /* Lambert coordinates of the centre */
    int32_t extIdx;            /* row of the per-beam minimum-extinction table */
    int32_t pad_;
} gf_pencil_beam;

/* Lambert azimuthal equal-area projection; mirrors class lambert, skygen.h:108-147. */
typedef struct gf_lambert {
    double l0, b0;             /* pole (radians) */
    float cl, cb, sl, sb;      /* cos/sin of the pole, as floats */
} gf_lambert;

/* ------------------------------------------------------------------ */
/* skygen configuration                                                */
/* ------------------------------------------------------------------ */

/* Raw binning keys of the skygen module (os_skygen.cpp:409-430): the library
 * applies the half-bin shifts and the luminosity-function hint itself. */
typedef struct gf_skygen_config {
    float m0, m1, dm;          /* apparent magnitude range and bin (keys m0/r0, m1/r1, dm) */
    float M0, M1;              /* absolute magnitude range (keys M0/ri0, M1/ri1); dM = dm */
    float dmin, dmax;          /* distance limits in pc (0, 0 = none) */
    int32_t nthreads;          /* crawl streams (reference grid*block, default 120*64 = 7680) */
    float nstars;              /* forced mean star count over all models (0 = from the model) */
    gf_lambert proj[2];        /* north/south projections */
} gf_skygen_config;

typedef enum {
    GF_MODEL_EXP_DISK = 1,                 /* src/skygen/model_expDisk.h */
    GF_MODEL_POWER_LAW_ELLIPSOID = 2,      /* src/skygen/model_powerLawEllipsoid.h */
    GF_MODEL_BROKEN_POWER_LAW = 3,         /* src/skygen/model_brokenPowerLaw.h: power-law ellipsoid with breaks */
    GF_MODEL_LCBULGE = 4,                  /* src/skygen/model_LCBulge.h: exp(-t/l), t = (x^n + (y/ba)^n + (z/ca)^n)^(1/n) */
    GF_MODEL_DENSITY_CUBE = 5              /* src/skygen/model_densityCube.h: f times a density grid, galactocentric */
} gf_model_type;

typedef enum {
    GF_FRAME_GALPLANE = 0,     /* center = orientation = galplane (transform.cpp:122-135) */
    GF_FRAME_EXPLICIT = 1      /* T and M given directly: xyz' = M (xyz + T) */
} gf_frame_kind;

/* A density model (model_*.cpp load()).  Parameters are the config-file values. */
typedef struct gf_model_config {
    int32_t type;              /* gf_model_type */
    int32_t comp;              /* sequential component id (0-based) */
    double f;                  /* key f: density at the LF sampling point */
    double l, h, rcut;         /* exponential disk: scale length, height, cylindrical cutoff (0 = none) */
    double n, ba, ca;          /* power-law ellipsoid: index, b/a, c/a */
    double rmin, rmax;         /* power-law ellipsoid radial limits (0, 0 = none) */
    int32_t frame;             /* gf_frame_kind */
    double Rg, z0;             /* galplane frame: Sun's distance to the centre and height */
    double T[3];               /* explicit frame translation */
    double M[9];               /* explicit frame rotation, row major */
    double lf_l, lf_b, lf_D;   /* where the LF was sampled (keys lf_l, lf_b, lf_D) */
    const double *lf_M;        /* LF knots (absolute magnitude); NULL = constant LF of 1 */
    const double *lf_phi;      /* LF values */
    int32_t lf_n;              /* number of knots */
    /* broken power law (keys n, rbreak; model_brokenPowerLaw.cpp:31-62): indices n_brk[0..nbreaks]
     * inside and beyond the ellipsoidal break radii rbreak[0..nbreaks-1] (pc), nbreaks <= 9 */
    int32_t nbreaks;
    double n_brk[10];
    double rbreak[9];
    /* The LC bulge (model_LCBulge.cpp:33-60) uses n, l, ba, ca and the frame, and scales the
     * LF by f instead of normalising the density at (lf_l, lf_b, lf_D). */
    /* The density cube (model_densityCube.h:34-79, .cpp:250-311): rho = f * cube(Rg - x, -y, z)
     * sampled at the nearest texel, value(X) = cube[k][j][i] with i = clamp(trunc((X - x0) * inv_dx
     * + 0.5), 0, nx - 1) per axis (x fastest in memory); f is not normalised at a point and the LF
     * (lf_M, lf_phi) is resampled to 1024 texels without clipping.  Uses Rg, f, the LF and these. */
    const float *cube;
    int32_t cube_n[3];                 /* nx, ny, nz */
    float cube_tc[3][2];               /* per axis (x0, inv_dx): the texture coordinates */
} gf_model_config;

typedef enum {
    GF_EXT_NONE = 0,           /* zero extinction (os_skygen.cpp:701-706) */
    GF_EXT_SCREEN_CSCB = 1,    /* Am = A0 / |sin b| in the bootstrap band at every distance */
    GF_EXT_MAPS = 2            /* 3-D maps of the two hemispheres (os_skygen.cpp:518-579, 699-814) */
} gf_extinction_kind;

/* One hemisphere's 3-D extinction map (load_extinction_map, os_skygen.cpp:518-579):
 * the bootstrap-band extinction on a grid of the hemisphere's Lambert coordinates
 * (X, Y) and distance modulus, already multiplied by the map's scale (nscale or
 * sscale).  Sampled at the nearest texel, as the reference's host build samples
 * its textures: index = clamp(trunc((v - x0) * inv_dx + 0.5), 0, n - 1) per axis. */
typedef struct gf_ext_map {
    const float *A;            /* [nz][ny][nx], x fastest */
    int32_t n[3];              /* nx (X), ny (Y), nz (DM) */
    float tc[3][2];            /* (x0, inv_dx) of X, Y and DM */
} gf_ext_map;

typedef struct gf_extinction {
    int32_t kind;
    float A0;                  /* bootstrap-band extinction towards the pole */
    /* GF_EXT_MAPS: the maps of the north (projection 0) and south (projection 1)
     * hemispheres; NULL = zero extinction there.  Both present: equal nz and DM axes.
     * The per-beam minima (beam_ammin of the requests) then hold nz values per beam,
     * beam_ammin[extIdx * nz + k] (gf_extinction_beam_minima). */
    const gf_ext_map *north, *south;
} gf_extinction;

/* Footprints of the analytic clipper (stars outside are flagged hidden). */
typedef enum {
    GF_FOOT_ALL = 0,           /* no clipping */
    GF_FOOT_LAMBERT_RECT = 1,  /* x0 <= X < x1, y0 <= Y < y1 in projection proj */
    GF_FOOT_CAP = 2,           /* angular distance from (l, b) <= r (degrees) */
    GF_FOOT_LATCUT = 3,        /* |b| > bmin (degrees) */
    GF_FOOT_LB_RECT = 4,       /* l0 <= l < l1 (degrees, through 360 when l0 > l1), b0 <= b < b1 */
    GF_FOOT_REGIONS = 5        /* the union of `regions` (footprint.cpp:729-758) */
} gf_footprint_kind;

/* One footprint specification of the reference (footprint.cpp: load_footprint_beam,
 * load_footprint_rect, clip_zone_of_avoidance): a beam (cap of radius r around
 * (lon, lat), minus a concentric hole of radius rhole) or a lon/lat rectangle, in
 * galactic or equatorial (J2000) coordinates, minus the galactic band |b| < bmin.
 * The reference approximates each region by a polygon sampled every dx and clips
 * stars against the polygon in the Lambert planes; here the regions are tested
 * exactly (a star on the sphere is inside or not), and pixels are covered by
 * supersampling the same test. */
typedef enum { GF_REGION_BEAM = 1, GF_REGION_RECT = 2 } gf_region_type;
typedef enum { GF_COORD_GAL = 0, GF_COORD_EQU = 1 } gf_coordsys;
#define GF_MAX_REGIONS 8
typedef struct gf_region {
    int32_t type;              /* gf_region_type */
    int32_t coordsys;          /* gf_coordsys */
    double a, b, c, d;         /* BEAM: lon lat r rhole; RECT: lon0 lon1 lat0 lat1 (degrees; lon0 == lon1: all longitudes) */
    double bmin;               /* galactic |b| < bmin removed (0: none) */
} gf_region;

typedef struct gf_footprint {
    int32_t kind;
    int32_t proj;
    double a, b, c, d;         /* RECT: x0 x1 y0 y1; CAP: l b r; LATCUT: bmin; LB_RECT: l0 l1 b0 b1 */
    int32_t nregions;          /* GF_FOOT_REGIONS: regions[0 .. nregions), nregions <= GF_MAX_REGIONS */
    int32_t pad_;
    gf_region regions[GF_MAX_REGIONS];
} gf_footprint;

/* ------------------------------------------------------------------ */
/* Output table: structure of arrays, row index fastest                */
/* (src/common/column.h:131-136, built-in schema otable.cpp:719-745)   */
/* Vector columns are stored component-major: col[k*pitch + row].      */
/* ------------------------------------------------------------------ */
#define GF_MAX_BANDS 17

typedef struct gf_table {
    int64_t capacity;          /* rows allocated (the pitch of vector columns) */
    int64_t size;              /* rows in use */
    int32_t nbands;            /* bands of the photometric system (0 = none) */
    /* skygen columns (os_skygen.cpp:838-858) */
    double  *lb;               /* [2]: l, b (degrees) */
    int32_t *projIdx;
    float   *projXY;           /* [2] */
    float   *DM;
    float   *absmag;           /* absolute magnitude in the bootstrap band */
    float   *XYZ;              /* [3] heliocentric, pc */
    int32_t *comp;
    float   *Am, *AmInf;
    int32_t *hidden;
    /* module columns */
    float   *FeH;
    float   *vcyl;             /* [3] vR, vPhi, vZ (km/s) */
    float   *mags;             /* [nbands] true magnitudes */
    int32_t *photoflags;
    float   *obsmags;          /* [nbands] magnitudes with photometric errors */
    float   *pm;               /* [3] mu_l/mu_ra, mu_b/mu_dec (mas/yr), v_r (km/s) */
    double  *radec;            /* [2] (degrees) */
    int32_t *FeH_comp;         /* Gaussian of the multi-Gaussian metallicity draw (GaussianFeH) */
    /* unresolved multiple systems (unresolvedMultiples_host.cpp:56-80): absmag + "Sys"[2] holds
     * the absolute magnitudes of the system's components (99.999 = absent), absmag + "SysNcomp"
     * their number; absmag then holds the system's total absolute magnitude */
    float   *absmagSys;        /* [2] */
    int32_t *absmagSysNcomp;
    int32_t systems;           /* 1: absmagSys is in use (set by gf_module_multiples); photometry then
                                * sums the luminosities of the system's components */
} gf_table;

/* ------------------------------------------------------------------ */
/* Module configurations (mirror the reference module data structs)    */
/* ------------------------------------------------------------------ */

typedef struct gf_fixedfeh_config {        /* fixedFeH_host.cpp:25-70 */
    float FeH;
    uint32_t comp_mask;                    /* bit c set: apply to component c */
} gf_fixedfeh_config;

typedef struct gf_vmoments {               /* Bond2010_gpu.cu.h:29-34 */
    float m[3][5];                         /* means: coefficients (a,b,c,d,e) of a + b|Z|^c + d R^e */
    float ss[6][5];                        /* dispersion tensor s11^.5 s12 s13 s22^.5 s23 s33^.5 */
} gf_vmoments;

typedef struct gf_bond2010_config {        /* os_Bond2010_data, Bond2010_gpu.cu.h:36-51 */
    uint32_t comp_thin, comp_thick, comp_halo;   /* component bit masks */
    float fk;                              /* probability of the first disk Gaussian */
    gf_vmoments disk_1, disk_2, halo;
    float M[9];                            /* galactic -> galplane rotation (row major) */
    float T[3];
} gf_bond2010_config;

typedef struct gf_photometry_config {      /* os_photometry_data + isochrone textures */
    int32_t nbands;                        /* ncolors + 1 */
    int32_t bidx;                          /* bootstrap band index */
    float reddening[GF_MAX_BANDS];
    int32_t nFeH, nMr;                     /* texture size */
    float tcFeH[2], tcMr[2];               /* texture coordinates (x0, 1/dx) */
    const float *colors;                   /* [ncolors][nMr][nFeH] */
    const uint8_t *eflags;                 /* [ncolors][nMr][nFeH], 1 = extrapolated */
    uint32_t comp_mask;
} gf_photometry_config;

typedef struct gf_photoerr_config {        /* os_photometricErrors: sigma(m) per band */
    int32_t nbands;
    int32_t nknots;                        /* knots per band */
    const double *mag;                     /* [nbands][nknots] */
    const double *sigma;                   /* [nbands][nknots] */
    uint64_t seed;                         /* key of the counter-based Gaussian draws */
} gf_photoerr_config;

typedef struct gf_feh_config {             /* os_FeH_data, src/modules/FeH_gpu.cu.h:26-36 (Ivezic et al. 2008) */
    float A[2];                            /* disk Gaussian amplitudes (normalised to sum 1, FeH_host.cpp:100-102) */
    float sigma[3];                        /* disk 1, disk 2, halo widths */
    float offs[3];                         /* disk 1, disk 2 offsets; halo mean */
    float Hmu, muInf, DeltaMu;             /* disk median: muInf + DeltaMu exp(-|Z| / Hmu) */
    uint32_t comp_thin, comp_thick, comp_halo;   /* component bit masks */
    float M[9];                            /* galactic -> model frame rotation (row major) */
    float T[3];
} gf_feh_config;

#define GF_GAUSSFEH_MAXCOMP 10
typedef struct gf_gaussfeh_config {        /* os_GaussianFeH_data, src/modules/GaussianFeH_gpu.cu.h:26-34 */
    int32_t ncomp;                         /* 1 .. GF_GAUSSFEH_MAXCOMP - 1 */
    float mean[GF_GAUSSFEH_MAXCOMP];
    float sigma[GF_GAUSSFEH_MAXCOMP];
    float pcum[GF_GAUSSFEH_MAXCOMP];       /* cumulative weights, pcum[ncomp - 1] = 1 */
    uint32_t comp_mask;                    /* components it applies to */
} gf_gaussfeh_config;

/* os_unresolvedMultiples (unresolvedMultiples_host.cpp:96-189, kernel
 * unresolvedMultiples_gpu.cu.h:36-123): each star of the selected components may
 * get a secondary with probability secprob(M1); its absolute magnitude is M1
 * (equal mass) or drawn from the inverse cumulative LF, above the primary's
 * cumulative LF value for GF_MULT_LF_M2_GT_M1.  The three tables are sampled at
 * the nearest texel, as the reference's host build samples its textures:
 * value(x) = tab[clamp(trunc((x - x0) * inv_dx + 0.5), 0, n - 1)]. */
typedef enum {
    GF_MULT_LF_M2_GT_M1 = 1,
    GF_MULT_LF = 2,
    GF_MULT_EQUAL_MASS = 3
} gf_multiples_algo;
#define GF_MULT_TEX 256
typedef struct gf_multiples_config {
    int32_t algo;                          /* gf_multiples_algo */
    uint32_t comp_mask;                    /* components it applies to */
    float sec_x0, sec_inv_dx;              /* probability of a secondary, against M1 */
    int32_t nsec;
    float secprob[64];
    float cum_x0, cum_inv_dx;              /* cumulative LF, against M */
    int32_t ncum;
    float cumlf[GF_MULT_TEX];
    float inv_x0, inv_inv_dx;              /* its inverse, against the cumulative value */
    int32_t ninv;
    float invcumlf[GF_MULT_TEX];
} gf_multiples_config;

typedef struct gf_vel2pm_config {          /* os_vel2pm_data, vel2pm_gpu.cu.h:26-34 */
    int32_t coordsys;                      /* 0 = GAL (pmlb), 1 = EQU (pmradec) */
    float vLSR, u0, v0, w0;
    float Rg;
} gf_vel2pm_config;

/* ------------------------------------------------------------------ */
/* Opaque handles                                                     */
/* ------------------------------------------------------------------ */
typedef struct gf_ctx gf_ctx;
typedef struct gf_skygen gf_skygen;
typedef struct gf_photometry gf_photometry;
typedef struct gf_photoerr gf_photoerr;

/* Description of the last error on this thread. */
const char *gf_last_error(void);

/* Create a context on CUDA device `device`. */
gf_status gf_ctx_create(int device, gf_ctx **out);
gf_status gf_ctx_destroy(gf_ctx *ctx);
/* Block until all work queued on the context's stream is done. */
gf_status gf_ctx_sync(gf_ctx *ctx);
/* Device-side timing on the context's stream: record event `slot` (0..15),
 * and read the elapsed milliseconds between two recorded slots. */
gf_status gf_ctx_mark(gf_ctx *ctx, int32_t slot);
gf_status gf_ctx_elapsed(gf_ctx *ctx, int32_t from, int32_t to, float *ms);
/* Number of this library's kernels launched by the process so far. */
int64_t gf_launch_count(void);

/* Per-phase device time (like the reference's kernelRunSwatch, gpu.h:251-254):
 * when enabled, every kernel phase is bracketed by CUDA events on the context's
 * stream; gf_profile_read returns the accumulated milliseconds and launch
 * counts per phase (GF_PROF_*) and resets them. */
enum {
    GF_PROF_INTEGRATE = 0, GF_PROF_DRAW_WINDOW = 1, GF_PROF_DRAW_RERUN = 2, GF_PROF_PLACE = 3,
    GF_PROF_SORT = 4, GF_PROF_CLIPPER = 5, GF_PROF_FEH = 6, GF_PROF_BOND2010 = 7, GF_PROF_PHOTOMETRY = 8,
    GF_PROF_PHOTOERR = 9, GF_PROF_VEL2PM = 10, GF_PROF_GAL2OTHER = 11,
    GF_PROF_SLOTS = 12,          /* batched draw: model density at the slot distances of each pixel */
    GF_PROF_EXPAND = 13,         /* batched draw: star records of the bins with stars */
    GF_PROF_BATCH_DRAW = 14,     /* batched draw: the Poisson draw of every stream (one launch per model pass) */
    GF_PROF_SETUP = 15,          /* many-request calls: host wall time from the call to the integrate pass (checks,
                                    model set-up, staging and upload of the pencil beams, stream seeding) */
    GF_PROF_PLAIN = 16,          /* many-request calls: device time of the requests run through the plain path
                                    inside the call (their own phases are counted as well) */
    GF_PROF_NPHASES = 17
};
gf_status gf_profile_enable(gf_ctx *ctx, int32_t on);
gf_status gf_profile_read(gf_ctx *ctx, double *ms, int64_t *launches);

/* ---- persistent multiply-with-carry streams (cux.cpp:404-435, cuda_rng.h:466-497) ---- */

/* Seed nstreams (<= 65536, rounded up to a multiple of 64) streams from the
 * srand48 seed `seed48`, the value the reference derives as
 * (uint32)(seeder.uniform() * 2^24) from its GSL generator. */
gf_status gf_rng_init(gf_ctx *ctx, uint32_t seed48, int32_t nstreams);
/* The srand48 seed the reference derives from a galfast command-line seed
 * (GSL's default mt19937 seeded with `seed`, first uniform, times 2^24). */
uint32_t gf_rng_seed48_from_cli_seed(uint64_t seed);
/* Copy the stream states to/from host memory: [3][nstreams] words a, c, x. */
gf_status gf_rng_get_state(gf_ctx *ctx, uint32_t *host_state, int32_t nstreams);
gf_status gf_rng_set_state(gf_ctx *ctx, const uint32_t *host_state, int32_t nstreams);

/* n Poisson deviates drawn one after another from ONE stream on the device:
 * out[i] = poisson(mu[i]) with rng_t::poisson (src/common/cuda_rng.h:344-376),
 * including its gamma / binomial reduction for mu > 10.  state[3] = (a, c, x),
 * host memory, updated to the stream's state after the draws.  A direct check
 * of the sampler the draw kernels use; means must lie in [0, 1e7). */
gf_status gf_rng_poisson(gf_ctx *ctx, uint32_t state[3], const float *mu, int32_t n, uint32_t *out);

/* ---- skygen ---- */

/* Build the generator for a footprint pixelisation and a list of models
 * (os_skygen::construct + skygenHost<T>::init for each model). */
gf_status gf_skygen_create(gf_ctx *ctx, const gf_skygen_config *cfg,
                           const gf_pencil_beam *pixels, int32_t npixels,
                           const float *beam_ammin,          /* [npixels] minimum extinction per beam, or NULL */
                           const gf_extinction *ext,
                           const gf_model_config *models, int32_t nmodels,
                           gf_skygen **out);
gf_status gf_skygen_destroy(gf_skygen *sky);

/* Derived per-model binning after the LF hint (skygenParams after init). */
typedef struct gf_skygen_model_info {
    float m0, m1, dm, M0, M1, dM;
    int32_t nm, nM, npixels, nthreads;
    float f;                               /* renormalised density factor */
    float lf_x0, lf_inv_dx;                /* LF texture coordinates */
    int32_t lf_n;
    float norm;
} gf_skygen_model_info;
gf_status gf_skygen_model_info_get(gf_skygen *sky, int32_t model, gf_skygen_model_info *info);
/* Copy the resampled LF of a model (lf_n floats) to host memory. */
gf_status gf_skygen_model_lf_get(gf_skygen *sky, int32_t model, float *lf);

/* Expected star counts of one model over all pixels (integrateCounts).
 * per_pixel (nullable, host, npixels doubles) receives the covered counts per beam. */
gf_status gf_skygen_integrate(gf_skygen *sky, int32_t model,
                              double *expected, double *expected_covered,
                              double *per_pixel);
gf_status gf_skygen_set_norm(gf_skygen *sky, int32_t model, float norm);

/* Draw the next output batch of one model into the device table `out`
 * (capacity rows).  The batch follows the reference CPU path: streams fill
 * the table in stream order; the batch is sorted by (hidden, l, b, DM, M, Am)
 * and truncated at the first hidden row.  *n_generated receives the stars
 * drawn in the batch (before truncation), out->size the rows kept, *done = 1
 * after the model's last batch.  Between calls the caller may run modules
 * that consume the streams (gf_module_bond2010), as the reference pipeline does. */
gf_status gf_skygen_draw(gf_skygen *sky, int32_t model, gf_table *out,
                         int64_t *n_generated, int32_t *done);

/* ---- device tables ---- */
gf_status gf_table_alloc(gf_ctx *ctx, int64_t capacity, int32_t nbands, gf_table *t);
gf_status gf_table_free(gf_ctx *ctx, gf_table *t);
/* Copy rows [0, t->size) of every allocated column to a host table with the same capacity layout. */
gf_status gf_table_download(gf_ctx *ctx, const gf_table *dev, gf_table *host);
/* rows [begin, end) of a device table into rows [0, end - begin) of a host table
 * (one request's rows of a gf_catalog_run_multi table, for instance) */
gf_status gf_table_download_rows(gf_ctx *ctx, const gf_table *dev, int64_t begin, int64_t end, gf_table *host);

/* ---- modules: process rows [begin, end) of a device table ---- */
gf_status gf_module_clipper(gf_ctx *ctx, const gf_footprint *foot, const gf_lambert proj[2],
                            gf_table *t, int64_t begin, int64_t end);
gf_status gf_module_fixedfeh(gf_ctx *ctx, const gf_fixedfeh_config *cfg, gf_table *t, int64_t begin, int64_t end);
/* os_FeH (FeH_host.cpp:60-78, kernel FeH_gpu.cu.h:43-87) and os_GaussianFeH
 * (GaussianFeH_host.cpp:56-76, kernel GaussianFeH_gpu.cu.h:42-73): metallicities
 * drawn from the context's streams, 256 rows per stream as the reference's
 * kernels take them (row r of [begin, end) uses stream (r - begin) / 256). */
gf_status gf_module_feh(gf_ctx *ctx, const gf_feh_config *cfg, gf_table *t, int64_t begin, int64_t end);
gf_status gf_module_gaussfeh(gf_ctx *ctx, const gf_gaussfeh_config *cfg, gf_table *t, int64_t begin, int64_t end);
gf_status gf_module_bond2010(gf_ctx *ctx, const gf_bond2010_config *cfg, gf_table *t, int64_t begin, int64_t end);
/* os_unresolvedMultiples: the tables from the binary fraction (knots frac_M, frac_p;
 * nfrac = 0: 1 everywhere) and the luminosity function of the secondaries (knots
 * lf_M, lf_phi; nlf = 0: flat over [-100, 100]) as os_unresolvedMultiples::construct
 * builds them; then the module on rows [begin, end), drawing from the context's
 * streams 256 rows per stream like the other modules.  Rows it skips (hidden,
 * other components) hold a single-star system: (absmag, 99.999) and 1. */
gf_status gf_multiples_build(const double *frac_M, const double *frac_p, int32_t nfrac, const double *lf_M,
                             const double *lf_phi, int32_t nlf, int32_t algo, uint32_t comp_mask, gf_multiples_config *out);
gf_status gf_module_multiples(gf_ctx *ctx, const gf_multiples_config *cfg, gf_table *t, int64_t begin, int64_t end);
/* Photometry: upload the colour grids once (os_photometry::construct), then process batches. */
gf_status gf_photometry_create(gf_ctx *ctx, const gf_photometry_config *cfg, gf_photometry **out);
gf_status gf_photometry_destroy(gf_photometry *p);
gf_status gf_module_photometry(gf_ctx *ctx, const gf_photometry *p, gf_table *t, int64_t begin, int64_t end);
/* Photometric errors: sigma(m) knots per band; the Gaussian deviate of (row, band) is
 * keyed by (seed, row_offset + row, band), so batches reproduce a single run. */
gf_status gf_photoerr_create(gf_ctx *ctx, const gf_photoerr_config *cfg, gf_photoerr **out);
gf_status gf_photoerr_destroy(gf_photoerr *p);
gf_status gf_module_photoerrors(gf_ctx *ctx, const gf_photoerr *p, int64_t row_offset,
                                gf_table *t, int64_t begin, int64_t end);
gf_status gf_module_vel2pm(gf_ctx *ctx, const gf_vel2pm_config *cfg, gf_table *t, int64_t begin, int64_t end);
gf_status gf_module_gal2other(gf_ctx *ctx, int32_t coordsys, gf_table *t, int64_t begin, int64_t end);

/* ---- the catalog path: os_skygen::run + drawSources + the module chain ---- */

typedef struct gf_job {
    gf_skygen_config sky;
    const gf_pencil_beam *pixels;
    int32_t npixels;
    const float *beam_ammin;                   /* [npixels] or NULL */
    gf_extinction ext;
    const gf_model_config *models;             /* run in component order */
    int32_t nmodels;
    uint32_t seed48;                           /* srand48 seed of the persistent streams */
    int32_t nstreams;                          /* streams to seed (0 = keep the context's streams) */
    int64_t capacity;                          /* rows per output batch (the otable capacity, KBATCH) */
    int32_t nbands;                            /* bands of the output table (photometry) */
    const gf_footprint *foot;                  /* clipper; NULL = no clipping */
    const gf_fixedfeh_config *feh;             /* NULL = module absent */
    const gf_bond2010_config *kin;
    const gf_photometry_config *phot;
    const gf_photoerr_config *perr;
    const gf_vel2pm_config *v2pm;
    int32_t gal2other;                         /* 0 = absent, 1 = equatorial (radec) */
    const gf_feh_config *feh_ivezic;           /* os_FeH (after fixedFeH), NULL = absent */
    const gf_gaussfeh_config *feh_gauss;       /* os_GaussianFeH (after os_FeH), NULL = absent */
    const gf_multiples_config *multiples;      /* os_unresolvedMultiples (after the metallicities), NULL = absent */
} gf_job;

#define GF_MAX_MODELS 32
typedef struct gf_catalog_stats {
    double expected[GF_MAX_MODELS];            /* integrateCounts: stars to generate */
    double expected_covered[GF_MAX_MODELS];    /* ... within the footprint */
    int64_t generated[GF_MAX_MODELS];          /* stars drawn (before truncation) */
    int64_t stored[GF_MAX_MODELS];             /* rows passed down the module chain */
    int32_t batches;
    float norm;                                /* density normalisation applied (1 = none) */
} gf_catalog_stats;

/* Called once per output batch with the device table after all modules ran;
 * row_offset is the number of rows delivered before this batch.  A nonzero
 * return stops the run (gf_catalog_run then returns GF_E_STATE). */
typedef int (*gf_batch_callback)(void *user, int32_t model, const gf_table *dev_batch, int64_t row_offset);

gf_status gf_catalog_run(gf_ctx *ctx, const gf_job *job, gf_batch_callback cb, void *user, gf_catalog_stats *stats);

/* ---- precision form ---- */

typedef struct gf_precision_report {
    double expected32;          /* FP32 bin counts (as generated), Kahan-summed per pixel in FP32 */
    double expected64;          /* FP64 evaluation of the same bins (same LF texels and anchors) */
    double total_rel_err;       /* |expected32 - expected64| / expected64 */
    double bin_max_rel_err;     /* over bins with >= 1e-30 expected stars (smaller counts pass through
                                   subnormal floats in the reference's expressions) */
    double bin_mean_rel_err;
    double pixel_max_rel_err;   /* per-pixel sums, over pixels with a nonzero FP64 count */
    double pixel_mean_rel_err;
    int64_t bins;               /* bins in the per-bin statistics */
} gf_precision_report;

/* The expected counts of one model in both precisions (see gf_precision_report).
 * per_pixel32/per_pixel64: npixels entries or NULL; dm_hist64: FP64 counts per
 * distance-modulus row d = im + iM (nm + nM - 1 entries, DM = m0 - M1 + d dm) or
 * NULL.  Needs nm*nM to be a multiple of 10 (the crawl's anchors per pixel). */
gf_status gf_skygen_precision(gf_skygen *s, int32_t model, gf_precision_report *rep, double *per_pixel32,
                              double *per_pixel64, double *dm_hist64);

/* ---- many requests per pass ---- */

/* Called once per model with the device table holding that model's rows of
 * every request: the rows of request j are [row_begin[j], row_begin[j] +
 * row_count[j]) (njobs entries each, host memory).  Requests that run alone
 * (below) deliver their batches through the same callback with only their own
 * entry nonzero.  A nonzero return stops the run (GF_E_STATE). */
typedef int (*gf_multi_callback)(void *user, int32_t model, const gf_table *dev_rows, const int64_t *row_begin,
                                 const int64_t *row_count);

/* The catalogs of njobs independent requests (os_skygen::run + the module
 * chain of each, as gf_catalog_run), generated together: every crawl, sort
 * and module pass covers all requests at once.  Each request's rows are those
 * gf_catalog_run produces for it alone, bit for bit.  A request whose expected
 * stars of some model reach its batch capacity (within 8 sigma, see
 * gf_multi_set_admission), or whose grid has nm*nM not a multiple of 10, runs
 * alone through gf_catalog_run after the others.  All requests need the same nthreads, model kinds (in component
 * order) and fixedFeH/Bond2010/vel2pm/gal2other settings, nstreams > 0 and
 * nstars = 0; footprints, models, grids, seeds, capacities and photometry may
 * differ.  stats: njobs entries or NULL.  No counterpart in the reference,
 * which generates one catalog per process (os_skygen.cpp:866-932). */
gf_status gf_catalog_run_multi(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, void *user,
                               gf_catalog_stats *stats);

/* The admission rule of gf_catalog_run_multi: a request is generated with the
 * others when every model's expected stars e satisfy e + sigmas sqrt(e) + 1024 <
 * its batch capacity (default sigmas = 8); otherwise it runs alone through
 * gf_catalog_run.  A batched request whose stars fill a whole batch anyway has
 * its rows of that model on withheld and runs alone at the end of the call,
 * delivering only the components not delivered yet, so its catalog is still the
 * one gf_catalog_run gives it. */
gf_status gf_multi_set_admission(gf_ctx *ctx, double sigmas);

/* Device memory that one chunk of a multi-request run may use for its draw
 * passes (records, placement, sort and output columns, about 320 bytes per
 * expected star of a request's largest model).  Requests are generated in
 * consecutive chunks that fit; the callback then sees each chunk's rows.
 * 0 (the default) = 60% of the free device memory at the start of the run. */
gf_status gf_multi_set_memory_budget(gf_ctx *ctx, int64_t bytes);

/* gf_catalog_run_multi with the rows delivered in host memory.  After each model
 * pass the library copies the pass's rows to a ring of page-locked host tables on
 * a second stream while the device generates the next pass, in pieces of at most
 * piece_rows rows (0: 16M).  cb sees one piece: request j's rows are
 * host rows row_begin[j] .. row_begin[j] + row_count[j] - 1 (count 0: none in
 * this piece); a request's rows of a model arrive in order, possibly over several
 * pieces.  The host table is valid until cb returns.  cb runs on a CUDA driver
 * thread, one piece at a time in delivery order, and must not call CUDA or this
 * library; a nonzero return stops the run (GF_E_STATE) and no later piece reaches
 * cb.  Requests that need several output batches run through the plain path after
 * the batched passes; their batches are staged on the device and follow the
 * batched rows through the same copy stream.  All callbacks have returned when
 * this function returns. */
typedef int (*gf_multi_host_callback)(void *user, int32_t model, const gf_table *host, const int64_t *row_begin,
                                      const int64_t *row_count);
gf_status gf_catalog_run_multi_host(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, int64_t piece_rows,
                                    gf_multi_host_callback cb, void *user, gf_catalog_stats *stats);

/* Columns of a gf_table (bits for gf_multi_set_host_columns). */
enum {
    GF_COL_LB = 1u << 0, GF_COL_PROJIDX = 1u << 1, GF_COL_PROJXY = 1u << 2, GF_COL_DM = 1u << 3,
    GF_COL_ABSMAG = 1u << 4, GF_COL_XYZ = 1u << 5, GF_COL_COMP = 1u << 6, GF_COL_AM = 1u << 7,
    GF_COL_AMINF = 1u << 8, GF_COL_HIDDEN = 1u << 9, GF_COL_FEH = 1u << 10, GF_COL_VCYL = 1u << 11,
    GF_COL_MAGS = 1u << 12, GF_COL_PHOTOFLAGS = 1u << 13, GF_COL_OBSMAGS = 1u << 14, GF_COL_PM = 1u << 15,
    GF_COL_RADEC = 1u << 16, GF_COL_FEHCOMP = 1u << 17, GF_COL_ABSMAGSYS = 1u << 18, GF_COL_SYSNCOMP = 1u << 19,
    GF_COL_ALL = (1u << 20) - 1,
    /* the output catalog of the full-sky form: ra, dec, DM, Mr, true and observed
     * magnitudes, vR/vPhi/vZ, proper motions (and radial velocity) */
    GF_COL_CATALOG = GF_COL_RADEC | GF_COL_DM | GF_COL_ABSMAG | GF_COL_MAGS | GF_COL_OBSMAGS | GF_COL_VCYL | GF_COL_PM
};

/* The columns gf_catalog_run_multi_host copies to host memory (default
 * GF_COL_ALL); the others are NULL in the host tables the callback sees.  The
 * column selection of galfast's text output (the output module's column list,
 * src/pipeline.cpp:199-289), applied before the copy instead of when writing. */
gf_status gf_multi_set_host_columns(gf_ctx *ctx, uint32_t columns);

/* Warps per CTA of the batched draw kernel (one warp per stream), by model kind
 * (GF_MODEL_*): 1, 2, 4 or 8.  The first gf_catalog_run_multi pass of each kind
 * times the four on the head of its work queue and keeps the fastest for the
 * context (0 = not tuned yet); gf_tuning_set fixes the choice, or with 0 asks
 * for a new trial. */
gf_status gf_tuning_get(gf_ctx *ctx, int32_t model_kind, int32_t *warps_per_cta);
gf_status gf_tuning_set(gf_ctx *ctx, int32_t model_kind, int32_t warps_per_cta);

/* ---- serving: continuous batching of requests ---- */

typedef struct gf_server gf_server;
/* rows [begin, begin + count) of dev hold this request's rows of one model
 * (called on a worker thread; ctx is that worker's context, for downloads such as
 * gf_table_download_rows; a nonzero return fails the request's batch) */
typedef int (*gf_server_rows)(void *user, int64_t request, int32_t model, gf_ctx *ctx, const gf_table *dev, int64_t begin,
                              int64_t count);
/* the request is complete (status GF_OK) or failed; stats are the request's own */
typedef void (*gf_server_done)(void *user, int64_t request, gf_status status, const gf_catalog_stats *stats);

/* A request server on one device: nworkers worker threads, each with its own
 * context and CUDA stream, take the compatible requests waiting at the head of
 * the queue (at most max_batch) and generate them together.  After a batch's
 * integrate pass each request's device-memory need is known from its expected
 * star counts; the worker reserves, from memory_budget bytes shared by all
 * workers, the needs of the leading requests that fit what the running batches
 * leave free, generates those, and returns the others to the head of the queue,
 * where they join the requests that arrived meanwhile in the next batch.  Batches
 * of several workers run side by side on the device when their reservations fit
 * together.  No counterpart in the reference. */
gf_status gf_server_create(int32_t device, int32_t nworkers, int64_t memory_budget, int32_t max_batch, gf_server **out);
/* Queue one request.  The job and the arrays and configurations it points to are
 * copied: the caller's memory may be reused when this returns.  *request
 * receives its id. */
gf_status gf_server_submit(gf_server *s, const gf_job *job, gf_server_rows rows, gf_server_done done, void *user,
                           int64_t *request);
/* Wait until every submitted request is done; returns the first error seen. */
gf_status gf_server_drain(gf_server *s);
typedef struct gf_server_info {
    int64_t runs;              /* batches generated */
    int64_t completed;         /* requests done (successfully or not) */
    int64_t deferred;          /* times a request went back to the queue at admission */
    int64_t peak_reserved;     /* most device memory reserved at once by running batches (bytes) */
    int32_t peak_running;      /* most batches generating at once */
    int32_t queued;            /* requests waiting now */
    int32_t active;            /* batches taken from the queue and not finished, now */
    int32_t pad;
} gf_server_info;
gf_status gf_server_get_info(gf_server *s, gf_server_info *out);
/* paused != 0: the workers take no new batch (running batches finish); 0 resumes */
gf_status gf_server_pause(gf_server *s, int32_t paused);
gf_status gf_server_destroy(gf_server *s);

/* ---- expected counts without device allocation ---- */

/* Expected star counts of ONE density model over a footprint, computed with
 * the integrate pass of gf_skygen_integrate but without allocating device
 * memory: for hosts that own all of the GPU's memory themselves (a framework
 * with its own arena, or a process that must not call cudaMalloc/cudaFree
 * while it runs).  No counterpart in the reference: galfast allocates its
 * buffers itself (skyconfig_impl.h:196-241).
 *   d_pixels, d_beam_ammin   caller's device buffers (d_beam_ammin may be NULL)
 *   d_result                 caller's device buffer of 2 doubles: expected, expected within the footprint
 *   cuda_stream              cudaStream_t to run on (NULL = default stream); synchronised before return
 * The scratch (per-stream partial sums, LF, distance table) is a fixed 1.3 MB
 * __device__ array of the library: at most 65536 streams, 1024 LF samples and
 * 65536 (m, M) bins per pixel; larger requests are rejected with GF_E_INVALID.
 * Devices 0-63 (GF_E_UNSUPPORTED above).  The first call on each device looks up
 * the array's address.  Every call synchronises its stream before returning,
 * also on failure, so it must not be called while its stream is being captured.
 * Calls share the array, so calls that overlap on the GPU race. */
gf_status gf_skygen_integrate_static(const gf_skygen_config *cfg, const gf_pencil_beam *d_pixels, int32_t npixels,
                                     const float *d_beam_ammin, const gf_extinction *ext,
                                     const gf_model_config *model, double *d_result, void *cuda_stream);

/* ---- catalog text output (os_textout, src/pipeline.cpp:199-289) ---- */

/* The columns of the text catalog and their names.  The file is the
 * reference's: a "# " header line with every output column's definition
 * (otable::serialize_header, src/common/otable.cpp:542-558), an optional
 * "# generated with galfast version ..." line, then one line per row that is
 * not hidden, each column component printed with the column's printf format
 * (otable.cpp:719-745) and separated by single spaces.  Columns come in the
 * reference's output order: lb, radec, XYZ, DM, the absolute magnitude, comp,
 * FeH, vcyl, pmlb/pmradec, Am, AmInf, then the photometry columns by name. */
typedef struct gf_textout_config {
    const char *bandset;             /* photometric system, e.g. "SDSSugriz" (NULL: no photometry columns) */
    const char *const *bands;        /* nbands band names, e.g. "SDSSu" ... */
    int32_t nbands;
    const char *band;                /* bootstrap band of the absolute magnitude, e.g. "SDSSr" */
    const char *absband;             /* its column name (NULL: "abs" + band) */
    int32_t radec;                   /* gal2other equatorial coordinates present */
    int32_t feh;                     /* FeH present */
    int32_t feh_comp;                /* FeH_comp present (GaussianFeH) */
    int32_t vcyl;                    /* Bond2010 velocities present */
    int32_t pm_coordsys;             /* vel2pm: -1 absent, 0 pmlb, 1 pmradec */
    int32_t photoerrors;             /* observed magnitudes present */
    const int32_t *comp_ids;         /* comp column value -> component id written (NULL: as stored) */
    int32_t ncomp;
    const char *version;             /* galfast version for the second header line (NULL: none) */
    int32_t threads;                 /* formatting threads (0: all hardware threads) */
    int32_t multiples;               /* unresolved multiples present: absmag + "Sys"[2] and + "SysNcomp" */
} gf_textout_config;

typedef struct gf_textout gf_textout;
gf_status gf_textout_open(const char *path, const gf_textout_config *cfg, gf_textout **out);
/* Append the rows [begin, end) of a HOST table that are not hidden (formatted on
 * the writer's threads, written in order).  One write at a time per writer. */
gf_status gf_textout_write(gf_textout *w, const gf_table *host, int64_t begin, int64_t end);
/* Close the file; rows and bytes written (nullable). */
gf_status gf_textout_close(gf_textout *w, int64_t *rows, int64_t *bytes);

/* A FITS catalog (os_fitsout, src/pipeline.cpp:767-1035) with the same columns:
 * an empty primary HDU, a binary table CATALOG (one column per output column,
 * TTYPE its name, TFORM its width and D/E/J type, big-endian rows of the
 * visible rows), then a binary table METADATA whose single row holds the
 * column definitions (and version line) of the text header.  The handle is a
 * catalog writer like gf_textout_open's: write with gf_textout_write, finish
 * with gf_textout_close (which writes the row count into the CATALOG header). */
gf_status gf_fitsout_open(const char *path, const gf_textout_config *cfg, gf_textout **out);

/* One writer per request of a multi-request run: pass gf_textout_multi_sink and
 * a gf_textout_set to gf_catalog_run_multi_host to write every request's
 * catalog while the device generates the next pass (writers[j] NULL: request
 * j is not written). */
typedef struct gf_textout_set {
    int32_t njobs;
    gf_textout *const *writers;
} gf_textout_set;
int gf_textout_multi_sink(void *set, int32_t model, const gf_table *host, const int64_t *row_begin, const int64_t *row_count);

/* ---- failure injection (tests) ---- */

/* Make the library's device allocations fail as if the device were out of
 * memory, without calling cudaMalloc for them: the allocations after the next
 * `after` ones fail, `count` of them (0: every one), then allocations succeed
 * again; after < 0 turns it off.  Process-wide.  gf_catalog_run and
 * gf_catalog_run_multi answer an out-of-memory failure before their first
 * delivered rows by freeing the context's cached buffers and running once more
 * (as src/common/cux.cpp:189-198 collects garbage and retries an allocation);
 * a second failure returns GF_E_OOM and leaves the context usable. */
gf_status gf_debug_fail_allocations(int64_t after, int64_t count);

/* ---- host-side setup helpers (no GPU needed) ---- */

/* Lambert projection with pole (l0, b0) in degrees (lambert::init, skygen.h:115-120). */
gf_status gf_lambert_init(double l0_deg, double b0_deg, gf_lambert *p);
/* Pixelise a footprint on the two hemispheres' Lambert grids (cell side dx_deg
 * degrees, grid anchored at each pole; b >= 0 belongs to the north grid), with
 * the covered fraction of each cell and, for the screen extinction, the minimum
 * extinction over the cell.  Replaces the GPC footprint pixelisation of
 * os_skygen::load_footprints (os_skygen.cpp:239-283) for analytic footprints.
 * Call with pixels == NULL to count. */
gf_status gf_footprint_pixelize(const gf_footprint *foot, double dx_deg, const gf_lambert proj[2],
                                const gf_extinction *ext, gf_pencil_beam *pixels, float *beam_ammin,
                                int64_t max_pixels, int64_t *npixels);
/* The per-beam extinction table of GF_EXT_MAPS (find_extinction_minima,
 * os_skygen.cpp:285-342, and load_extinction_maps, :770-800): for every beam (its
 * extIdx) and every DM texel z of the maps, the smallest extinction one texel
 * closer (A(x, y, z - 1), 0 at z = 0) over the map texels that may overlap the
 * beam, in each given map projected with its hemisphere's Lambert pole; +inf where
 * no texel qualifies.  out[npixels * nz]; *nz receives the depth (call with
 * out == NULL to get it). */
gf_status gf_extinction_beam_minima(const gf_extinction *ext, const gf_lambert proj[2], const gf_pencil_beam *pixels,
                                    int32_t npixels, float *out, int32_t *nz);
/* Resample a photometric-system table (rows: Mr, FeH, c_1..c_ncolors) to the colour
 * and extrapolation-flag grids of os_photometry::construct (photometry_host.cpp:233-344).
 * colors/eflags: [ncolors][nMr][nFeH]; call with colors == NULL for the sizes. */
gf_status gf_photometry_build(const double *rows, int32_t nrows, int32_t ncolors, double dFeH, double dMr,
                              float *colors, uint8_t *eflags, int32_t *nFeH, int32_t *nMr,
                              float tcFeH[2], float tcMr[2]);
/* The model setup of gf_skygen_create on the host alone: info[nmodels], lf[nmodels][1024] (nullable). */
gf_status gf_skygen_setup_host(const gf_skygen_config *cfg, int32_t npixels, const gf_model_config *models, int32_t nmodels,
                               gf_skygen_model_info *info, float *lf);
/* The stream multipliers a_i (safe primes a_i 2^32 - 1, cuda_rng.h:466-497). */
int gf_multipliers(uint32_t *out, int32_t n);
/* The seeded stream states [3][nstreams] that gf_rng_init uploads. */
void gf_rng_seed_host(uint32_t seed48, int32_t nstreams, uint32_t *state);
/* First n outputs of MT19937 seeded with `seed` (the GSL default generator's core). */
void gf_mt19937_outputs(uint32_t seed, int n, uint32_t *out);

#ifdef __cplusplus
}
#endif

#endif /* GALFAST_B200_H */
