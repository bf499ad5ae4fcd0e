/*
 * gf_internal.h -- structures shared by the host setup code and the sm_100a
 * kernels of the galfast_b200 library (not part of the public ABI).
 */
#pragma once
#include <stdint.h>
#include "../../include/galfast_b200.h"

#define GF_BLOCK 10                 /* bins per crawl block (skygen.cu.h:467) */
#define GF_POGSON 0.4605170185988091f

/* One density model as the crawl kernel sees it: the model parameters of
 * model_expDisk.h / model_powerLawEllipsoid.h after load(), and the
 * skygenParams of skygenHost<T> after init() (skyconfig_impl.h:244-297). */
struct SkyModel {
    int32_t type, comp;
    float f, l, h, r_cut2;
    float n, ba, ca, rminSq, rmaxSq;
    float T[3];
    float M[9];
    float m0, m1, dm, M0, M1, dM, dmin, dmax;
    int32_t npixels, nm, nM, nthreads;
    float norm;
    float lf_x0, lf_inv_dx;
    int32_t lf_n;
    const float *lf;               /* device pointer, lf_n samples */
    /* power-law ellipsoids: index nArr[k] and scale fArr[k] between break radii
     * rbreakSq[k - 1] and rbreakSq[k] (a plain power law: nbreaks = 0, nArr[0] = n, fArr[0] = 1) */
    int32_t nbreaks;
    float nArr[10], fArr[10], rbreakSq[9];
    /* density cube: device grid (x fastest) and per-axis texture coordinates (x0, inv_dx) */
    const float *cube;
    int32_t cube_n[3];
    float cube_tc[3][2];
};

/* Sky geometry shared by all models of a generator. */
struct SkyGeom {
    const gf_pencil_beam *pixels;  /* device */
    int32_t npixels;
    const float *ammin;            /* device, per-beam minimum extinction, or null (GF_EXT_MAPS: ext_nz per beam) */
    int32_t ext_kind;
    float A0;
    gf_lambert proj[2];
    /* GF_EXT_MAPS: depth and DM texture coordinates of the per-beam rows, and the
     * north/south maps (device, x fastest; null = zero extinction) */
    int32_t ext_nz;
    float ext_tcz[2];
    const float *map[2];
    int32_t map_n[2][3];
    float map_tc[2][3][2];
};

/* A star drawn by the crawl, to be placed by the star kernel. */
struct StarRecord {
    int32_t stream;                /* crawl stream; (request << 16) | stream in a multi-request launch */
    int32_t ilb;                   /* pixel */
    int16_t im, iM;                /* bin */
    int32_t seq;                   /* ordinal of the star among its stream's stars in this batch */
    float u[4];                    /* uniforms x, y, M, m (u[2..3] = 0 if hidden by x^2+y^2>2) */
};

/* A bin with stars found by the batched draw: its stars' uniforms start at the
 * stream state v_star (after the Poisson sampler's uniforms), and the stream
 * had drawn nstars stars before it.  Expanded into k StarRecords. */
struct EventRecord {
    int32_t stream;                /* (request << 16) | stream */
    int32_t ilb;                   /* pixel */
    int16_t im, iM;                /* bin */
    int32_t k;                     /* stars in the bin */
    int32_t nstars;                /* the stream's stars before this bin */
    int32_t pad;
    uint64_t v_star;               /* stream state c*2^32 + x before the first star's first uniform */
};

/* Anchor quantities of a bin in the form the per-bin loop consumes:
 *   Am  beam extinction, or +inf when the anchor's distance is outside [dmin, dmax)
 *   ms  model density at the anchor position
 *   D3  D*D*D
 *   K   dA * POGSON * dm * dM of the anchor's pixel
 * so that mu = ((((LF(M) * ms) * norm) * D3) * K), cut when m + Am > m1
 * (skygen.cu.h:551-565, the same float operations in the same order). */
struct AnchorX {
    float Am, ms, D3, K;
};

/* Per-stream crawl state (structure of arrays over the crawl streams).
 * The stream's bin sequence is a list of blocks; block j starts at local
 * diagonal index k_j in pixel ilb_j (the reference's jump, skygen.cu.h:522-531). */
struct CrawlState {
    int32_t *status;               /* 0 fresh, 1 paused/running, 2 finished */
    int32_t *blk_ilb;              /* start pixel of the current block */
    int32_t *blk_k;                /* local diagonal index of the current block start */
    int32_t *pos;                  /* next bin within the current block, 0..10 */
    int32_t *ndraw;                /* stars still to draw for the last processed bin */
    int32_t *cur_ilb, *cur_im, *cur_iM;   /* last processed bin */
    AnchorX *anc;                  /* anchor in effect at the cursor */
    int64_t *nstars;               /* stars drawn by the stream in the current batch */
};

/* Resumable position of a stream just before one of its bins with stars:
 * restarting the crawl from it replays that bin's Poisson draw. */
struct Checkpoint {
    int32_t stream;                /* as StarRecord::stream */
    int32_t nstars;                /* stars the stream had drawn in the batch before this bin */
    int32_t blk_ilb, blk_k, pos;   /* cursor: block start pixel, block start index, bin in block */
    int32_t pad;
    AnchorX anc;                   /* anchor in effect at the bin */
    uint64_t v;                    /* stream state c*2^32 + x before the bin's first uniform */
};

/* Division by a loop-invariant divisor d >= 1 for numerators below 2^31:
 * n / d = (umulhi(n, mul) + n) >> shift with shift = ceil(log2 d) and
 * mul = floor(2^32 (2^shift - d) / d) + 1 (Granlund and Montgomery, "Division
 * by invariant integers using multiplication", 1994, the round-up variant). */
struct FastDiv {
    uint32_t d, mul, shift;
};

static inline FastDiv make_fastdiv(uint32_t d)
{
    FastDiv f;
    f.d = d;
    uint32_t s = 0;
    while ((1ull << s) < (unsigned long long)d) s++;
    f.shift = s;
    f.mul = (uint32_t)((((1ull << 32) * ((1ull << s) - d)) / d) + 1);
    return f;
}

/* Multiplier tables for jump-ahead: for stream s, lo[s][l] = a^(l-3) mod p
 * (l < 32) and hi[s][h] = a^(32 h - 3) mod p (h < 64), the scaled multipliers
 * of gfr::mwc_mulmod_scaled; two products jump any distance below 2048. */
#define GF_JUMP_HI 64
struct JumpTables {
    uint64_t *lo;                  /* [nstreams][32] */
    uint64_t *hi;                  /* [nstreams][GF_JUMP_HI] */
};

/* One model crawl of one request: everything the CTA of a stream needs. */
struct CrawlJob {
    SkyModel m;
    SkyGeom g;
    CrawlState st;
    uint32_t *rng;                 /* persistent stream state [3][rng_nstreams] */
    int32_t rng_nstreams;
    int32_t pix_base;              /* first pixel of this launch within the generator's pixel list */
    const int64_t *limits;         /* per-stream star limit for this launch (draw) */
    double *counts, *countsCovered;   /* integrate outputs, per stream */
    double *per_pixel;             /* integrate output, per pixel (optional) */
    const float *Dtab;             /* distances D[im][iM] of the model's bins */
    FastDiv fx, fy;                /* division by nm and by nM */
    int32_t job_id;                /* bits 16.. of StarRecord::stream */
    int32_t pad;
    int64_t limit_all;             /* star limit of every stream when limits is null */
};
