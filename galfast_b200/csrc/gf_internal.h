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
};

/* Sky geometry shared by all models of a generator. */
struct SkyGeom {
    const gf_pencil_beam *pixels;  /* device */
    int32_t npixels;
    const float *ammin;            /* device, per-beam minimum extinction, or null */
    int32_t ext_kind;
    float A0;
    gf_lambert proj[2];
};

/* A star drawn by the crawl, to be placed by the star kernel. */
struct StarRecord {
    int32_t stream;
    int32_t ilb;                   /* pixel */
    int16_t im, iM;                /* bin */
    float AmMin;                   /* beam extinction at the bin's anchor */
    float u[4];                    /* uniforms x, y, M, m (u[2..3] = 0 if hidden by x^2+y^2>2) */
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
    float *D, *Am, *ms;            /* anchor of the last processed bin */
    int64_t *nstars;               /* stars drawn by the stream in the current batch */
};

/* Multiplier tables for jump-ahead: for stream s, lane l holds
 * a^(l-3) mod p and a^(32 l - 3) mod p (scaled multipliers of gfr::mwc_mulmod_scaled). */
struct JumpTables {
    uint64_t *lo;                  /* [nstreams][32] */
    uint64_t *hi;                  /* [nstreams][32] */
};
