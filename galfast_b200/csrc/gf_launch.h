/*
 * gf_launch.h -- launch descriptors of the sm_100a kernels, used by the host
 * orchestration (gf_api.cu).
 */
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "gf_internal.h"

namespace gfk {

struct LaunchCrawl {
    SkyModel m;
    SkyGeom g;
    CrawlState st;
    uint32_t *rng;
    int32_t rng_nstreams;
    JumpTables jt;
    int32_t stream_begin, stream_end;
    const int64_t *limits;
    StarRecord *rec;
    float *rec_am;                 /* GF_EXT_MAPS: anchor extinction per record (parallel to rec), or null */
    int64_t rec_capacity;
    unsigned long long *rec_count;
    unsigned long long *err;
    double *counts, *countsCovered, *per_pixel;
    int32_t pix_base;
    const float *Dtab;
    Checkpoint *ck;                /* draw: checkpoints at the first bin with stars and every ck_every stars */
    uint32_t *ck_count;
    int32_t ck_capacity, ck_every;
    int32_t cw;                    /* draw: warps per stream (1, 2 or 4; 0 = 4) */
};

struct LaunchPlace {
    SkyModel m;
    SkyGeom g;
    const StarRecord *rec;
    const float *rec_am;           /* GF_EXT_MAPS: anchor extinction per record, or null */
    int64_t n;
    double *lb;
    int32_t *projIdx;
    float *projXY, *DM, *absmag, *XYZ, *Am, *AmInf;
    int32_t *hidden;
    uint64_t *key;
    unsigned long long *nvis;
};

struct LaunchSort {
    int64_t n, nvisible;
    uint64_t *key_in, *key_out;
    uint32_t *idx_in, *idx_out;
    void *temp;
    size_t temp_bytes;
    const double *lb;
    const int32_t *projIdx;
    const float *projXY, *DM, *absmag, *XYZ, *Am, *AmInf;
    int32_t comp;
    gf_table out;
};

/* one model pass over many requests: jobs[k] per request, items (job << 16) | stream */
struct LaunchCrawlMulti {
    const CrawlJob *jobs;          /* device */
    const uint32_t *items;         /* device, in the order the work queue hands them out */
    int32_t nitems;
    uint32_t *counter;             /* device work-queue counter */
    int32_t model_type;            /* GF_MODEL_* shared by all jobs */
    int32_t max_tab;               /* max over jobs of nm + nM */
    JumpTables jt;
    StarRecord *rec;
    int64_t rec_capacity;
    unsigned long long *rec_count, *err;
    int32_t cw;                    /* draw: warps per stream (1, 2 or 4; 0 = 4) */
};

struct LaunchPlaceMulti {
    const CrawlJob *jobs;
    const int32_t *job_slot;       /* output position of each request */
    const StarRecord *rec;
    int64_t n;
    uint64_t *key, *key_b;         /* sort keys, before and after the sort */
    uint32_t *idx_a, *idx_b;       /* record index after and before the sort */
    int slot_bits;             /* bits of the output slot at the top of the sort key */
    void *temp;
    size_t temp_bytes;
    int64_t *seg_begin, *vis_end, *seg_end;     /* per slot, preset to zero by the caller */
};

int sm_count();
/* set the message returned by gf_last_error() on this thread */
void set_last_error(const std::string &msg);
/* count of kernel launches issued by the library (for the benchmark's launch census) */
void count_launches(int n);
long long launches();
cudaError_t launch_crawl(const LaunchCrawl &L, int draw, cudaStream_t s);
cudaError_t launch_place(const LaunchPlace &L, cudaStream_t s);
cudaError_t sort_temp_bytes(int64_t n, size_t *bytes);
cudaError_t launch_sort_gather(const LaunchSort &L, cudaStream_t s);
cudaError_t launch_dtab(const SkyModel &m, float *D, cudaStream_t s);
cudaError_t launch_jump_tables(const uint32_t *mult, int n, uint64_t *lo, uint64_t *hi, cudaStream_t s);
cudaError_t launch_seed_streams(const uint32_t *seeds, int njobs, const uint32_t *mult, int NS, uint32_t *rng, cudaStream_t s);
cudaError_t launch_crawl_multi(const LaunchCrawlMulti &L, int draw, cudaStream_t s);
cudaError_t sort_temp_bytes_multi(int64_t n, size_t *bytes);
cudaError_t launch_place_sort_multi(const LaunchPlaceMulti &L, cudaStream_t s);
cudaError_t launch_tie_place_multi(const LaunchPlaceMulti &L, const int64_t *row_begin, const int32_t *slot_comp,
                                    gf_table out, int32_t *row_slot, cudaStream_t s);

/* modules (gf_modules.cu) */
cudaError_t launch_clipper(const gf_footprint &foot, gf_table t, int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_poisson_stream(uint32_t *st, const float *mu, int32_t n, uint32_t *out, cudaStream_t s);
/* os_FeH (fp) or os_GaussianFeH (gp): the one that is not NULL */
cudaError_t launch_feh(const gf_feh_config *fp, const gf_gaussfeh_config *gp, uint32_t *rng, int32_t NS, gf_table t,
                       int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_fixedfeh(const gf_fixedfeh_config &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_bond2010(const gf_bond2010_config &c, uint32_t *rng, int32_t rng_nstreams, gf_table t,
                            int64_t begin, int64_t end, cudaStream_t s);
struct PhotTables {
    int32_t nbands, bidx, nFeH, nMr;
    float reddening[GF_MAX_BANDS];
    float tcFeH[2], tcMr[2];
    const float *colors;          /* device */
    const uint8_t *eflags;        /* device */
    uint32_t comp_mask;
};
cudaError_t launch_photometry(const PhotTables &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_multiples(const gf_multiples_config &c, uint32_t *rng, int32_t NS, gf_table t, int64_t begin, int64_t end,
                             cudaStream_t s);
struct PerrTables {
    int32_t nbands, nknots;
    const double *mag, *sigma;    /* device */
    uint64_t seed;
    /* Bracket guide of strictly increasing knots (null otherwise): the magnitude axis
     * of band b is cut into nguide equal cells, cell(x) = floor((x - gx0[b]) * ginv[b])
     * clamped to [0, nguide), and guide[b * nguide + g] is the last knot index
     * (<= nknots - 2) whose own cell is before g, or 0.  A lookup starts there and
     * steps forward to the bisection's bracket. */
    const int32_t *guide;
    int32_t nguide;
    double gx0[GF_MAX_BANDS], ginv[GF_MAX_BANDS];
};
/* the cell of the bracket guide (host and device evaluate it alike) */
__host__ __device__ inline int perr_cell(double x, double x0, double inv, int n)
{
    const double t = (x - x0) * inv;
    return t < 0.0 ? 0 : (t >= (double)n ? n - 1 : (int)t);
}
cudaError_t launch_photoerrors(const PerrTables &c, int64_t row_offset, gf_table t, int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_vel2pm(const gf_vel2pm_config &c, gf_table t, int64_t begin, int64_t end, cudaStream_t s);
cudaError_t launch_gal2other(int32_t coordsys, gf_table t, int64_t begin, int64_t end, cudaStream_t s);

cudaError_t launch_precision(const SkyModel &m, const SkyGeom &g, const float *Dtab, double *pix32, double *pix64,
                             double *hist64, unsigned long long *max_rel, double *sum_rel, unsigned long long *nbins,
                             cudaStream_t s);

/* expected counts pixel by pixel (gf_integrate.cu) */
/* Anchor plan of one magnitude grid (nm x nM, nm * nM a multiple of 10), one
 * device buffer: this header, then
 *   int2     diag[nd]        per diagonal: first anchor ordinal, first block start after its first bin
 *   float    slotD[]         distance of every slot (distinct anchor distance of a diagonal)
 *   uint16_t anc[]           slot of every anchor, diagonal by diagonal
 *   uint32_t blk[nblocks]    per block of 10 bins (local index 10 b): i | j << 16 of its first bin
 *   uint16_t bslot[nblocks]  slot of the block-start anchor
 *   uint16_t dslot[nd]       slot of each diagonal's first bin
 *   uint32_t binfo[nblocks]  per block: largest apparent-magnitude row im of its bins (bits 0-15)
 *                            and which of its bins 1..9 start a diagonal (bits 16-25) */
struct IntegPlanHdr {
    int32_t nd, nanchors, nslots, ok;      /* ok = 0: the plan did not fit its buffer */
    int32_t off_slot, off_anc;             /* byte offsets of the tables */
    int32_t max_anchors, max_slots;
    int32_t off_blk, off_bslot, off_dslot, nblocks;
    int32_t bytes;                         /* size of the plan buffer */
    int32_t off_binfo;                     /* uint32_t binfo[nblocks]: largest m row of the block | diagonal starts << 16 */
    int32_t pad[2];
};
struct IntegPlanDesc {
    const float *Dtab;             /* D[im][iM], rows of nM_tab */
    int32_t nm, nM, nM_tab;
    int32_t max_anchors, max_slots;
    unsigned char *plan;           /* integ_plan_bytes(nm, nM) bytes */
};
struct IntegPixParams {
    const CrawlJob *jobs;          /* per request: model, geometry (pixels, extinction) */
    const unsigned char *const *plans;   /* per request: plan of its grid, or null (request skipped) */
    const int32_t *pix_off;        /* [njobs + 1] first flat pixel of each request */
    int32_t njobs, total_pix;
    double2 *pix_sum;              /* [total_pix] (expected, expected covered) */
    int32_t off_lf, off_mr, off_q, warp_bytes;   /* per-warp shared-memory layout (integ_warp_bytes) */
    uint32_t *next;                /* device counter of the pixel runs handed out (reset by the launch) */
};
size_t integ_plan_bytes(int nm, int nM, int *max_anchors, int *max_slots);
cudaError_t launch_integ_plans(const IntegPlanDesc *desc_dev, int nplans, cudaStream_t s);
size_t integ_warp_bytes(int nm_max, int nM_max, int slots_max, IntegPixParams *P);
/* per-pixel sums into P.pix_sum, then per-request totals into tot[njobs] */
cudaError_t launch_integrate_pixels(const IntegPixParams &P, int model_type, double2 *tot, cudaStream_t s);

/* the batched draw (gf_batchdraw.cu) */
struct SlotDensityParams {
    const CrawlJob *jobs;
    const unsigned char *const *plans;   /* per request */
    float2 *const *ms;             /* per request, per pixel, nslots + 1 pairs: (model density, D^3) of each
                                    * slot, then (first cut apparent-magnitude row as int bits, K = dA POGSON dm dM) */
    const int32_t *job_list;       /* requests of the launch */
    const int32_t *pix_off;        /* [njobs + 1] first flat pixel of each listed request */
    int32_t njobs, total_pix;
};
struct BlockLfParams {
    const CrawlJob *jobs;
    const unsigned char *const *plans;   /* per request */
    uint4 *const *brec;            /* per request, per block: blk, binfo, bslot | first diagonal-start slot << 16,
                                    * largest LF value of its bins (float bits, at least 0) */
    const int32_t *job_list;       /* requests of the launch */
    const int64_t *blk_off;        /* [njobs + 1] first flat block of each listed request */
    int32_t njobs;
    int64_t total;
};
struct BatchDrawParams {
    const CrawlJob *jobs;
    const unsigned char *const *plans;   /* per request */
    const float2 *const *ms;       /* per request: slot densities (SlotDensityParams::ms) */
    const uint4 *const *brec;      /* per request: block records (null: exact test for every bin) */
    const uint32_t *items;         /* (request << 16) | first of 32 consecutive streams */
    int32_t nitems;
    uint32_t *next_item;           /* work-queue counter */
    EventRecord *ev;
    int64_t ev_capacity;
    unsigned long long *ev_count;  /* events found (may exceed the capacity) */
    unsigned long long *err;       /* set when a bin's expected count is infinite */
    int32_t off_view, off_tab, off_ev, warp_bytes;   /* per-warp shared-memory layout (batch_draw_warp_bytes) */
};
cudaError_t launch_slot_density(const SlotDensityParams &P, int model_type, cudaStream_t s);
cudaError_t launch_block_records(const BlockLfParams &P, cudaStream_t s);
size_t batch_draw_warp_bytes(int max_tab, BatchDrawParams *P);
/* bound: every request of P takes the block bound of its expected counts (see
 * batch_draw_kernel); otherwise every bin is tested exactly */
cudaError_t launch_batch_draw(const BatchDrawParams &P, int model_type, int warps_per_cta, bool bound, cudaStream_t s);
cudaError_t expand_temp_bytes(int64_t nev, size_t *bytes);
/* star records of the events at offsets from a scan over k; *total = the stars of all events */
cudaError_t launch_expand_events(const EventRecord *ev, int64_t nev, const CrawlJob *jobs, int64_t *k64, int64_t *off64,
                                 void *temp, size_t temp_bytes, StarRecord *rec, int64_t rec_capacity, int64_t *total,
                                 cudaStream_t s);

/* module kernels over the rows of many requests (row_slot: the request slot of each row) */
struct MultiRows {
    const int32_t *row_slot;       /* [rows] */
    const int64_t *slot_row_begin; /* [nslots] first row of each slot */
    const int32_t *slot_job;       /* [nslots] request index of each slot */
};
cudaError_t launch_clipper_multi(const gf_footprint *foot_by_job, MultiRows R, gf_table t, int64_t begin, int64_t end,
                                 cudaStream_t s);
cudaError_t launch_bond2010_multi(const gf_bond2010_config &c, uint32_t *rng_all, int32_t NS, MultiRows R,
                                  const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks,
                                  const int64_t *slot_rows, gf_table t, cudaStream_t s);
cudaError_t launch_feh_multi(const gf_feh_config *fp, const gf_gaussfeh_config *gp, uint32_t *rng_all, int32_t NS,
                             MultiRows R, const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks,
                             const int64_t *slot_rows, gf_table t, cudaStream_t s);
cudaError_t launch_multiples_multi(const gf_multiples_config &c, uint32_t *rng_all, int32_t NS, MultiRows R,
                                   const int64_t *slot_chunk_begin, int32_t nslots, int64_t nchunks, const int64_t *slot_rows,
                                   gf_table t, cudaStream_t s);
cudaError_t launch_photoerrors_multi(const PerrTables &c, const uint64_t *seed_by_job, const int64_t *catalog_offset_by_job,
                                     MultiRows R, gf_table t, int64_t begin, int64_t end, cudaStream_t s);

}  // namespace gfk
