/*
 * gf_skygen.cu -- sm_100a kernels of the skygen hot path.
 *
 *   crawl_kernel<DRAW>   integrate pass (DRAW = 0) and Poisson draw pass (DRAW = 1)
 *                        of skygenGPU<T>::kernel (src/skygen/skygen.cu.h:469-618)
 *   place_kernel         per-star placement of draw_stars (skygen.cu.h:366-457)
 *   batch sort           star_comp ordering and truncation (skyconfig_impl.h:34-68, 467-515)
 *
 * Parallel layout.  The reference runs one thread per RNG stream; each stream
 * crawls blocks of 10 consecutive diagonal bins, jumping 10*nthreads bins
 * ahead between blocks.  Here one CTA of 4 warps owns one stream and thread L
 * owns block j+L of it, a window of 128 blocks (1280 bins):
 *   pass 1  each thread lists the anchor bins of its block (block start and
 *           diagonal starts); the warp evaluates them compacted, one anchor
 *           per lane (distance, extinction, model density: the expensive part);
 *   pass 2  each thread computes the expected count mu of its 10 bins from
 *           the anchors and two per-model shared-memory tables (LF at each
 *           absolute-magnitude row, m at each apparent-magnitude row);
 *   phase B only the uniforms are sequential: the MWC stream is a Lehmer
 *           generator modulo its safe prime, so thread L jumps directly to the
 *           uniform its first bin would consume if every earlier bin drew zero
 *           stars (two 128-bit modular multiplications) and walks its block with
 *           plain MWC steps.  The first thread that finds a bin with stars
 *           (u > exp(-mu), or mu > 10) hands the bin to its warp, which runs the
 *           reference's Poisson sampler and star draws, and the window restarts
 *           right after it.
 * Results are bin-for-bin and draw-for-draw those of the reference CPU path.
 */
#include "gf_crawl.cuh"
#include "gf_rng.h"
#include <cub/cub.cuh>
#include <atomic>

namespace gfk {

struct CrawlParams {
    CrawlJob job0;                 /* the job of a single-request launch */
    const CrawlJob *jobs;          /* multi-request launch: device job table, or null */
    const uint32_t *items;         /* multi-request launch: (job << 16) | stream per CTA item */
    int32_t nitems;                /* streams (CTA items) in the launch */
    int32_t stream_begin;          /* single-request launch: stream of item 0 */
    JumpTables jt;
    StarRecord *rec;
    float *rec_am;                 /* GF_EXT_MAPS: the anchor extinction of each record (parallel to rec), or null */
    int64_t rec_capacity;
    unsigned long long *rec_count;
    unsigned long long *err;       /* set when a bin's expected count is infinite */
    Checkpoint *ck;                /* draw: checkpoint buffer, or null */
    uint32_t *ck_count;
    int32_t ck_capacity, ck_every;
    uint32_t *next_item;           /* persistent launch: work-queue counter (items taken in order), or null */
};

/* CW (a template parameter of the crawl): warps per stream; a window holds CW * 32
 * blocks of the stream, one per thread.  1, 2 or 4, picked by the autotuner. */
#define FULLMASK 0xffffffffu

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src)
{
    uint32_t lo = __shfl_sync(FULLMASK, (uint32_t)v, src);
    uint32_t hi = __shfl_sync(FULLMASK, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ int warp_incl_scan(int v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(FULLMASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

/* One MWC step on the combined state v = c*2^32 + x. */
__device__ __forceinline__ float mwc_step(uint64_t &v, uint32_t a)
{
    uint64_t t = (uint64_t)a * (uint32_t)v + (v >> 32);
    v = t;
    return GF_MWC_SCALE * (float)(uint32_t)t;
}

/* v * a^n mod p for 0 <= n < 2048 from the stream's scaled powers
 * lo[l] = a^(l-3) and hi[h] = a^(32 h - 3) (L1-resident, 768 bytes per stream). */
__device__ __forceinline__ uint64_t jump(uint64_t v, int n, const uint64_t *lo, const uint64_t *hi, uint32_t a)
{
    const uint64_t p = ((uint64_t)a << 32) - 1;
    const uint64_t w = gfr::mwc_mulmod_scaled(__ldg(lo + (n & 31)), v, a, p);
    return gfr::mwc_mulmod_scaled(__ldg(hi + (n >> 5)), w, a, p);
}

/* Lower bound of expf(-mu) used to accept "no star" without evaluating expf:
 * exp(-mu) >= 1 - mu, and the portable expf is within one ulp of exp. */
__device__ __forceinline__ bool surely_empty(float u, float mu)
{
    return u <= (1.0f - mu) - 3.0e-7f;
}

/* The bin at position s of the block starting at local index k0 in pixel ilb0,
 * by following advance() from the block start (skygen.cu.h:307-358).  Also
 * returns the last anchor bin at or after position s_from (-1 if none). */
struct BinPos {
    int ilb, im, iM;
    int anchor_s;
};

__device__ BinPos bin_at(int ilb0, int k0, int s, int s_from, int x, int y)
{
    BinPos r;
    int i, j;
    gfc::diag_to_ij(k0, x, y, i, j);
    int ilb = ilb0;
    int anc = (s_from <= 0) ? 0 : -1;
    for (int q = 1; q <= s; q++) {
        bool inc;
        bool mv = gfc::advance(i, j, x, y, inc);
        if (inc) ilb++;
        if (mv && q >= s_from) anc = q;
    }
    r.ilb = ilb; r.im = i; r.iM = j; r.anchor_s = anc;
    return r;
}

/* Crawl cursor of one stream, identical in every thread of its CTA. */
struct Cursor {
    int blk_ilb, blk_k, pos;
    int ndraw;
    int cur_ilb, cur_im, cur_iM;
    AnchorX anc;
};

#define GF_RECBUF 64               /* star records staged in shared memory per stream */

template <int DRAW, int CW>
struct CrawlSmem {
    CrawlJob job;
    float4 slot[(CW * 32) * GF_BLOCK];           /* anchor inputs (pixel, i<<16|j), then AnchorX; thread L owns [10L, 10L+10) */
    uint16_t dense[(CW * 32) * GF_BLOCK];        /* compacted list of the window's anchor slots */
    float mu[DRAW ? CW : 1][GF_BLOCK][32]; /* mu of bin s of each thread's block */
    StarRecord recbuf[DRAW ? GF_RECBUF : 1];
    float ambuf[DRAW ? GF_RECBUF : 1];
    int nrec;
    int wtot[CW];
    int wev[CW];
    int scan[CW];
    unsigned long long v_end;
    /* stream state shared by the CTA; written by one thread between barriers */
    Cursor cur;
    unsigned long long v;
    unsigned long long mult;       /* scaled a^(k-1) after a bin with stars that drew k uniforms */
    long long nstars, limit;
    int next_ck, flag, fL, es;
    double red[2][CW];
};

/* Write the staged star records to the global buffer (one warp, all lanes). */
template <int DRAW, int CW>
__device__ void flush_records(const CrawlParams &P, CrawlSmem<DRAW, CW> &S, int lane)
{
    __syncwarp();
    const int n = S.nrec;
    if (n == 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(P.rec_count, (unsigned long long)n);
    base = __shfl_sync(FULLMASK, base, 0);
    for (int q = lane; q < n; q += 32) {
        const unsigned long long slot = base + q;
        if (slot < (unsigned long long)P.rec_capacity) {
            P.rec[slot] = S.recbuf[q];
            if (P.rec_am) P.rec_am[slot] = S.ambuf[q];
        }
    }
    __syncwarp();
    if (lane == 0) S.nrec = 0;
    __syncwarp();
}

/* Draw up to ndraw stars of the bin (ilb, im, iM) while the stream is under its
 * limit (draw_stars, skygen.cu.h:366-457); the uniforms are staged as star
 * records for the placement kernel.  Executed identically by all lanes of one
 * warp; lane 0 writes. */
template <int DRAW, int CW>
__device__ void draw_stars(const CrawlParams &P, CrawlSmem<DRAW, CW> &S, int sid, int lane, gfr::Mwc &r, int &ndraw,
                           long long &nstars, long long limit, int ilb, int im, int iM, float am)
{
    if (!ndraw) return;
    const CrawlJob &J = S.job;
    long long room = limit - nstars;
    int todo = (int)(room < (long long)ndraw ? (room > 0 ? room : 0) : ndraw);
    if (todo <= 0) return;
    const gf_pencil_beam pix = J.g.pixels[ilb];
    for (int n = 0; n < todo; n++) {
        StarRecord rec;
        rec.stream = sid;
        rec.ilb = ilb + J.pix_base;
        rec.im = (short)im;
        rec.iM = (short)iM;
        rec.seq = (int32_t)(nstars + n);
        rec.u[0] = r.uniform();
        rec.u[1] = r.uniform();
        float x = pix.X, y = pix.Y;
        x += pix.dx * (rec.u[0] - 0.5f);
        y += pix.dx * (rec.u[1] - 0.5f);
        if (x * x + y * y > 2.f) {
            rec.u[2] = rec.u[3] = 0.f;
        } else {
            rec.u[2] = r.uniform();
            rec.u[3] = r.uniform();
        }
        __syncwarp();
        const int k = S.nrec;
        __syncwarp();
        if (lane == 0) { S.recbuf[k] = rec; S.ambuf[k] = am; S.nrec = k + 1; }
        if (k + 1 == GF_RECBUF) flush_records(P, S, lane);
    }
    nstars += todo;
    ndraw -= todo;
}

__device__ __forceinline__ AnchorX ax_from(const float4 t) { AnchorX a; a.Am = t.x; a.ms = t.y; a.D3 = t.z; a.K = t.w; return a; }

template <int MODEL>
__device__ __noinline__ AnchorX anchor_cold(const SkyModel &m, const SkyGeom &g, const float *Dtab, int ilb, int im, int iM)
{
    return gfc::anchor_x<MODEL>(m, g, Dtab, ilb, im, iM);
}

/* Non-surely-empty bins: the exact test of the reference's sampler, u > exp(-mu)
 * or mu > 10 (the branch that does not compare with exp(-mu) at all). */
__device__ __noinline__ bool has_stars(float u, float mu)
{
    return mu > 10.f || gfr::exceeds_exp_neg(u, mu);
}

/* A bin with stars found by phase B: thread fL = 32 fw + fl of the CTA, bin es of
 * its block.  Runs the reference's Poisson sampler and star draws for it on the
 * calling warp (all lanes, identical control flow), records a checkpoint when
 * one is due, and leaves the outcome in S (flag 0: continue, 1: the stream
 * reached its limit and pauses after the bin, 2: stop on an infinite expected
 * count).  For a block inside one pixel the bin and its anchor are found by
 * stepping from the block start and reading the window's anchor slots. */
template <int DRAW, int MODEL, int CW>
__device__ __noinline__ void handle_event(const CrawlParams &P, CrawlSmem<DRAW, CW> &S, int sid, int lane, int fL, int es,
                                          uint64_t vb, float emu, int f_ilb, int f_k, int f_i0, int f_j0, bool f_fast,
                                          uint32_t a, const uint64_t *jlo, const uint64_t *jhi)
{
    const CrawlJob &J = S.job;
    const SkyModel &m = J.m;
    const int x = m.nm, y = m.nM;
    const int f_sbeg = (fL == 0) ? S.cur.pos : 0;
    int e_ilb, e_im, e_iM;
    AnchorX anc_es = S.cur.anc;
    if (f_fast) {
        int ci = f_i0, cj = f_j0, n = (f_sbeg == 0) ? 0 : -1;
        for (int s = 1; s <= es; s++) {
            if (gfc::step_in_pixel(ci, cj, x, y) && s >= f_sbeg) n++;
        }
        e_ilb = f_ilb; e_im = ci; e_iM = cj;
        if (n >= 0) anc_es = ax_from(S.slot[fL * GF_BLOCK + n]);
    } else {
        const BinPos eb = bin_at(f_ilb, f_k, es, f_sbeg, x, y);
        e_ilb = eb.ilb; e_im = eb.im; e_iM = eb.iM;
        if (eb.anchor_s >= 0) {
            const BinPos ab = bin_at(f_ilb, f_k, eb.anchor_s, 0, x, y);
            anc_es = anchor_cold<MODEL>(m, J.g, J.Dtab, ab.ilb, ab.im, ab.iM);
        }
    }
    int flag = 0, nd = 0;
    long long ns = S.nstars;
    int nck = S.next_ck;
    uint64_t vnew = vb;
    if (!(emu < 3.0e38f)) {
        /* an infinite expected count would never leave the sampler's gamma loop */
        if (lane == 0) atomicOr(P.err, 1ull);
        flag = 2;
    } else {
        if (P.ck && ns >= nck) {
            if (lane == 0) {
                const uint32_t slot = atomicAdd(P.ck_count, 1u);
                if (slot < (uint32_t)P.ck_capacity) {
                    Checkpoint ck;
                    ck.stream = sid; ck.nstars = (int32_t)ns;
                    ck.blk_ilb = f_ilb; ck.blk_k = f_k; ck.pos = es; ck.pad = 0;
                    ck.anc = anc_es; ck.v = vb;
                    P.ck[slot] = ck;
                }
            }
            nck = (int)ns + P.ck_every;
        }
        gfr::Mwc r;
        r.a = a;
        r.set_v(vb);
        r.used = 0;
        nd = (int)r.poisson(emu);
        draw_stars<DRAW, CW>(P, S, sid, lane, r, nd, ns, S.limit, e_ilb, e_im, e_iM, anc_es.Am);
        vnew = r.v();
        if (nd) flag = 1;             /* the stream reached its limit: pause right after the bin */
        /* The walk assumed one uniform for this bin; it drew r.used >= 1.  Every later
         * bin's start state moves by a^(used-1): the scaled multiplier of that power. */
        const uint64_t p = ((uint64_t)a << 32) - 1;
        uint32_t n = r.used - 1;
        uint64_t ms = __ldg(jlo);                                 /* scaled a^0 */
        if (n >= 2048) {
            const uint64_t m2047 = gfr::mwc_mulmod_scaled(__ldg(jlo + 31), __ldg(jhi + 63), a, p);
            while (n >= 2047) { ms = gfr::mwc_mulmod_scaled(ms, m2047, a, p); n -= 2047; }
        }
        ms = gfr::mwc_mulmod_scaled(ms, gfr::mwc_mulmod_scaled(__ldg(jlo + (n & 31)), __ldg(jhi + (n >> 5)), a, p), a, p);
        if (lane == 0) S.mult = ms;
    }
    __syncwarp();
    if (lane == 0) {
        S.v = vnew; S.nstars = ns; S.flag = flag; S.fL = fL; S.es = es; S.next_ck = nck;
        S.cur.ndraw = nd; S.cur.cur_ilb = e_ilb; S.cur.cur_im = e_im; S.cur.cur_iM = e_iM;
        if (flag == 1) {
            S.cur.blk_ilb = f_ilb; S.cur.blk_k = f_k; S.cur.pos = es + 1;
            S.cur.anc = anc_es;
        }
    }
    __syncwarp();
}

/* Finish the draw that did not complete before the previous batch filled
 * (skygen.cu.h:497-502); warp 0. */
template <int DRAW, int CW>
__device__ __noinline__ void finish_pending(const CrawlParams &P, CrawlSmem<DRAW, CW> &S, int sid, int lane, uint32_t a)
{
    gfr::Mwc r;
    r.a = a;
    r.set_v(S.v);
    int nd = S.cur.ndraw;
    long long ns = S.nstars;
    draw_stars<DRAW, CW>(P, S, sid, lane, r, nd, ns, S.limit, S.cur.cur_ilb, S.cur.cur_im, S.cur.cur_iM, S.cur.anc.Am);
    __syncwarp();
    if (lane == 0) { S.v = r.v(); S.nstars = ns; S.cur.ndraw = nd; S.next_ck = (int)ns; }
    __syncwarp();
}

/* A block that runs past the end of its pixel (possible only when nm*nM is not
 * a multiple of 10): follow advance() bin by bin with the anchors inline.
 * Returns whether the crawl left the last pixel inside the block. */
template <int DRAW, int MODEL, int CW>
__device__ __noinline__ bool slow_block(CrawlSmem<DRAW, CW> &S, const float *LFM, const float *MMr, int L, int i0, int j0,
                                        int my_ilb, int s_begin, uint32_t &live, double &cnt_sum, double &cov_sum)
{
    const CrawlJob &J = S.job;
    const SkyModel &m = J.m;
    const int x = m.nm, y = m.nM, npix = J.g.npixels;
    int i = i0, j = j0, ilb = my_ilb;
    bool dd = false, ended = false;
    AnchorX A = S.cur.anc;
    float cf = 0.f;
    for (int s = 0; s < GF_BLOCK; s++) {
        bool moved = true;
        if (s > 0 && !dd) {
            bool pinc;
            moved = gfc::advance(i, j, x, y, pinc);
            if (pinc) ilb++;
            if (moved && ilb >= npix) dd = true;
        }
        if (dd) ended = true;
        float mus = gfc::cut_marker();
        if (!dd && s >= s_begin) {
            if (moved) {
                A = gfc::anchor_x<MODEL>(m, J.g, J.Dtab, ilb, i, j);
                if (!DRAW) cf = J.g.pixels[ilb].coveredFraction;
            }
            /* i (and j) can leave the grid after a pixel change: see bin_distance */
            const float lfv = ((unsigned)j < (unsigned)y) ? LFM[j] : gfc::lf_sample(m, m.lf, m.M1 - (float)j * m.dM);
            const float mrow = ((unsigned)i < (unsigned)x) ? MMr[i] : m.m0 + m.dm * (float)i;
            mus = gfc::bin_mu_x(A, lfv, mrow, m.norm, m.m1);
        }
        const bool ok = !gfc::is_cut(mus);
        if (DRAW) {
            S.mu[L >> 5][s][L & 31] = mus;
            live |= ok ? (1u << s) : 0u;
        } else if (ok) {
            cnt_sum += (double)mus;
            const double cv = (double)(mus * cf);
            cov_sum += cv;
            if (J.per_pixel) atomicAdd(&J.per_pixel[ilb + J.pix_base], cv);
        }
    }
    return ended;
}

/* Crawl of one stream by one CTA (integrate when DRAW = 0, Poisson draw when
 * DRAW = 1).  Thread L of the CTA owns block j+L of the stream's window. */
template <int DRAW, int MODEL, int CW>
__device__ void crawl_item(const CrawlParams &P, CrawlSmem<DRAW, CW> &S, const float *LFM, const float *MMr, int tid)
{
    const CrawlJob &J = S.job;
    const SkyModel &m = J.m;
    const int L = threadIdx.x, warp = L >> 5, lane = L & 31;
    const int x = m.nm, y = m.nM, kmax = x * y;
    const int npix = J.g.npixels;
    const float norm = m.norm, m1 = m.m1;
    const CrawlState &st = J.st;
    const long long step = (long long)GF_BLOCK * m.nthreads;
    const long long offL = (long long)L * step;
    const int qL = (int)(offL / kmax), rL = (int)(offL % kmax);
    const long long offW = (long long)(CW * 32) * step;
    const int QW = (int)(offW / kmax), RW = (int)(offW % kmax);
    const int sid = (J.job_id << 16) | tid;

    const int status = DRAW ? st.status[tid] : 0;
    if (status == 2) return;
    if (L == 0) {
        Cursor &c = S.cur;
        if (status == 0) {
            long long k = (long long)GF_BLOCK * tid;
            c.blk_ilb = (int)(k / kmax);
            c.blk_k = (int)(k % kmax);
            c.pos = 0;
            c.ndraw = 0;
            c.cur_ilb = c.cur_im = c.cur_iM = 0;
            c.anc.Am = c.anc.ms = c.anc.D3 = c.anc.K = 0.f;
        } else {
            c.blk_ilb = st.blk_ilb[tid]; c.blk_k = st.blk_k[tid]; c.pos = st.pos[tid];
            c.ndraw = st.ndraw[tid];
            c.cur_ilb = st.cur_ilb[tid]; c.cur_im = st.cur_im[tid]; c.cur_iM = st.cur_iM[tid];
            c.anc = st.anc[tid];
        }
        if (DRAW) {
            const int NS = J.rng_nstreams;
            S.v = ((uint64_t)J.rng[NS + tid] << 32) | J.rng[2 * NS + tid];
            S.nstars = st.nstars[tid];
            S.limit = J.limits ? J.limits[tid] : J.limit_all;
            S.next_ck = (int)S.nstars;
            S.nrec = 0;
        }
    }
    __syncthreads();

    uint32_t a = 0;
    uint64_t v = 0;
    const uint64_t *jlo = nullptr, *jhi = nullptr;
    if (DRAW) {
        a = J.rng[tid];
        jlo = P.jt.lo + (size_t)tid * 32;
        jhi = P.jt.hi + (size_t)tid * GF_JUMP_HI;
        if (S.cur.ndraw) {
            if (warp == 0) finish_pending<DRAW, CW>(P, S, sid, lane, a);
            __syncthreads();
        }
        v = S.v;
    }
    int blk_ilb = S.cur.blk_ilb, blk_k = S.cur.blk_k, pos = S.cur.pos;

    double cnt_sum = 0.0, cov_sum = 0.0;
    bool finished = false;

    while (!(DRAW && S.cur.ndraw)) {
        /* ---------- the window: block j+L of the stream for thread L ---------- */
        int my_k = blk_k + rL, my_q = qL;
        if (my_k >= kmax) { my_k -= kmax; my_q++; }
        const bool fast = my_k + GF_BLOCK - 1 < kmax;
        const int drift = fast ? 0 : gfc::block_drift(my_k, x, y);
        int dexcl = 0, dtot = 0;
        if (__syncthreads_or(drift != 0)) {
            const int inc = warp_incl_scan(drift, lane);
            if (lane == 31) S.scan[warp] = inc;
            __syncthreads();
            int woff = 0;
            for (int q = 0; q < CW; q++) {
                const int t = S.scan[q];
                woff += (q < warp) ? t : 0;
                dtot += t;
            }
            dexcl = woff + inc - drift;
            __syncthreads();
        }
        const long long ilb_ll = (long long)blk_ilb + my_q + dexcl;
        const int my_ilb = ilb_ll > npix ? npix : (int)ilb_ll;
        const int s_begin = (L == 0) ? pos : 0;
        const bool dead0 = my_ilb >= npix;
        bool lane_end = dead0;

        /* ---------- pass 1: anchor bins of the block, evaluated compacted over the CTA ---------- */
        int i0 = 0, j0 = 0;
        if (!dead0) gfc::diag_to_ij_fast(my_k, x, y, J.fx, J.fy, i0, j0);
        const int base = L * GF_BLOCK;
        int na = 0;
        if (!dead0 && fast) {
            int ci = i0, cj = j0, s = 0;
            if (s_begin == 0) {
                S.slot[base] = make_float4(__int_as_float(my_ilb), __int_as_float((ci << 16) | cj), 0.f, 0.f);
                na = 1;
            }
            for (;;) {
                const int rem = min(cj, x - 1 - ci) + 1;     /* bins left on this diagonal */
                s += rem;
                if (s >= GF_BLOCK) break;
                const int d1 = ci + cj + 1;
                ci = max(0, d1 - (y - 1));
                cj = d1 - ci;
                if (s >= s_begin) {
                    S.slot[base + na] = make_float4(__int_as_float(my_ilb), __int_as_float((ci << 16) | cj), 0.f, 0.f);
                    na++;
                }
            }
        }
        {
            const int inc = warp_incl_scan(na, lane);
            if (lane == 31) S.scan[warp] = inc;
            __syncthreads();
            int woff = 0, T = 0;
            for (int q = 0; q < CW; q++) {
                const int t = S.scan[q];
                woff += (q < warp) ? t : 0;
                T += t;
            }
            const int excl = woff + inc - na;
            for (int n = 0; n < na; n++) S.dense[excl + n] = (uint16_t)(base + n);
            __syncthreads();
            for (int d = L; d < T; d += (CW * 32)) {
                const int sl = S.dense[d];
                const float4 in = S.slot[sl];
                const int ij = __float_as_int(in.y);
                const AnchorX ax = gfc::anchor_x<MODEL>(m, J.g, J.Dtab, __float_as_int(in.x), ij >> 16, ij & 0xffff);
                S.slot[sl] = make_float4(ax.Am, ax.ms, ax.D3, ax.K);
            }
            __syncthreads();
        }

        /* ---------- pass 2: expected count of every bin ---------- */
        uint32_t live = 0;                 /* bins with an expected count (not cut) */
        if (!dead0 && fast) {
            int ci = i0, cj = j0, n = (s_begin == 0) ? 0 : -1;
            AnchorX A = (s_begin == 0) ? ax_from(S.slot[base]) : S.cur.anc;
            const float cf = DRAW ? 0.f : J.g.pixels[my_ilb].coveredFraction;
            double bcov = 0.0;
#pragma unroll
            for (int s = 0; s < GF_BLOCK; s++) {
                if (s > 0) {
                    const bool wrap = gfc::step_in_pixel(ci, cj, x, y);
                    if (wrap && s >= s_begin) { n++; A = ax_from(S.slot[base + n]); }
                }
                float mus = gfc::cut_marker();
                if (s >= s_begin) mus = gfc::bin_mu_x(A, LFM[cj], MMr[ci], norm, m1);
                const bool ok = !gfc::is_cut(mus);
                if (DRAW) {
                    S.mu[warp][s][lane] = mus;
                    live |= ok ? (1u << s) : 0u;
                } else if (ok) {
                    cnt_sum += (double)mus;
                    const double cv = (double)(mus * cf);
                    cov_sum += cv;
                    bcov += cv;
                }
            }
            if (!DRAW && J.per_pixel) atomicAdd(&J.per_pixel[my_ilb + J.pix_base], bcov);
        } else if (!dead0) {
            if (slow_block<DRAW, MODEL, CW>(S, LFM, MMr, L, i0, j0, my_ilb, s_begin, live, cnt_sum, cov_sum)) lane_end = true;
        }
        const int any_end = __syncthreads_or(lane_end);

        if (DRAW) {
            /* ---------- phase B: uniforms, restarted after each bin with stars ---------- */
            /* start state of each thread's first bin, if no bin before it has stars */
            const uint32_t act0 = s_begin >= GF_BLOCK ? 0u : ((live >> s_begin) << s_begin);
            uint32_t act = act0;
            uint64_t wst;
            {
                const int cnt = __popc(act);
                const int inc = warp_incl_scan(cnt, lane);
                if (lane == 31) S.wtot[warp] = inc;
                __syncthreads();
                int woff = 0;
                for (int q = 0; q < CW; q++) woff += (q < warp) ? S.wtot[q] : 0;
                wst = jump(v, woff + inc - cnt, jlo, jhi, a);
            }
            const uint64_t pmod = ((uint64_t)a << 32) - 1;
            for (;;) {
                int ev_s = -1;
                uint64_t w = wst, w_before = 0;
                float ev_mu = 0.f;
                if (act) {
#pragma unroll
                    for (int s = 0; s < GF_BLOCK; s++) {
                        if (ev_s < 0 && ((act >> s) & 1u)) {
                            const float mus = S.mu[warp][s][lane];
                            const uint64_t wb = w;
                            const float u = mwc_step(w, a);
                            if (!surely_empty(u, mus) && has_stars(u, mus)) {
                                ev_s = s;
                                w_before = wb;
                                ev_mu = mus;
                            }
                        }
                    }
                }
                const unsigned evm = __ballot_sync(FULLMASK, ev_s >= 0);
                if (lane == 0) S.wev[warp] = evm ? (__ffs(evm) - 1) : -1;
                if (L == (CW * 32) - 1) S.v_end = w;
                __syncthreads();
                int fw = -1, fl = 0;
                for (int q = 0; q < CW; q++) {
                    const int e = S.wev[q];
                    if (fw < 0 && e >= 0) { fw = q; fl = e; }
                }
                if (fw < 0) {
                    v = S.v_end;
                    break;
                }
                if (warp == fw) {
                    const int es = __shfl_sync(FULLMASK, ev_s, fl);
                    const uint64_t vb = shfl64(w_before, fl);
                    const float emu = __shfl_sync(FULLMASK, ev_mu, fl);
                    const int f_ilb = __shfl_sync(FULLMASK, my_ilb, fl);
                    const int f_k = __shfl_sync(FULLMASK, my_k, fl);
                    const int f_i0 = __shfl_sync(FULLMASK, i0, fl);
                    const int f_j0 = __shfl_sync(FULLMASK, j0, fl);
                    const bool f_fast = __shfl_sync(FULLMASK, fast ? 1 : 0, fl) != 0;
                    handle_event<DRAW, MODEL, CW>(P, S, sid, lane, fw * 32 + fl, es, vb, emu, f_ilb, f_k, f_i0, f_j0, f_fast,
                                              a, jlo, jhi);
                }
                __syncthreads();
                const int flag = S.flag;
                if (flag) {
                    v = S.v;
                    if (flag == 2) finished = true;
                    break;
                }
                /* continue with the bins after the one with stars: the thread that had it
                 * resumes from the state after the draw, later threads shift by a^(used-1) */
                const int fL = fw * 32 + fl;
                if (L < fL) {
                    act = 0u;
                } else if (L == fL) {
                    const int lo = S.es + 1;
                    act = lo >= GF_BLOCK ? 0u : ((live >> lo) << lo);
                    wst = S.v;
                } else {
                    wst = gfr::mwc_mulmod_scaled(S.mult, wst, a, pmod);
                }
            }
            if (finished || S.cur.ndraw) break;
        }
        if (any_end) { finished = true; break; }
        /* next window */
        int nk = blk_k + RW, carry = 0;
        if (nk >= kmax) { nk -= kmax; carry = 1; }
        blk_ilb = blk_ilb + QW + carry + dtot;
        blk_k = nk;
        pos = 0;
        if (L == 0) S.cur.pos = 0;        /* read by the event handler of the next window */
    }

    if (!DRAW) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cnt_sum += __shfl_xor_sync(FULLMASK, cnt_sum, o);
            cov_sum += __shfl_xor_sync(FULLMASK, cov_sum, o);
        }
        if (lane == 0) { S.red[0][warp] = cnt_sum; S.red[1][warp] = cov_sum; }
        __syncthreads();
        if (L == 0) {
            double e = 0.0, ec = 0.0;
            for (int q = 0; q < CW; q++) { e += S.red[0][q]; ec += S.red[1][q]; }
            J.counts[tid] += e;
            J.countsCovered[tid] += ec;
        }
        return;
    }

    __syncthreads();
    if (warp == 0) flush_records<DRAW, CW>(P, S, lane);
    if (L == 0) {
        const Cursor &c = S.cur;
        const bool paused = c.ndraw != 0;
        st.status[tid] = finished ? 2 : 1;
        st.blk_ilb[tid] = paused ? c.blk_ilb : blk_ilb;
        st.blk_k[tid] = paused ? c.blk_k : blk_k;
        st.pos[tid] = paused ? c.pos : pos;
        st.ndraw[tid] = c.ndraw;
        st.cur_ilb[tid] = c.cur_ilb; st.cur_im[tid] = c.cur_im; st.cur_iM[tid] = c.cur_iM;
        st.anc[tid] = c.anc;
        st.nstars[tid] = S.nstars;
        const int NS = J.rng_nstreams;
        J.rng[NS + tid] = (uint32_t)(v >> 32);
        J.rng[2 * NS + tid] = (uint32_t)v;
    }
}

/* Per-model tables in shared memory: LF(M) of every absolute-magnitude row
 * (nearest texel, cux.h:778-792) and m0 + dm*im of every apparent-magnitude row. */
__device__ void fill_tables(const SkyModel &m, float *LFM, float *MMr)
{
    for (int q = threadIdx.x; q < m.nM; q += blockDim.x) LFM[q] = gfc::lf_sample(m, m.lf, m.M1 - (float)q * m.dM);
    for (int q = threadIdx.x; q < m.nm; q += blockDim.x) MMr[q] = m.m0 + m.dm * (float)q;
}

/* next work item of a CTA: a static stride, or the shared queue of a persistent launch */
__device__ __forceinline__ int next_work_item(const CrawlParams &P, int *slot, int it)
{
    if (!P.next_item) return it + gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) *slot = (int)atomicAdd(P.next_item, 1u);
    __syncthreads();
    return *slot;
}

template <int DRAW, int MODEL, int CW>
__global__ void __launch_bounds__(CW * 32, DRAW ? 16 / CW : 24 / CW) crawl_kernel(CrawlParams P)
{
    extern __shared__ float s_tab[];
    __shared__ CrawlSmem<DRAW, CW> S;
    __shared__ int s_item;
    int loaded = -1;
    int it = P.next_item ? next_work_item(P, &s_item, 0) : (int)blockIdx.x;
    for (; it < P.nitems; it = next_work_item(P, &s_item, it)) {
        int job = 0, tid;
        if (P.items) {
            const uint32_t w = P.items[it];
            job = (int)(w >> 16);
            tid = (int)(w & 0xffffu);
        } else {
            tid = P.stream_begin + it;
        }
        if (job != loaded) {
            __syncthreads();
            const int *src = P.jobs ? (const int *)&P.jobs[job] : (const int *)&P.job0;
            for (int q = threadIdx.x; q < (int)(sizeof(CrawlJob) / 4); q += blockDim.x) ((int *)&S.job)[q] = src[q];
            __syncthreads();
            fill_tables(S.job.m, s_tab, s_tab + S.job.m.nM);
            loaded = job;
        }
        __syncthreads();
        crawl_item<DRAW, MODEL, CW>(P, S, s_tab, s_tab + S.job.m.nM, tid);
    }
}

/* D[im][iM] = powf(10, 0.2 DM + 1) with DM = (m0 + im dm) - (M1 - iM dM), skygen.cu.h:219-222 */
__global__ void dtab_kernel(SkyModel m, float *D)
{
    int n = m.nm * m.nM;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        int im = q / m.nM, iM = q - im * m.nM;
        float M = m.M1 - (float)iM * m.dM;
        float mm = m.m0 + (float)im * m.dm;
        float DM = mm - M;
        D[q] = gfm::powf_(10.f, 0.2f * DM + 1.f);
    }
}

/* ------------------------------------------------------------------ */
/* Star placement (draw_stars, skygen.cu.h:376-456)                    */
/* ------------------------------------------------------------------ */
struct PlaceParams {
    SkyModel m;
    SkyGeom g;
    const StarRecord *rec;
    const float *rec_am;    /* GF_EXT_MAPS: the anchor extinction of each record, or null */
    int64_t n;
    /* unsorted columns */
    double *lb;             /* [2][n] */
    int32_t *projIdx;
    float *projXY;          /* [2][n] */
    float *DM, *absmag;
    float *XYZ;             /* [3][n] */
    float *Am, *AmInf;
    int32_t *hidden;
    uint64_t *key;          /* sort key: l bits for visible stars, all ones for hidden */
    unsigned long long *nvis;   /* number of visible stars */
};

__device__ __forceinline__ void deproject(const gf_lambert &p, double &l, double &b, const float x, const float y)
{
    double r2 = (double)(x * x + y * y);
    if (r2 == 0.) { b = p.b0; l = 0.; return; }
    double ir = 1. / sqrt(r2);
    double sc = 1. / ir * sqrt(1. - 0.25 * r2);
    double cc = 1. - 0.5 * r2;
    b = gfm::asin_d(cc * (double)p.sb + (double)y * sc * (double)p.cb * ir);
    l = p.l0 + gfm::atan2_d((double)x * sc, (double)p.cb * cc / ir - (double)(y * p.sb) * sc);
}

/* The placed values of one star record (draw_stars, skygen.cu.h:376-456). */
struct Placed {
    double l, b;            /* degrees */
    float x, y;             /* Lambert coordinates */
    float DM, M;
    float X, Y, Z;
    float Am, AmInf;
    int32_t projIdx;
    int edge;               /* x^2 + y^2 > 2: beyond the projection edge, nothing else is set */
    int vis;                /* visible: not beyond the edge and no fainter than m1 after extinction */
};

/* Placement of one star record (draw_stars, skygen.cu.h:376-456).  am points to
 * the record's anchor extinction (3-D maps) or is null.  Every caller that places
 * the same record gets the same bits: the expressions are evaluated in one order
 * and the device code is compiled without contraction. */
__device__ __forceinline__ void place_values(const SkyModel &m, const SkyGeom &g, const StarRecord &rec, const float *am,
                                             Placed &v)
{
    const double r2d = 57.2957795130823208767981548;
    const gf_pencil_beam pix = g.pixels[rec.ilb];
    float M = m.M1 - (float)rec.iM * m.dM;
    float x = pix.X, y = pix.Y;
    x += pix.dx * (rec.u[0] - 0.5f);
    y += pix.dx * (rec.u[1] - 0.5f);
    v.x = x;
    v.y = y;
    if (x * x + y * y > 2.f) {
        v.edge = 1;
        v.vis = 0;
        v.l = 0.;
        return;
    }
    v.edge = 0;
    v.projIdx = pix.projIdx;
    double l, b;
    deproject(g.proj[pix.projIdx], l, b, x, y);
    float cl = (float)gfm::cos_d(l), cb = (float)gfm::cos_d(b);
    float sl = (float)gfm::sin_d(l), sb = (float)gfm::sin_d(b);
    l *= r2d;
    if (l < 0.) l += 360.;
    if (l > 360.) l -= 360.;
    b *= r2d;
    v.l = l;
    v.b = b;
    float Mtmp = M + m.dM * (rec.u[2] - 0.5f);
    float mtmp = m.m0 + m.dm * ((float)rec.im + rec.u[3] - 0.5f);
    float DM = mtmp - Mtmp;
    v.M = Mtmp;
    v.DM = DM;
    float D = gfm::powf_(10.f, 0.2f * DM + 1.f);
    v.X = D * cl * cb;
    v.Y = D * sl * cb;
    v.Z = D * sb;
    float Am0, AmInf;
    if (g.ext_kind == GF_EXT_MAPS) {
        /* sampleExtinction at the star's DM and at DM = 100 (skygen.cu.h:421-424) */
        Am0 = gfc::map_extinction(g, pix.projIdx, x, y, DM);
        const float Am1 = gfc::map_extinction(g, pix.projIdx, x, y, 100.f);
        AmInf = Am1 > Am0 ? Am1 : Am0;
    } else {
        Am0 = (g.ext_kind == GF_EXT_SCREEN_CSCB) ? g.A0 / fabsf(sb) : 0.f;
        AmInf = Am0;
    }
    v.vis = (mtmp + Am0 > m.m1) ? 0 : 1;
    /* the extinction at the bin's anchor (draw_stars, skygen.cu.h:437-446): carried with
     * the record for 3-D maps (it depends on the anchor's distance), else the beam's */
    const float AmMin = (g.ext_kind == GF_EXT_MAPS && am) ? *am : gfc::beam_extinction(g, pix);
    if (AmMin > Am0) AmInf = -AmMin;
    v.Am = Am0;
    v.AmInf = AmInf;
}

/* Placement of one star record into row i of the unsorted columns; returns
 * whether the star is visible. */
__device__ __forceinline__ int place_one(const SkyModel &m, const SkyGeom &g, const StarRecord &rec, int64_t i, int64_t n,
                                         const PlaceParams &P)
{
    Placed v;
    place_values(m, g, rec, P.rec_am ? P.rec_am + i : nullptr, v);
    if (v.edge) {
        P.hidden[i] = 1;
        P.key[i] = ~0ull;
        return 0;
    }
    P.projIdx[i] = v.projIdx;
    P.projXY[i] = v.x;
    P.projXY[n + i] = v.y;
    P.lb[i] = v.l;
    P.lb[n + i] = v.b;
    P.absmag[i] = v.M;
    P.DM[i] = v.DM;
    P.XYZ[i] = v.X;
    P.XYZ[n + i] = v.Y;
    P.XYZ[2 * n + i] = v.Z;
    P.Am[i] = v.Am;
    P.AmInf[i] = v.AmInf;
    P.hidden[i] = v.vis ? 0 : 1;
    /* l >= 0 here (-0.0 compares equal to 0.0 and maps to key 0) */
    P.key[i] = v.vis ? (v.l == 0.0 ? 0ull : (uint64_t)__double_as_longlong(v.l)) : ~0ull;
    return v.vis;
}

__global__ void __launch_bounds__(256) place_kernel(PlaceParams P)
{
    unsigned vis_local = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += (int64_t)gridDim.x * blockDim.x) {
        const StarRecord rec = P.rec[i];
        vis_local += (unsigned)place_one(P.m, P.g, rec, i, P.n, P);
    }
    /* warp-aggregated count of visible stars */
    for (int o = 16; o > 0; o >>= 1) vis_local += __shfl_xor_sync(0xffffffffu, vis_local, o);
    if ((threadIdx.x & 31) == 0 && vis_local) atomicAdd(P.nvis, (unsigned long long)vis_local);
}

/* Order the runs of equal l by (b, DM, M, Am) (star_comp, skyconfig_impl.h:58-67). */
__global__ void tie_kernel(const uint64_t *key, uint32_t *idx, int64_t n, const double *lb, const float *DM,
                           const float *absmag, const float *Am, int64_t pitch)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i + 1 >= n || key[i] != key[i + 1]) continue;
        if (i > 0 && key[i - 1] == key[i]) continue;     /* not a run start */
        int64_t e = i + 1;
        while (e + 1 < n && key[e + 1] == key[i]) e++;
        /* insertion sort of idx[i..e] */
        for (int64_t q = i + 1; q <= e; q++) {
            uint32_t cur = idx[q];
            int64_t r = q - 1;
            while (r >= i) {
                uint32_t o = idx[r];
                bool less;
                if (lb[pitch + cur] != lb[pitch + o]) less = lb[pitch + cur] < lb[pitch + o];
                else if (DM[cur] != DM[o]) less = DM[cur] < DM[o];
                else if (absmag[cur] != absmag[o]) less = absmag[cur] < absmag[o];
                else less = Am[cur] < Am[o];
                if (!less) break;
                idx[r + 1] = o;
                r--;
            }
            idx[r + 1] = cur;
        }
    }
}

/* Gather the visible stars into the output table in sorted order. */
struct GatherParams {
    const uint32_t *idx;
    int64_t n, src_pitch;
    const double *lb; const int32_t *projIdx; const float *projXY; const float *DM, *absmag, *XYZ, *Am, *AmInf;
    int32_t comp;
    gf_table out;
};

__global__ void __launch_bounds__(256) gather_kernel(GatherParams G)
{
    const int64_t P = G.out.capacity, S = G.src_pitch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < G.n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s = G.idx[i];
        G.out.lb[i] = G.lb[s];
        G.out.lb[P + i] = G.lb[S + s];
        G.out.projIdx[i] = G.projIdx[s];
        G.out.projXY[i] = G.projXY[s];
        G.out.projXY[P + i] = G.projXY[S + s];
        G.out.DM[i] = G.DM[s];
        G.out.absmag[i] = G.absmag[s];
        G.out.XYZ[i] = G.XYZ[s];
        G.out.XYZ[P + i] = G.XYZ[S + s];
        G.out.XYZ[2 * P + i] = G.XYZ[2 * S + s];
        G.out.comp[i] = G.comp;
        G.out.Am[i] = G.Am[s];
        G.out.AmInf[i] = G.AmInf[s];
        G.out.hidden[i] = 0;
    }
}

__global__ void iota_kernel(uint32_t *idx, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        idx[i] = (uint32_t)i;
}

}  // namespace gfk

/* ------------------------------------------------------------------ */
/* launch wrappers used by the host orchestration                      */
/* ------------------------------------------------------------------ */
#include "gf_launch.h"

namespace gfk {

static std::atomic<long long> g_launches(0);
void count_launches(int n) { g_launches += n; }
long long launches() { return g_launches.load(); }

/* SM count of the current device, cached per device (any host thread) */
static std::atomic<int> g_sm_count[64];
int sm_count()
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64) {
        const int c = g_sm_count[dev].load(std::memory_order_relaxed);
        if (c > 0) return c;
    }
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
    if (dev >= 0 && dev < 64) g_sm_count[dev].store(n, std::memory_order_relaxed);
    return n;
}

static void fill_job(CrawlJob &J, const LaunchCrawl &L)
{
    memset(&J, 0, sizeof(J));
    J.m = L.m;
    J.g = L.g;
    J.st = L.st;
    J.rng = L.rng;
    J.rng_nstreams = L.rng_nstreams;
    J.pix_base = L.pix_base;
    J.limits = L.limits;
    J.counts = L.counts;
    J.countsCovered = L.countsCovered;
    J.per_pixel = L.per_pixel;
    J.Dtab = L.Dtab;
    J.fx = make_fastdiv((uint32_t)L.m.nm);
    J.fy = make_fastdiv((uint32_t)L.m.nM);
    J.job_id = 0;
}

/* one launch of crawl_kernel: one CTA per stream (the hardware scheduler balances them) */
template <int DRAW, int MODEL, int CW>
static cudaError_t start_crawl(const CrawlParams &P, size_t smem, cudaStream_t s)
{
    /* the per-model tables may exceed the 48 KB default; the opt-in is a property of
     * the current device's context, so it is set before every launch (it is cheap) */
    cudaError_t e = cudaFuncSetAttribute(crawl_kernel<DRAW, MODEL, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    if (e != cudaSuccess) return e;
    crawl_kernel<DRAW, MODEL, CW><<<P.nitems, (CW * 32), smem, s>>>(P);
    return cudaSuccess;
}

cudaError_t dispatch_crawl(int draw, int model_type, int cw, bool persistent, const CrawlParams &P, size_t smem,
                           cudaStream_t s);
template <int DRAW, int MODEL, int CW>
static cudaError_t start_crawl_persistent(const CrawlParams &P, size_t smem, cudaStream_t s);

cudaError_t launch_crawl(const LaunchCrawl &L, int draw, cudaStream_t s)
{
    CrawlParams P;
    memset(&P, 0, sizeof(P));
    fill_job(P.job0, L);
    P.nitems = L.stream_end - L.stream_begin;
    P.stream_begin = L.stream_begin;
    P.jt = L.jt;
    P.rec = L.rec;
    P.rec_am = L.rec_am;
    P.rec_capacity = L.rec_capacity;
    P.rec_count = L.rec_count;
    P.err = L.err;
    P.ck = L.ck;
    P.ck_count = L.ck_count;
    P.ck_capacity = L.ck_capacity;
    P.ck_every = L.ck_every > 0 ? L.ck_every : 64;
    if (P.nitems <= 0) return cudaSuccess;
    const size_t smem = (size_t)(L.m.nm + L.m.nM) * sizeof(float);
    if (smem > 64 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = dispatch_crawl(draw, L.m.type, L.cw, false, P, smem, s);
    if (e != cudaSuccess) return e;
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_place(const LaunchPlace &L, cudaStream_t s)
{
    if (L.n <= 0) return cudaSuccess;
    PlaceParams P;
    P.m = L.m; P.g = L.g; P.rec = L.rec; P.rec_am = L.rec_am; P.n = L.n;
    P.lb = L.lb; P.projIdx = L.projIdx; P.projXY = L.projXY; P.DM = L.DM; P.absmag = L.absmag;
    P.XYZ = L.XYZ; P.Am = L.Am; P.AmInf = L.AmInf; P.hidden = L.hidden; P.key = L.key;
    P.nvis = L.nvis;
    int blocks = (int)std::min<int64_t>((L.n + 255) / 256, (int64_t)sm_count() * 16);
    place_kernel<<<blocks, 256, 0, s>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t sort_temp_bytes(int64_t n, size_t *bytes)
{
    *bytes = 0;
    return cub::DeviceRadixSort::SortPairs(nullptr, *bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                           (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n);
}

cudaError_t launch_sort_gather(const LaunchSort &L, cudaStream_t s)
{
    if (L.n <= 0) return cudaSuccess;
    int blocks = (int)std::min<int64_t>((L.n + 255) / 256, (int64_t)sm_count() * 16);
    iota_kernel<<<blocks, 256, 0, s>>>(L.idx_in, L.n);
    size_t tb = L.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(L.temp, tb, L.key_in, L.key_out, L.idx_in, L.idx_out, (int)L.n, 0, 64, s);
    if (e != cudaSuccess) return e;
    if (L.nvisible <= 0) return cudaGetLastError();
    tie_kernel<<<blocks, 256, 0, s>>>(L.key_out, L.idx_out, L.nvisible, L.lb, L.DM, L.absmag, L.Am, L.n);
    GatherParams G;
    G.idx = L.idx_out; G.n = L.nvisible; G.src_pitch = L.n;
    G.lb = L.lb; G.projIdx = L.projIdx; G.projXY = L.projXY; G.DM = L.DM; G.absmag = L.absmag;
    G.XYZ = L.XYZ; G.Am = L.Am; G.AmInf = L.AmInf; G.comp = L.comp; G.out = L.out;
    gather_kernel<<<blocks, 256, 0, s>>>(G);
    count_launches(3);     /* iota, tie, gather (the radix sort itself is CUB's) */
    return cudaGetLastError();
}

/* Jump tables: lo[l] = a^(l-3), hi[h] = a^(32h-3) mod p (scaled multipliers). */
__global__ void jump_table_kernel(const uint32_t *mult, int n, uint64_t *lo, uint64_t *hi)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t a = mult[s];
    uint64_t p = ((uint64_t)a << 32) - 1;
    uint64_t b1 = (1ull << 32) % p;                       /* a^-1 */
    uint64_t b2 = gfr::mulmod_generic(b1, b1, p);         /* a^-2 */
    uint64_t b3 = gfr::mulmod_generic(b2, b1, p);         /* a^-3 */
    uint64_t t = b3;
    uint64_t a32 = 1;
    for (int l = 0; l < 32; l++) {
        lo[(size_t)s * 32 + l] = t;                       /* a^(l-3) */
        t = gfr::mulmod_generic(t, a, p);
    }
    /* a^32 = lo entry 35: t is now a^29; continue */
    uint64_t tt = t;
    for (int l = 32; l < 35; l++) tt = gfr::mulmod_generic(tt, a, p);
    a32 = tt;
    uint64_t h = b3;
    for (int l = 0; l < GF_JUMP_HI; l++) {
        hi[(size_t)s * GF_JUMP_HI + l] = h;               /* a^(32 l - 3) */
        h = gfr::mulmod_generic(h, a32, p);
    }
}

cudaError_t launch_dtab(const SkyModel &m, float *D, cudaStream_t s)
{
    int n = m.nm * m.nM;
    dtab_kernel<<<(n + 255) / 256, 256, 0, s>>>(m, D);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_jump_tables(const uint32_t *mult, int n, uint64_t *lo, uint64_t *hi, cudaStream_t s)
{
    jump_table_kernel<<<(n + 127) / 128, 128, 0, s>>>(mult, n, lo, hi);
    return cudaGetLastError();
}

}  // namespace gfk

/* ------------------------------------------------------------------ */
/* Device side of the multi-request run (gf_catalog_run_multi)        */
/* ------------------------------------------------------------------ */
namespace gfk {

/* x_n of the 48-bit LCG behind drand48/lrand48 (x' = 0x5DEECE66D x + 11 mod 2^48)
 * after n steps from x0, by composing the affine map with itself. */
__device__ __forceinline__ uint64_t lcg48_jump(uint64_t x0, uint64_t n)
{
    const uint64_t M = (1ull << 48) - 1;
    uint64_t acc_a = 1, acc_c = 0, cur_a = 0x5DEECE66Dull, cur_c = 0xBull;
    while (n) {
        if (n & 1) {
            acc_a = (acc_a * cur_a) & M;
            acc_c = (acc_c * cur_a + cur_c) & M;
        }
        cur_c = (cur_c * cur_a + cur_c) & M;
        cur_a = (cur_a * cur_a) & M;
        n >>= 1;
    }
    return (acc_a * x0 + acc_c) & M;
}

/* The stream states of many requests at once, identical to gfh::seed_streams:
 * srand48(seed); per stream i in order: c = (int)(drand48() * a_i) (x86 gives
 * INT_MIN out of range), x = lrand48() (cux.cpp:404-414). */
__global__ void seed_streams_kernel(const uint32_t *seeds, int njobs, const uint32_t *mult, int NS, uint32_t *rng)
{
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (int64_t)njobs * NS) return;
    const int j = (int)(g / NS), i = (int)(g % NS);
    const uint64_t x0 = ((uint64_t)seeds[j] << 16) | 0x330Eull;
    const uint64_t x1 = lcg48_jump(x0, 2ull * i + 1);
    const uint64_t x2 = (0x5DEECE66Dull * x1 + 0xBull) & ((1ull << 48) - 1);
    const uint32_t prime = mult[i];
    const double t = ((double)x1 * 0x1p-48) * (double)prime;
    const int32_t c = (t >= 2147483648.0) ? INT32_MIN : (int32_t)t;
    uint32_t *r = rng + (size_t)j * 3 * NS;
    r[i] = prime;
    r[NS + i] = (uint32_t)c;
    r[2 * NS + i] = (uint32_t)(x2 >> 17);
}

cudaError_t launch_seed_streams(const uint32_t *seeds, int njobs, const uint32_t *mult, int NS, uint32_t *rng, cudaStream_t s)
{
    const int64_t n = (int64_t)njobs * NS;
    if (n <= 0) return cudaSuccess;
    seed_streams_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(seeds, njobs, mult, NS, rng);
    count_launches(1);
    return cudaGetLastError();
}

template <int DRAW, int MODEL, int CW>
static cudaError_t start_crawl_persistent(const CrawlParams &P, size_t smem, cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(crawl_kernel<DRAW, MODEL, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, crawl_kernel<DRAW, MODEL, CW>, (CW * 32), smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int grid = sm_count() * per_sm;
    if (grid > P.nitems) grid = P.nitems;
    crawl_kernel<DRAW, MODEL, CW><<<grid, (CW * 32), smem, s>>>(P);
    return cudaSuccess;
}

/* the crawl instance for (pass, model kind, warps per stream); the integrate pass
 * always runs 4 warps per stream (it has no sequential phase to shorten) */
cudaError_t dispatch_crawl(int draw, int model_type, int cw, bool persistent, const CrawlParams &P, size_t smem,
                           cudaStream_t s)
{
#define GF_GO(D, M, W) return persistent ? start_crawl_persistent<D, M, W>(P, smem, s) : start_crawl<D, M, W>(P, smem, s)
    const bool disk = model_type == GF_MODEL_EXP_DISK;
    if (!draw) {
        if (disk) GF_GO(0, GF_MODEL_EXP_DISK, 4);
        GF_GO(0, GF_MODEL_POWER_LAW_ELLIPSOID, 4);
    }
    if (disk) {
        if (cw == 1) GF_GO(1, GF_MODEL_EXP_DISK, 1);
        if (cw == 2) GF_GO(1, GF_MODEL_EXP_DISK, 2);
        GF_GO(1, GF_MODEL_EXP_DISK, 4);
    }
    if (cw == 1) GF_GO(1, GF_MODEL_POWER_LAW_ELLIPSOID, 1);
    if (cw == 2) GF_GO(1, GF_MODEL_POWER_LAW_ELLIPSOID, 2);
    GF_GO(1, GF_MODEL_POWER_LAW_ELLIPSOID, 4);
#undef GF_GO
}

cudaError_t launch_crawl_multi(const LaunchCrawlMulti &L, int draw, cudaStream_t s)
{
    if (L.nitems <= 0) return cudaSuccess;
    CrawlParams P;
    memset(&P, 0, sizeof(P));
    P.jobs = L.jobs;
    P.items = L.items;
    P.nitems = L.nitems;
    P.next_item = L.counter;
    P.jt = L.jt;
    P.rec = L.rec;
    P.rec_capacity = L.rec_capacity;
    P.rec_count = L.rec_count;
    P.err = L.err;
    P.ck_every = 64;
    const size_t smem = (size_t)L.max_tab * sizeof(float);
    if (smem > 64 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    e = dispatch_crawl(draw, L.model_type, L.cw, true, P, smem, s);
    if (e != cudaSuccess) return e;
    count_launches(1);
    return cudaGetLastError();
}

/* Sort keys of a many-request pass.  A record's key holds its request's output
 * slot in the top sb bits and below them l in fixed point, floor(l * 2^(lbits-9))
 * with lbits = key bits - sb (l <= 360 < 2^9, so the all-ones value of lbits bits
 * is never reached and marks a hidden record, which sorts after every visible
 * record of its slot).  The floor is monotone in l, so the sorted order is l's order
 * up to runs of equal keys (records within 2^-(lbits-9) degrees of each other),
 * which the tie pass orders on the full (l, b, DM, M, Am): star_comp's order
 * (skyconfig_impl.h:34-68).  The key width is sb + 32 bits rounded up to whole
 * 8-bit radix digits, so l keeps at least 23 fractional bits (1.2e-7 deg). */
int multi_key_bits(int sb)
{
    const int t = (sb + 32 + 7) / 8 * 8;
    return t > 64 ? 64 : t;
}

struct MultiKeyParams {
    const StarRecord *rec;
    int64_t n;
    const CrawlJob *jobs;
    const int32_t *job_slot;
    int lbits;
    double lscale;          /* 2^(lbits-9) */
    uint64_t *key;
    uint32_t *idx;
};

/* the sort key of every record, and the identity permutation beside it */
__global__ void __launch_bounds__(256) key_multi_kernel(MultiKeyParams K)
{
    const uint64_t lmask = (1ull << K.lbits) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < K.n; i += (int64_t)gridDim.x * blockDim.x) {
        const StarRecord rec = K.rec[i];
        const int job = rec.stream >> 16;
        const CrawlJob &J = K.jobs[job];
        Placed v;
        place_values(J.m, J.g, rec, nullptr, v);
        const uint64_t lk = v.vis ? (uint64_t)(v.l * K.lscale) : lmask;
        K.key[i] = ((uint64_t)(uint32_t)K.job_slot[job] << K.lbits) | lk;
        K.idx[i] = (uint32_t)i;
    }
}

/* per output slot: first sorted position, end of its visible records (hidden
 * records sort last within the slot) and end of the slot */
__global__ void segment_bounds_kernel(const uint64_t *key, int lbits, int64_t n, int64_t *seg_begin, int64_t *vis_end,
                                      int64_t *seg_end)
{
    const uint64_t lmask = (1ull << lbits) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        const uint32_t sl = (uint32_t)(k >> lbits);
        const bool first = (i == 0) || (uint32_t)(key[i - 1] >> lbits) != sl;
        const bool last = (i + 1 == n) || (uint32_t)(key[i + 1] >> lbits) != sl;
        if (first) seg_begin[sl] = i;
        if (last) seg_end[sl] = i + 1;
        const bool hid = (k & lmask) == lmask;
        if (hid && (first || (key[i - 1] & lmask) != lmask)) vis_end[sl] = i;
        if (!hid && last) vis_end[sl] = i + 1;
    }
}

/* star_comp's fields of a record: l, b, DM, M, Am (floats widened exactly) */
__device__ __forceinline__ void tie_fields(const StarRecord *recs, const CrawlJob *jobs, uint32_t s, double f[5])
{
    const StarRecord rec = recs[s];
    const CrawlJob &J = jobs[rec.stream >> 16];
    Placed v;
    place_values(J.m, J.g, rec, nullptr, v);
    f[0] = v.l; f[1] = v.b; f[2] = v.DM; f[3] = v.M; f[4] = v.Am;
}

__device__ __forceinline__ bool star_less(const double *a, const double *b)
{
    for (int q = 0; q < 4; q++)
        if (a[q] != b[q]) return a[q] < b[q];
    return a[4] < b[4];
}

/* Runs of visible records with equal keys, ordered by (l, b, DM, M, Am)
 * (star_comp, skyconfig_impl.h:34-68) with an insertion sort of their indices;
 * the fields are recomputed from the records (runs up to kTieCache long keep
 * them in registers, longer ones recompute them per comparison). */
__global__ void __launch_bounds__(256) tie_multi_kernel(const uint64_t *key, int lbits, uint32_t *idx, int64_t n,
                                                        const StarRecord *recs, const CrawlJob *jobs)
{
    constexpr int kTieCache = 8;
    const uint64_t lmask = (1ull << lbits) - 1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = key[i];
        if ((k & lmask) == lmask) continue;
        if (i + 1 >= n || key[i + 1] != k) continue;
        if (i > 0 && key[i - 1] == k) continue;     /* not a run start */
        int64_t e = i + 1;
        while (e + 1 < n && key[e + 1] == k) e++;
        const int64_t len = e - i + 1;
        if (len <= kTieCache) {
            double f[kTieCache][5];
            uint32_t id[kTieCache];
#pragma unroll
            for (int q = 0; q < kTieCache; q++) {
                if (q < len) {
                    id[q] = idx[i + q];
                    tie_fields(recs, jobs, id[q], f[q]);
                }
            }
            /* insertion sort over the cached fields (stable: equal records keep their order) */
            int ord[kTieCache];
#pragma unroll
            for (int q = 0; q < kTieCache; q++) ord[q] = q;
            for (int q = 1; q < (int)len; q++) {
                const int cur = ord[q];
                int r = q - 1;
                while (r >= 0 && star_less(f[cur], f[ord[r]])) {
                    ord[r + 1] = ord[r];
                    r--;
                }
                ord[r + 1] = cur;
            }
            for (int q = 0; q < (int)len; q++) {
                uint32_t v = id[0];
#pragma unroll
                for (int t = 1; t < kTieCache; t++)
                    if (ord[q] == t) v = id[t];
                idx[i + q] = v;
            }
        } else {
            for (int64_t q = i + 1; q <= e; q++) {
                const uint32_t cur = idx[q];
                double fc[5];
                tie_fields(recs, jobs, cur, fc);
                int64_t r = q - 1;
                while (r >= i) {
                    const uint32_t o = idx[r];
                    double fo[5];
                    tie_fields(recs, jobs, o, fo);
                    if (!star_less(fc, fo)) break;
                    idx[r + 1] = o;
                    r--;
                }
                idx[r + 1] = cur;
            }
        }
    }
}

struct PlaceSortedParams {
    const StarRecord *rec;
    const CrawlJob *jobs;
    const uint64_t *key;
    const uint32_t *idx;
    int64_t n;
    int lbits;
    const int64_t *seg_begin, *vis_end, *row_begin;
    const int32_t *slot_comp;
    gf_table out;
    int32_t *row_slot;
};

/* Placement in sorted order: the visible records of each slot, placed straight
 * into the output table at row_begin[slot] (consecutive sorted records of a slot
 * are consecutive rows, so the column stores coalesce); row_slot maps rows back
 * to their slot. */
__global__ void __launch_bounds__(256) place_sorted_multi_kernel(PlaceSortedParams S)
{
    const int64_t P = S.out.capacity;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t sl = (uint32_t)(S.key[i] >> S.lbits);
        if (i >= S.vis_end[sl]) continue;
        const int64_t o = S.row_begin[sl] + (i - S.seg_begin[sl]);
        const StarRecord rec = S.rec[S.idx[i]];
        const CrawlJob &J = S.jobs[rec.stream >> 16];
        Placed v;
        place_values(J.m, J.g, rec, nullptr, v);
        S.out.lb[o] = v.l;
        S.out.lb[P + o] = v.b;
        S.out.projIdx[o] = v.projIdx;
        S.out.projXY[o] = v.x;
        S.out.projXY[P + o] = v.y;
        S.out.DM[o] = v.DM;
        S.out.absmag[o] = v.M;
        S.out.XYZ[o] = v.X;
        S.out.XYZ[P + o] = v.Y;
        S.out.XYZ[2 * P + o] = v.Z;
        S.out.comp[o] = S.slot_comp[sl];
        S.out.Am[o] = v.Am;
        S.out.AmInf[o] = v.AmInf;
        S.out.hidden[o] = 0;
        S.row_slot[o] = (int32_t)sl;
    }
}

cudaError_t launch_place_sort_multi(const LaunchPlaceMulti &L, cudaStream_t s)
{
    if (L.n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>((L.n + 255) / 256, (int64_t)sm_count() * 16);
    const int kb = multi_key_bits(L.slot_bits);
    const int lbits = kb - L.slot_bits;
    MultiKeyParams K;
    K.rec = L.rec; K.n = L.n; K.jobs = L.jobs; K.job_slot = L.job_slot;
    K.lbits = lbits; K.lscale = ldexp(1.0, lbits - 9);
    K.key = L.key; K.idx = L.idx_b;
    key_multi_kernel<<<blocks, 256, 0, s>>>(K);
    /* one radix sort by (slot, l) over the key's bits: each request's records in l order */
    size_t tb = L.temp_bytes;
    cudaError_t e = cub::DeviceRadixSort::SortPairs(L.temp, tb, L.key, L.key_b, L.idx_b, L.idx_a, (int)L.n, 0, kb, s);
    if (e != cudaSuccess) return e;
    segment_bounds_kernel<<<blocks, 256, 0, s>>>(L.key_b, lbits, L.n, L.seg_begin, L.vis_end, L.seg_end);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_tie_place_multi(const LaunchPlaceMulti &L, const int64_t *row_begin, const int32_t *slot_comp,
                                   gf_table out, int32_t *row_slot, cudaStream_t s)
{
    if (L.n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>((L.n + 255) / 256, (int64_t)sm_count() * 16);
    const int lbits = multi_key_bits(L.slot_bits) - L.slot_bits;
    tie_multi_kernel<<<blocks, 256, 0, s>>>(L.key_b, lbits, L.idx_a, L.n, L.rec, L.jobs);
    PlaceSortedParams S;
    S.rec = L.rec; S.jobs = L.jobs; S.key = L.key_b; S.idx = L.idx_a; S.n = L.n; S.lbits = lbits;
    S.seg_begin = L.seg_begin; S.vis_end = L.vis_end; S.row_begin = row_begin; S.slot_comp = slot_comp;
    S.out = out; S.row_slot = row_slot;
    place_sorted_multi_kernel<<<blocks, 256, 0, s>>>(S);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t sort_temp_bytes_multi(int64_t n, size_t *bytes)
{
    *bytes = 0;
    return cub::DeviceRadixSort::SortPairs(nullptr, *bytes, (const uint64_t *)nullptr, (uint64_t *)nullptr,
                                           (const uint32_t *)nullptr, (uint32_t *)nullptr, (int)n);
}

}  // namespace gfk
