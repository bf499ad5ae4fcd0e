/*
 * gf_batchdraw.cu -- the Poisson draw pass of many requests (the batched form).
 *
 * The bins, uniforms and star draws are exactly those of the reference's
 * draw pass (skygenGPU<T>::kernel with draw = 1, skygen.cu.h:469-618, and
 * draw_stars, :366-457): stream t of a request crawls blocks t, t + N, t + 2N, ...
 * of 10 consecutive bins (N streams), takes one uniform per uncut bin, and a
 * bin with stars consumes the Poisson sampler's uniforms and 2 or 4 per star.
 * The arrangement is this library's, for requests whose nm * nM is a multiple
 * of 10 (so every pixel's blocks start at local indices 0, 10, 20, ...):
 *
 *   slot densities  (warp per pixel) the model density at each slot distance of
 *                   the request's anchor plan along the pixel's direction: the
 *                   anchor quantity that depends on the pixel.  The anchor of any
 *                   bin is then a table lookup: block-start anchors through the
 *                   plan's per-block slot, diagonal starts through its
 *                   per-diagonal slot.
 *   draw            one warp per 32 consecutive streams, one lane per stream.
 *                   The lanes' blocks at the same step are consecutive blocks of
 *                   one pixel (stream t + L takes block t + L + r N at step r), so
 *                   the plan and slot-density loads coalesce.  Each lane computes
 *                   mu of its block's 10 bins in registers and walks them with
 *                   plain MWC steps; the lanes whose bin has stars run the
 *                   reference's Poisson sampler and the star uniforms together,
 *                   record the bin (an event: its k and the stream state at its
 *                   first star) and walk on from the state after the stars.
 *   expand          (thread per event) the star records of each event, regenerated
 *                   from its stream state, at offsets from a scan over k.
 * The stream states left behind are the reference's, for the modules that
 * continue the streams (Bond2010).
 */
#include "gf_crawl.cuh"
#include "gf_launch.h"
#include "gf_rng.h"
#include <cub/cub.cuh>

namespace gfk {

namespace {

#define BD_FULL 0xffffffffu
#define GF_EVBUF 32                /* events staged in shared memory per warp */

__device__ __forceinline__ float bd_mwc_step(uint64_t &v, uint32_t a)
{
    const uint64_t t = (uint64_t)a * (uint32_t)v + (v >> 32);
    v = t;
    return GF_MWC_SCALE * (float)(uint32_t)t;
}

/* one MWC step; returns the new x (the uniform is 2^-32 x) */
__device__ __forceinline__ uint32_t bd_mwc_x(uint64_t &v, uint32_t a)
{
    const uint64_t t = (uint64_t)a * (uint32_t)v + (v >> 32);
    v = t;
    return (uint32_t)t;
}

/* exp(-mu) >= 1 - mu: bins that surely draw no star, without exp */
__device__ __forceinline__ bool bd_surely_empty(float u, float mu)
{
    return u <= (1.0f - mu) - 3.0e-7f;
}

/* the sampler's exact test (mu > 10 takes the branch that never compares with exp(-mu)) */
__device__ __forceinline__ bool bd_has_stars(float u, float mu)
{
    return mu > 10.f || u > gfm::expf_(-mu);
}

/* a request's view for the draw walk (per warp, in shared memory) */
struct DrawJobView {
    const uint32_t *blk, *binfo;
    const uint16_t *bslot, *dslot;
    const float *slotD, *msbase, *lfmx;
    const gf_pencil_beam *pixels;
    int nslots, Bp, npix, x, y, N;
    int QN, RN;                    /* N = QN Bp + RN: a stream's step in (pixel, block) */
    float norm, dmin, dmax;
    bool dlim, bound;
};

template <class T>
__device__ __forceinline__ const T *plan_at(const unsigned char *plan, int off)
{
    return (const T *)(plan + off);
}

template <int MODEL>
__global__ void __launch_bounds__(256) slot_density_kernel(SlotDensityParams P)
{
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < P.total_pix; p += nwarps) {
        int lo = 0, hi = P.njobs;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (P.pix_off[mid] <= p) lo = mid; else hi = mid;
        }
        const int job = P.job_list[lo];
        const int ilb = p - P.pix_off[lo];
        const CrawlJob &J = P.jobs[job];
        const unsigned char *plan = P.plans[job];
        const IntegPlanHdr *h = (const IntegPlanHdr *)plan;
        const int nslots = h->nslots;
        const float *slotD = plan_at<float>(plan, h->off_slot);
        const gf_pencil_beam pix = J.g.pixels[ilb];
        float *row = P.ms[job] + (size_t)ilb * (nslots + 2);
        for (int s = lane; s < nslots; s += 32) {
            const float D = slotD[s];
            const float px = D * pix.cl * pix.cb;
            const float py = D * pix.sl * pix.cb;
            const float pz = D * pix.sb;
            row[s] = gfc::model_rho<MODEL>(J.m, px, py, pz);
        }
        /* the pixel's first cut apparent-magnitude row (m0 + dm im + Am > m1; increasing in im)
         * and its volume factor K = dA * POGSON * dm * dM */
        const SkyModel &m = J.m;
        const float Am = gfc::beam_extinction(J.g, pix);
        int icut = m.nm;
        for (int i = lane; i < m.nm; i += 32)
            if (m.m0 + m.dm * (float)i + Am > m.m1) { icut = i; break; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int t = __shfl_xor_sync(0xffffffffu, icut, o);
            icut = t < icut ? t : icut;
        }
        if (lane == 0) {
            row[nslots] = __int_as_float(icut);
            row[nslots + 1] = pix.dA * GF_POGSON * m.dm * m.dM;
        }
    }
}

/* A bin with stars, on the lane (stream) that found it: the reference's Poisson
 * sampler from the bin's stream state wb, then the stars' uniforms (draw_stars:
 * x, y, and M, m unless x^2 + y^2 > 2).  Returns the number of stars and the
 * stream state after them; fills the event record when there are stars. */
__device__ __forceinline__ int draw_event(uint32_t a, uint64_t wb, float mu, const gf_pencil_beam *pp, uint64_t &vnew,
                                       uint64_t &v_star)
{
    gfr::Mwc r;
    r.a = a;
    r.set_v(wb);
    r.used = 0;
    const int k = (int)r.poisson(mu);
    v_star = r.v();
    if (k > 0) {
        const float X = pp->X, Y = pp->Y, dx = pp->dx;
        for (int n = 0; n < k; n++) {
            const float u0 = r.uniform();
            const float u1 = r.uniform();
            float xx = X, yy = Y;
            xx += dx * (u0 - 0.5f);
            yy += dx * (u1 - 0.5f);
            if (!(xx * xx + yy * yy > 2.f)) {
                r.uniform();
                r.uniform();
            }
        }
    }
    vnew = r.v();
    return k;
}

/* stage one event from divergent code (any lanes of the warp) */
__device__ __forceinline__ void stage_event(const BatchDrawParams &P, EventRecord *evb, int *nev, const EventRecord &e)
{
    const int q = atomicAdd(nev, 1);
    if (q < GF_EVBUF) {
        evb[q] = e;
    } else {
        const unsigned long long sl = atomicAdd(P.ev_count, 1ull);
        if (sl < (unsigned long long)P.ev_capacity) P.ev[sl] = e;
    }
}

/* write the warp's staged events to the global list (all lanes) */
__device__ __forceinline__ void flush_events(const BatchDrawParams &P, EventRecord *evb, int *nev, int lane)
{
    __syncwarp();
    const int n = *nev < GF_EVBUF ? *nev : GF_EVBUF;     /* events past the buffer went straight to the list */
    if (n == 0) {
        if (lane == 0) *nev = 0;
        __syncwarp();
        return;
    }
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(P.ev_count, (unsigned long long)n);
    base = __shfl_sync(BD_FULL, base, 0);
    for (int q = lane; q < n; q += 32)
        if (base + q < (unsigned long long)P.ev_capacity) P.ev[base + q] = evb[q];
    __syncwarp();
    if (lane == 0) *nev = 0;
    __syncwarp();
}

/* Per request of a chunk and block of its grid: the largest LF value over the
 * block's 10 bins (the same LF(M) samples the draw's shared table holds). */
__global__ void __launch_bounds__(256) block_lfmax_kernel(BlockLfParams P)
{
    for (long long f = blockIdx.x * (long long)blockDim.x + threadIdx.x; f < P.total; f += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = P.njobs;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (P.blk_off[mid] <= f) lo = mid; else hi = mid;
        }
        const int job = P.job_list[lo];
        const int b = (int)(f - P.blk_off[lo]);
        const SkyModel &m = P.jobs[job].m;
        const unsigned char *plan = P.plans[job];
        const IntegPlanHdr *h = (const IntegPlanHdr *)plan;
        const uint32_t bij = plan_at<uint32_t>(plan, h->off_blk)[b];
        int i = (int)(bij & 0xffffu), j = (int)(bij >> 16);
        float mx = gfc::lf_sample(m, m.lf, m.M1 - (float)j * m.dM);
        for (int s = 1; s < GF_BLOCK; s++) {
            gfc::step_in_pixel(i, j, m.nm, m.nM);
            mx = fmaxf(mx, gfc::lf_sample(m, m.lf, m.M1 - (float)j * m.dM));
        }
        P.lfmax[job][b] = mx;
    }
}

/* One warp per 32 consecutive streams of a request, one lane per stream.  Lane L
 * walks its stream block by block: the blocks of the 32 streams at the same step
 * are 32 consecutive blocks of (mostly) one pixel, so the table loads coalesce.
 * Lanes whose bin has stars run the sampler together and go on from the state
 * after the stars.  BOUND: every request of the launch takes the block bound
 * (non-negative densities, no distance limits, per-block LF maxima present);
 * otherwise every bin's expected count is formed and tested exactly. */
template <int MODEL, bool BOUND>
__global__ void __launch_bounds__(256, 4) batch_draw_kernel(BatchDrawParams P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *mine = smem + (size_t)wib * P.warp_bytes;
    SkyModel &m = *(SkyModel *)mine;
    float *LFM = (float *)(mine + P.off_tab);
    EventRecord *evb = (EventRecord *)(mine + P.off_ev);
    int *nev = (int *)(evb + GF_EVBUF);
    if (lane == 0) *nev = 0;
    __syncwarp();

    /* the request's tables and scalars live in the warp's shared memory, not in
     * registers: the walk keeps its registers for the stream state and the block */
    DrawJobView &V = *(DrawJobView *)(mine + P.off_view);
    int loaded = -1;

    for (;;) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(P.next_item, 1u);
        it = __shfl_sync(BD_FULL, it, 0);
        if (it >= P.nitems) break;
        const uint32_t wi = P.items[it];
        const int job = (int)(wi >> 16), t = (int)(wi & 0xffffu) + lane;
        const CrawlJob &J = P.jobs[job];
        if (job != loaded) {
            __syncwarp();
            const uint32_t *src = (const uint32_t *)&J.m;
            for (int w = lane; w < (int)(sizeof(SkyModel) / 4); w += 32) ((uint32_t *)&m)[w] = src[w];
            __syncwarp();
            for (int q = lane; q < m.nM; q += 32) LFM[q] = gfc::lf_sample(m, m.lf, m.M1 - (float)q * m.dM);
            if (lane == 0) {
                const unsigned char *plan = P.plans[job];
                const IntegPlanHdr *h = (const IntegPlanHdr *)plan;
                V.x = m.nm; V.y = m.nM; V.N = m.nthreads;
                V.nslots = h->nslots;
                V.Bp = h->nblocks;
                V.QN = V.N / V.Bp;
                V.RN = V.N - V.QN * V.Bp;
                V.slotD = plan_at<float>(plan, h->off_slot);
                V.blk = plan_at<uint32_t>(plan, h->off_blk);
                V.bslot = plan_at<uint16_t>(plan, h->off_bslot);
                V.dslot = plan_at<uint16_t>(plan, h->off_dslot);
                V.binfo = plan_at<uint32_t>(plan, h->off_binfo);
                V.msbase = P.ms[job];
                V.pixels = J.g.pixels;
                V.npix = J.g.npixels;
                V.norm = m.norm;
                V.dmin = m.dmin;
                V.dmax = m.dmax;
                V.dlim = m.dmin != 0.f || m.dmax != 0.f;
                V.lfmx = P.lfmax ? P.lfmax[job] : nullptr;
                /* the block bound needs non-negative densities (f >= 0) and normalisation */
                V.bound = V.lfmx && !V.dlim && m.f >= 0.f && m.norm >= 0.f;
            }
            __syncwarp();
            loaded = job;
        }
        if (BOUND && !V.bound) {
            /* the host put a request that needs the exact test into the bound launch */
            if (lane == 0) atomicOr(P.err, 2ull);
            continue;
        }
        const int NS = J.rng_nstreams;
        uint32_t *rng = J.rng;
        const bool stream_ok = t < V.N;
        const uint32_t a = stream_ok ? rng[t] : 0u;
        uint64_t w = stream_ok ? (((uint64_t)rng[NS + t] << 32) | rng[2 * NS + t]) : 0ull;
        const int sid = (job << 16) | t;
        /* block r of stream t is the (t + r N)-th block of the request */
        int pix = stream_ok ? t / V.Bp : V.npix, lb = stream_ok ? t - (t / V.Bp) * V.Bp : 0;
        int nst = 0;
        bool stop = !stream_ok;
        for (;;) {
            const bool valid = !stop && pix < V.npix;
            if (!__any_sync(BD_FULL, valid)) break;
            if constexpr (BOUND) {
                /* Upper bound of the block's expected counts: the reference's float product
                 * with each factor at its largest over the block (correctly rounded products of
                 * non-negative factors are monotone).  u <= 1 - bound - 3e-7 proves a bin
                 * empty; only the bins whose uniform exceeds it need their exact mu. */
                uint32_t live = 0, cand = 0;
                int i0 = 0, j0 = 0, sl0 = 0;
                float K = 0.f, thr = 0.f;
                int64_t xthr = -1;             /* uniform u = 2^-32 x passes the bound iff x <= xthr */
                const float *msr = V.msbase;
                const uint64_t w0 = w;
                if (valid) {
                    const uint32_t bij = __ldg(V.blk + lb);
                    i0 = (int)(bij & 0xffffu);
                    j0 = (int)(bij >> 16);
                    const uint32_t bi = __ldg(V.binfo + lb);
                    const int imax = (int)(bi & 0xffffu);
                    const uint32_t wm = (bi >> 16) & 0x3ffu;
                    sl0 = __ldg(V.bslot + lb);
                    msr = V.msbase + (size_t)pix * (V.nslots + 2);
                    const int icut = __float_as_int(msr[V.nslots]);
                    K = msr[V.nslots + 1];
                    float msmax = msr[sl0], Dmax = __ldg(V.slotD + sl0);
                    int d = i0 + j0;
                    for (uint32_t mm = wm; mm; mm &= mm - 1u) {
                        d++;
                        const int sl = __ldg(V.dslot + d);
                        msmax = fmaxf(msmax, msr[sl]);
                        Dmax = fmaxf(Dmax, __ldg(V.slotD + sl));
                    }
                    float mub = fmaxf(__ldg(V.lfmx + lb), 0.f) * msmax;
                    mub *= V.norm;
                    mub *= Dmax * Dmax * Dmax;
                    mub *= K;
                    thr = (1.0f - mub) - 3.0e-7f;
                    xthr = gfr::uniform_threshold(thr);
                    if (imax < icut) {
                        live = (1u << GF_BLOCK) - 1u;
                    } else {
                        int ii = i0, dd = i0 + j0;
                        live = ii < icut ? 1u : 0u;
                        for (int s = 1; s < GF_BLOCK; s++) {
                            if ((wm >> s) & 1u) {
                                dd++;
                                ii = dd - (V.y - 1) > 0 ? dd - (V.y - 1) : 0;
                            } else {
                                ii++;
                            }
                            live |= ii < icut ? (1u << s) : 0u;
                        }
                    }
                    if (xthr < 0) {
                        cand = live;                   /* the bound proves nothing: exact test throughout */
                    } else {
                        const uint32_t X = (uint32_t)xthr;
#pragma unroll
                        for (int s = 0; s < GF_BLOCK; s++) {
                            if ((live >> s) & 1u) {
                                if (bd_mwc_x(w, a) > X) cand |= 1u << s;
                            }
                        }
                    }
                }
                if (cand) {
                    /* Exact tests from the first candidate bin on.  The state before bin
                     * s is w0 advanced over the live bins before s; the bin's position
                     * follows from the block's diagonal starts (wm), as step_in_pixel
                     * walks it.  While no star is drawn the uniforms are the bound
                     * walk's, so once no candidate is left the walk's end state stands. */
                    const uint64_t w_end = w;
                    const bool walked = xthr >= 0;
                    const uint32_t bi = __ldg(V.binfo + lb);
                    const uint32_t wm = (bi >> 16) & 0x3ffu;
                    int s = __ffs(cand) - 1;
                    w = w0;
                    for (uint32_t q = live & ((1u << s) - 1u); q; q &= q - 1u) bd_mwc_x(w, a);
                    /* position and anchor of bin s */
                    const uint32_t starts = wm & ((2u << s) - 2u);         /* diagonal starts in bins 1..s */
                    int d = i0 + j0 + __popc(starts), i, j, slot;
                    if (starts) {
                        const int s1 = 31 - __clz(starts);
                        i = d - (V.y - 1) > 0 ? d - (V.y - 1) : 0;
                        i += s - s1;
                        j = d - i;
                        slot = __ldg(V.dslot + d);
                    } else {
                        i = i0 + s;
                        j = j0 - s;
                        slot = sl0;
                    }
                    float ms = msr[slot], D = __ldg(V.slotD + slot);
                    float D3 = D * D * D;
                    bool star = false;
                    for (const int s0 = s; s < GF_BLOCK; s++) {
                        if (s > s0) {
                            if ((wm >> s) & 1u) {
                                d++;
                                i = d - (V.y - 1) > 0 ? d - (V.y - 1) : 0;
                                j = d - i;
                                slot = __ldg(V.dslot + d);
                                ms = msr[slot];
                                D = __ldg(V.slotD + slot);
                                D3 = D * D * D;
                            } else {
                                i++;
                                j--;
                            }
                        }
                        if (!((live >> s) & 1u)) continue;
                        if (walked && !star && !(cand >> s)) { w = w_end; break; }
                        const uint64_t wb = w;
                        const uint32_t xs = bd_mwc_x(w, a);
                        if ((int64_t)xs <= xthr) continue;
                        const float u = GF_MWC_SCALE * (float)xs;
                        float r = LFM[j] * ms;
                        r *= V.norm;
                        r *= D3;
                        r *= K;
                        if (bd_surely_empty(u, r) || !bd_has_stars(u, r)) continue;
                        if (!(r < 3.0e38f)) {
                            /* an infinite expected count would never leave the sampler's gamma loop */
                            atomicOr(P.err, 1ull);
                            stop = true;
                            break;
                        }
                        uint64_t v_star = 0;
                        const int k = draw_event(a, wb, r, V.pixels + pix, w, v_star);
                        star = true;
                        if (k > 0) {
                            EventRecord e;
                            e.stream = sid;
                            e.ilb = pix;
                            e.im = (int16_t)i;
                            e.iM = (int16_t)j;
                            e.k = k;
                            e.nstars = nst;
                            e.pad = 0;
                            e.v_star = v_star;
                            stage_event(P, evb, nev, e);
                            nst += k;
                        }
                    }
                }
                __syncwarp();
                if (*nev >= GF_EVBUF / 2) flush_events(P, evb, nev, lane);
                pix += V.QN;
                lb += V.RN;
                if (lb >= V.Bp) { lb -= V.Bp; pix++; }
                continue;
            } else {
            float mu[GF_BLOCK];
            uint32_t live = 0;
            int i0 = 0, j0 = 0;
            if (valid) {
                const uint32_t bij = __ldg(V.blk + lb);
                i0 = (int)(bij & 0xffffu);
                j0 = (int)(bij >> 16);
                int slot = __ldg(V.bslot + lb);
                const float *msr = V.msbase + (size_t)pix * (V.nslots + 2);
                const int icut = __float_as_int(msr[V.nslots]);
                const float K = msr[V.nslots + 1];
                float ms = msr[slot], D = __ldg(V.slotD + slot);
                float D3 = D * D * D;
                bool dc = V.dlim && (V.dmin > D || V.dmax <= D);      /* anchor outside [V.dmin, V.dmax): Am = inf */
                int i = i0, j = j0;
#pragma unroll
                for (int s = 0; s < GF_BLOCK; s++) {
                    if (s > 0 && gfc::step_in_pixel(i, j, V.x, V.y)) {
                        slot = __ldg(V.dslot + i + j);
                        ms = msr[slot];
                        D = __ldg(V.slotD + slot);
                        D3 = D * D * D;
                        dc = V.dlim && (V.dmin > D || V.dmax <= D);
                    }
                    float r = LFM[j] * ms;
                    r *= V.norm;
                    r *= D3;
                    r *= K;
                    mu[s] = r;
                    live |= (i < icut && !dc) ? (1u << s) : 0u;
                }
            } else {
#pragma unroll
                for (int s = 0; s < GF_BLOCK; s++) mu[s] = 0.f;
            }
            uint32_t todo = live;
            for (;;) {
                /* walk the lane's remaining bins up to the first with stars */
                int ev_s = -1;
                uint64_t wb_ev = 0;
                float mu_ev = 0.f;
                for (;;) {
                    int c = -1;
                    uint64_t cwb = 0;
                    float cu = 0.f, cmu = 0.f;
#pragma unroll
                    for (int s = 0; s < GF_BLOCK; s++) {
                        if (c < 0 && ((todo >> s) & 1u)) {
                            const uint64_t wb = w;
                            const float u = bd_mwc_step(w, a);
                            if (!bd_surely_empty(u, mu[s])) { c = s; cwb = wb; cu = u; cmu = mu[s]; }
                        }
                    }
                    if (c < 0) { todo = 0; break; }
                    todo &= ~((2u << c) - 1u);
                    if (bd_has_stars(cu, cmu)) {
                        ev_s = c;
                        wb_ev = cwb;
                        mu_ev = cmu;
                        break;
                    }
                }
                const bool ev = ev_s >= 0;
                if (!__any_sync(BD_FULL, ev)) break;
                int k = 0;
                uint64_t v_star = 0;
                int ei = 0, ej = 0;
                if (ev) {
                    if (!(mu_ev < 3.0e38f)) {
                        /* an infinite expected count would never leave the sampler's gamma loop */
                        atomicOr(P.err, 1ull);
                        stop = true;
                        todo = 0;
                    } else {
                        k = draw_event(a, wb_ev, mu_ev, V.pixels + pix, w, v_star);
                        ei = i0; ej = j0;
                        for (int s = 1; s <= ev_s; s++) gfc::step_in_pixel(ei, ej, V.x, V.y);
                    }
                }
                /* stage the bins with stars (all lanes converged) */
                const bool rec = ev && k > 0;
                const unsigned rm = __ballot_sync(BD_FULL, rec);
                if (rm) {
                    if (*nev + __popc(rm) > GF_EVBUF) flush_events(P, evb, nev, lane);      /* leaves *nev = 0 */
                    if (rec) {
                        EventRecord e;
                        e.stream = sid;
                        e.ilb = pix;
                        e.im = (int16_t)ei;
                        e.iM = (int16_t)ej;
                        e.k = k;
                        e.nstars = nst;
                        e.pad = 0;
                        e.v_star = v_star;
                        evb[*nev + __popc(rm & ((1u << lane) - 1u))] = e;
                        nst += k;
                    }
                    __syncwarp();
                    if (lane == 0) *nev += __popc(rm);
                    __syncwarp();
                }
            }
            if (*nev >= GF_EVBUF / 2) flush_events(P, evb, nev, lane);
            /* the stream's next block: N blocks further */
            pix += V.QN;
            lb += V.RN;
            if (lb >= V.Bp) { lb -= V.Bp; pix++; }
            }
        }
        if (stream_ok && !stop) {
            rng[NS + t] = (uint32_t)(w >> 32);
            rng[2 * NS + t] = (uint32_t)w;
        }
    }
    flush_events(P, evb, nev, lane);
}

__global__ void event_k_kernel(const EventRecord *ev, int64_t n, int64_t *k64)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        k64[e] = ev[e].k;
}

/* the star records of each event (draw_stars' uniforms, skygen.cu.h:366-457) */
__global__ void __launch_bounds__(256) expand_kernel(const EventRecord *ev, int64_t n, const int64_t *off, const int64_t *k64,
                                                     const CrawlJob *jobs, StarRecord *rec, int64_t cap, int64_t *total)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
        const EventRecord E = ev[e];
        const int job = E.stream >> 16, t = E.stream & 0xffff;
        const CrawlJob &J = jobs[job];
        const gf_pencil_beam pix = J.g.pixels[E.ilb];
        gfr::Mwc r;
        r.a = J.rng[t];
        r.set_v(E.v_star);
        r.used = 0;
        const int64_t o = off[e];
        for (int q = 0; q < E.k; q++) {
            StarRecord s;
            s.stream = E.stream;
            s.ilb = E.ilb + J.pix_base;
            s.im = E.im;
            s.iM = E.iM;
            s.seq = E.nstars + q;
            s.u[0] = r.uniform();
            s.u[1] = r.uniform();
            float xx = pix.X, yy = pix.Y;
            xx += pix.dx * (s.u[0] - 0.5f);
            yy += pix.dx * (s.u[1] - 0.5f);
            if (xx * xx + yy * yy > 2.f) {
                s.u[2] = s.u[3] = 0.f;
            } else {
                s.u[2] = r.uniform();
                s.u[3] = r.uniform();
            }
            if (o + q < cap) rec[o + q] = s;
        }
        if (e == n - 1) *total = o + k64[e];
    }
}

}  // namespace

cudaError_t launch_slot_density(const SlotDensityParams &P, int model_type, cudaStream_t s)
{
    if (P.total_pix <= 0) return cudaSuccess;
    const long long need = ((long long)P.total_pix + 7) / 8;
    const int blocks = (int)std::min<long long>(need, (long long)sm_count() * 8);
    if (model_type == GF_MODEL_EXP_DISK)
        slot_density_kernel<GF_MODEL_EXP_DISK><<<blocks, 256, 0, s>>>(P);
    else
        slot_density_kernel<GF_MODEL_POWER_LAW_ELLIPSOID><<<blocks, 256, 0, s>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_block_lfmax(const BlockLfParams &P, cudaStream_t s)
{
    if (P.total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((P.total + 255) / 256, (long long)sm_count() * 16);
    block_lfmax_kernel<<<blocks, 256, 0, s>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

size_t batch_draw_warp_bytes(int max_tab, BatchDrawParams *P)
{
    size_t off = (sizeof(SkyModel) + 15) & ~(size_t)15;
    P->off_view = (int32_t)off;
    off += (sizeof(DrawJobView) + 15) & ~(size_t)15;
    P->off_tab = (int32_t)off;
    off += ((size_t)4 * max_tab + 15) & ~(size_t)15;
    P->off_ev = (int32_t)off;
    off += sizeof(EventRecord) * GF_EVBUF + 16;
    off = (off + 15) & ~(size_t)15;
    P->warp_bytes = (int32_t)off;
    return off;
}

template <int MODEL, bool BOUND>
cudaError_t launch_batch_draw_t(const BatchDrawParams &P, int warps_per_cta, size_t smem, cudaStream_t s)
{
    const int threads = 32 * warps_per_cta;
    cudaError_t e = cudaFuncSetAttribute(batch_draw_kernel<MODEL, BOUND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_draw_kernel<MODEL, BOUND>, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const long long want = ((long long)P.nitems + warps_per_cta - 1) / warps_per_cta;
    const int blocks = (int)std::min<long long>(want, (long long)sm_count() * per_sm);
    batch_draw_kernel<MODEL, BOUND><<<blocks, threads, smem, s>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_batch_draw(const BatchDrawParams &P, int model_type, int warps_per_cta, bool bound, cudaStream_t s)
{
    if (P.nitems <= 0) return cudaSuccess;
    if (warps_per_cta < 1 || warps_per_cta > 8) warps_per_cta = 4;
    const size_t smem = (size_t)warps_per_cta * P.warp_bytes;
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(P.next_item, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (model_type == GF_MODEL_EXP_DISK)
        return bound ? launch_batch_draw_t<GF_MODEL_EXP_DISK, true>(P, warps_per_cta, smem, s)
                     : launch_batch_draw_t<GF_MODEL_EXP_DISK, false>(P, warps_per_cta, smem, s);
    return bound ? launch_batch_draw_t<GF_MODEL_POWER_LAW_ELLIPSOID, true>(P, warps_per_cta, smem, s)
                 : launch_batch_draw_t<GF_MODEL_POWER_LAW_ELLIPSOID, false>(P, warps_per_cta, smem, s);
}

cudaError_t expand_temp_bytes(int64_t nev, size_t *bytes)
{
    *bytes = 0;
    if (nev <= 0) return cudaSuccess;
    return cub::DeviceScan::ExclusiveSum(nullptr, *bytes, (const int64_t *)nullptr, (int64_t *)nullptr, (int)nev);
}

cudaError_t launch_expand_events(const EventRecord *ev, int64_t nev, const CrawlJob *jobs, int64_t *k64, int64_t *off64,
                                 void *temp, size_t temp_bytes, StarRecord *rec, int64_t rec_capacity, int64_t *total,
                                 cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(total, 0, sizeof(int64_t), s);
    if (e != cudaSuccess || nev <= 0) return e;
    const int blocks = (int)std::min<long long>((nev + 255) / 256, (long long)sm_count() * 16);
    event_k_kernel<<<blocks, 256, 0, s>>>(ev, nev, k64);
    size_t tb = temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(temp, tb, k64, off64, (int)nev, s);
    if (e != cudaSuccess) return e;
    expand_kernel<<<blocks, 256, 0, s>>>(ev, nev, off64, k64, jobs, rec, rec_capacity, total);
    count_launches(3);
    return cudaGetLastError();
}

}  // namespace gfk
