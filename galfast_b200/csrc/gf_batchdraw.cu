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
    return mu > 10.f || gfr::exceeds_exp_neg(u, mu);
}

/* a request's view for the draw walk (per warp, in shared memory) */
struct DrawJobView {
    const uint32_t *blk, *binfo;
    const uint16_t *bslot, *dslot;
    const float *slotD;
    const float2 *ms2;             /* per pixel: (density, D^3) of each slot, then (first cut row, K) */
    const uint4 *brec;             /* per block: blk, binfo, bslot | first diagonal-start slot << 16, LF max */
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
        float2 *row = P.ms[job] + (size_t)ilb * (nslots + 1);
        for (int s = lane; s < nslots; s += 32) {
            const float D = slotD[s];
            const float px = D * pix.cl * pix.cb;
            const float py = D * pix.sl * pix.cb;
            const float pz = D * pix.sb;
            /* D^3 with the reference's float product (skygen.cu.h:554) */
            row[s] = make_float2(gfc::model_rho<MODEL>(J.m, px, py, pz), D * D * D);
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
        if (lane == 0) row[nslots] = make_float2(__int_as_float(icut), pix.dA * GF_POGSON * m.dm * m.dM);
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

/* Per request of a chunk and block of its grid, the record the bound walk loads
 * in one piece: the block's first bin (i | j << 16), its binfo word, its
 * block-start slot | the slot of its first diagonal start << 16, and the largest
 * LF value over its 10 bins (the same LF(M) samples the draw's shared table
 * holds; negative values count as 0). */
__global__ void __launch_bounds__(256) block_records_kernel(BlockLfParams P)
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
        const uint32_t bi = plan_at<uint32_t>(plan, h->off_binfo)[b];
        const uint32_t wm = (bi >> 16) & 0x3ffu;
        const uint32_t s0 = plan_at<uint16_t>(plan, h->off_bslot)[b];
        const uint32_t s1 = wm ? plan_at<uint16_t>(plan, h->off_dslot)[i + j + 1] : 0u;
        float mx = gfc::lf_sample(m, m.lf, m.M1 - (float)j * m.dM);
        for (int s = 1; s < GF_BLOCK; s++) {
            gfc::step_in_pixel(i, j, m.nm, m.nM);
            mx = fmaxf(mx, gfc::lf_sample(m, m.lf, m.M1 - (float)j * m.dM));
        }
        P.brec[job][b] = make_uint4(bij, bi, s0 | (s1 << 16), __float_as_uint(fmaxf(mx, 0.f)));
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
                V.ms2 = P.ms[job];
                V.pixels = J.g.pixels;
                V.npix = J.g.npixels;
                V.norm = m.norm;
                V.dmin = m.dmin;
                V.dmax = m.dmax;
                V.dlim = m.dmin != 0.f || m.dmax != 0.f;
                V.brec = P.brec ? P.brec[job] : nullptr;
                /* the block bound needs non-negative densities (f >= 0) and normalisation */
                V.bound = V.brec && !V.dlim && m.f >= 0.f && m.norm >= 0.f;
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
                 * empty, so the walk only steps the stream over the block's live bins and
                 * compares the largest uniform with the threshold; a block whose largest
                 * uniform exceeds it is walked again with the exact expected counts. */
                uint32_t live = 0;
                bool any = false;
                int64_t xthr = -1;             /* uniform u = 2^-32 x passes the bound iff x <= xthr */
                uint4 br = make_uint4(0u, 0u, 0u, 0u);
                const float2 *row = V.ms2;
                float K = 0.f;
                const uint64_t w0 = w;
                if (valid) {
                    br = __ldg(V.brec + lb);
                    const int i0 = (int)(br.x & 0xffffu), j0 = (int)(br.x >> 16);
                    const int imax = (int)(br.y & 0xffffu);
                    const uint32_t wm = (br.y >> 16) & 0x3ffu;
                    row = V.ms2 + (size_t)pix * (V.nslots + 1);
                    const float2 ik = row[V.nslots];
                    const int icut = __float_as_int(ik.x);
                    K = ik.y;
                    const float2 q0 = row[br.z & 0xffffu];
                    float msmax = q0.x, D3max = q0.y;
                    if (wm) {
                        const float2 q1 = row[br.z >> 16];
                        msmax = fmaxf(msmax, q1.x);
                        D3max = fmaxf(D3max, q1.y);
                        /* further diagonal starts in the block (short diagonals only) */
                        int d = i0 + j0 + 1;
                        for (uint32_t mm = wm & (wm - 1u); mm; mm &= mm - 1u) {
                            d++;
                            const float2 q2 = row[__ldg(V.dslot + d)];
                            msmax = fmaxf(msmax, q2.x);
                            D3max = fmaxf(D3max, q2.y);
                        }
                    }
                    float mub = __uint_as_float(br.w) * msmax;
                    mub *= V.norm;
                    mub *= D3max;
                    mub *= K;
                    xthr = gfr::uniform_threshold_lower((1.0f - mub) - 3.0e-7f);
                    if (imax < icut) {
                        live = (1u << GF_BLOCK) - 1u;
                    } else if (!(wm & (wm - 1u))) {
                        /* At most one diagonal start (bin p): bins before it continue the
                         * first diagonal (im = i0 + s), bins from it on the next one from
                         * im = max(0, d + 1 - (y - 1)); a bin is live while im < icut, so
                         * each run's live bins are a prefix of it. */
                        const int p = wm ? __ffs(wm) - 1 : GF_BLOCK;
                        live = (1u << min(p, max(0, icut - i0))) - 1u;
                        if (wm) {
                            const int dB = i0 + j0 + 1;
                            const int iB = dB - (V.y - 1) > 0 ? dB - (V.y - 1) : 0;
                            live |= ((1u << min(GF_BLOCK - p, max(0, icut - iB))) - 1u) << p;
                        }
                    } else {
                        /* several diagonal starts (short diagonals at the grid's corners) */
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
                        any = live != 0;               /* the bound proves nothing: exact test throughout */
                    } else {
                        /* one predicated walk for full and partial blocks alike (no divergence) */
                        uint32_t mx = 0;
#pragma unroll
                        for (int s = 0; s < GF_BLOCK; s++)
                            if ((live >> s) & 1u) mx = max(mx, bd_mwc_x(w, a));
                        any = mx > (uint32_t)xthr;
                    }
                }
                if (any) {
                    /* The candidate bins (uniform above the threshold), the first of them and the
                     * stream state before it.  While no star is drawn the uniforms are the bound
                     * walk's, so once no candidate is left the walk's end state stands. */
                    const uint64_t w_end = w;
                    const bool walked = xthr >= 0;
                    uint32_t cand = 0;
                    int s = -1;
                    {
                        uint64_t ww = w0, wf = w0;
#pragma unroll
                        for (int q = 0; q < GF_BLOCK; q++) {
                            if ((live >> q) & 1u) {
                                const uint64_t wb = ww;
                                const uint32_t x = bd_mwc_x(ww, a);
                                if (!walked || (int64_t)x > xthr) {
                                    cand |= 1u << q;
                                    if (s < 0) { s = q; wf = wb; }
                                }
                            }
                        }
                        w = wf;
                    }
                    const int i0 = (int)(br.x & 0xffffu), j0 = (int)(br.x >> 16);
                    const uint32_t wm = (br.y >> 16) & 0x3ffu;
                    const int sl0 = (int)(br.z & 0xffffu);
                    /* exact tests from the first candidate bin s on; the bin's position
                     * follows from the block's diagonal starts (wm), as step_in_pixel walks it */
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
                    float2 q = row[slot];
                    float ms = q.x, D3 = q.y;
                    bool star = false;
                    for (const int s0 = s; s < GF_BLOCK; s++) {
                        if (s > s0) {
                            if ((wm >> s) & 1u) {
                                d++;
                                i = d - (V.y - 1) > 0 ? d - (V.y - 1) : 0;
                                j = d - i;
                                slot = __ldg(V.dslot + d);
                                q = row[slot];
                                ms = q.x;
                                D3 = q.y;
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
                const float2 *row = V.ms2 + (size_t)pix * (V.nslots + 1);
                const float2 ik = row[V.nslots];
                const int icut = __float_as_int(ik.x);
                const float K = ik.y;
                float2 q = row[slot];
                float ms = q.x, D3 = q.y;
                float D = V.dlim ? __ldg(V.slotD + slot) : 0.f;
                bool dc = V.dlim && (V.dmin > D || V.dmax <= D);      /* anchor outside [V.dmin, V.dmax): Am = inf */
                int i = i0, j = j0;
#pragma unroll
                for (int s = 0; s < GF_BLOCK; s++) {
                    if (s > 0 && gfc::step_in_pixel(i, j, V.x, V.y)) {
                        slot = __ldg(V.dslot + i + j);
                        q = row[slot];
                        ms = q.x;
                        D3 = q.y;
                        D = V.dlim ? __ldg(V.slotD + slot) : 0.f;
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

cudaError_t launch_block_records(const BlockLfParams &P, cudaStream_t s)
{
    if (P.total <= 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((P.total + 255) / 256, (long long)sm_count() * 16);
    block_records_kernel<<<blocks, 256, 0, s>>>(P);
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
