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
 * ahead between blocks.  Here one warp owns one stream and lane l owns block
 * j+l of it: the bin enumeration, the per-diagonal anchor (distance, extinction,
 * model density) and each bin's expected count mu are evaluated for 32 blocks
 * (320 bins) at once.  Only the uniforms are sequential: the MWC stream is a
 * Lehmer generator modulo its safe prime, so lane l jumps directly to the
 * uniform its first bin would consume if every earlier bin drew zero stars
 * (two 128-bit modular multiplications), then walks its block with plain MWC
 * steps.  The first lane that finds a bin with stars ("event": u > exp(-mu),
 * or mu > 10) hands that bin to the whole warp, which runs the reference's
 * Poisson sampler and star draws sequentially, and the window restarts right
 * after it.  Results are bin-for-bin and draw-for-draw those of the reference
 * CPU path.
 */
#include "gf_crawl.cuh"
#include "gf_rng.h"
#include <cub/cub.cuh>
#include <atomic>

namespace gfk {

struct CrawlParams {
    SkyModel m;
    SkyGeom g;
    CrawlState st;
    uint32_t *rng;                 /* persistent stream state [3][rng_nstreams] */
    int32_t rng_nstreams;
    JumpTables jt;
    int32_t stream_begin, stream_end;
    const int64_t *limits;         /* per-stream star limit for this launch (draw) */
    StarRecord *rec;
    int64_t rec_capacity;
    unsigned long long *rec_count;
    unsigned long long *err;       /* set when a bin's expected count is infinite */
    /* integrate outputs */
    double *counts, *countsCovered;
    double *per_pixel;
    int32_t pix_base;              /* first pixel of this launch within the generator's pixel list */
    const float *Dtab;             /* distances D[im][iM] of the model's bins */
};

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src)
{
    uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src);
    uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

/* One MWC step on the combined state v = c*2^32 + x. */
__device__ __forceinline__ float mwc_step(uint64_t &v, uint32_t a)
{
    uint64_t t = (uint64_t)a * (uint32_t)v + (v >> 32);
    v = t;
    return GF_MWC_SCALE * (float)(uint32_t)t;
}

/* v * a^n mod p for 0 <= n < 1024 using the lane-held scaled powers. */
__device__ __forceinline__ uint64_t jump(uint64_t v, int n, uint64_t jlo, uint64_t jhi, uint32_t a, uint64_t p)
{
    uint64_t ml = shfl64(jlo, n & 31);
    uint64_t mh = shfl64(jhi, (n >> 5) & 31);
    uint64_t w = gfr::mwc_mulmod_scaled(ml, v, a, p);
    return gfr::mwc_mulmod_scaled(mh, w, a, p);
}

/* Lower bound of expf(-mu) used to accept "no star" without evaluating expf:
 * exp(-mu) >= 1 - mu, and the portable expf is within one ulp of exp. */
__device__ __forceinline__ bool surely_empty(float u, float mu)
{
    return u <= (1.0f - mu) - 3.0e-7f;
}

/* The bin at position s of the block starting at local index k0 in pixel ilb0,
 * by following advance() from the block start (skygen.cu.h:307-358).  Also
 * returns whether the bin is alive (the crawl has not left the last pixel) and
 * the last anchor bin at or after position s_from (-1 if none). */
struct BinPos {
    int ilb, im, iM;
    bool alive;
    int anchor_s;
};

__device__ BinPos bin_at(int ilb0, int k0, int s, int s_from, int x, int y, int npix)
{
    BinPos r;
    int i, j;
    gfc::diag_to_ij(k0, x, y, i, j);
    int ilb = ilb0;
    bool alive = ilb0 < npix;
    int anc = (s_from <= 0) ? 0 : -1;
    for (int q = 1; q <= s; q++) {
        bool inc;
        bool mv = gfc::advance(i, j, x, y, inc);
        if (inc) ilb++;
        if (mv && ilb >= npix) alive = false;
        if (mv && q >= s_from) anc = q;
    }
    r.ilb = ilb; r.im = i; r.iM = j; r.alive = alive; r.anchor_s = anc;
    return r;
}

/* State of the crawl cursor of one stream, uniform across its warp. */
struct Cursor {
    int blk_ilb, blk_k, pos;
    int ndraw;
    int cur_ilb, cur_im, cur_iM;
    gfc::Anchor anc;
};

/* Draw up to ndraw stars of the bin (ilb, im, M) while the stream is under its
 * limit (draw_stars, skygen.cu.h:366-457); uniforms are recorded for the
 * placement kernel.  Executed identically by all lanes; lane 0 writes. */
__device__ void draw_stars(const CrawlParams &P, int tid, int lane, gfr::Mwc &r, int &ndraw, int64_t &nstars,
                           int64_t limit, int ilb, int im, int iM, float AmMin)
{
    if (!ndraw) return;
    int64_t room = limit - nstars;
    int todo = (int)(room < (int64_t)ndraw ? (room > 0 ? room : 0) : ndraw);
    if (todo <= 0) return;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(P.rec_count, (unsigned long long)todo);
    base = __shfl_sync(0xffffffffu, base, 0);
    const gf_pencil_beam pix = P.g.pixels[ilb];
    for (int n = 0; n < todo; n++) {
        StarRecord rec;
        rec.stream = tid;
        rec.ilb = ilb + P.pix_base;
        rec.im = (short)im;
        rec.iM = (short)iM;
        rec.AmMin = AmMin;
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
        unsigned long long slot = base + n;
        if (lane == 0 && slot < (unsigned long long)P.rec_capacity) P.rec[slot] = rec;
    }
    nstars += todo;
    ndraw -= todo;
}

/* Anchor quantities with the distance taken from the per-model table
 * D[im][iM] = powf(10, 0.2 DM + 1) (identical to compute_pos, skygen.cu.h:216-229). */
__device__ __forceinline__ gfc::Anchor anchor(const CrawlParams &P, const gf_pencil_beam &pix, int im, int iM)
{
    const SkyModel &m = P.m;
    gfc::Anchor a;
    a.D = P.Dtab[im * m.nM + iM];
    a.Am = gfc::beam_extinction(P.g, pix);
    float x = a.D * pix.cl * pix.cb;
    float y = a.D * pix.sl * pix.cb;
    float z = a.D * pix.sb;
    a.ms = gfc::model_rho(m, x, y, z);
    return a;
}

template <int DRAW>
__device__ void crawl_stream(const CrawlParams &P, const float *lf, float *mu_sm, int tid, int lane)
{
    const SkyModel &m = P.m;
    const int x = m.nm, y = m.nM, kmax = x * y, N = m.nthreads;
    const int npix = P.g.npixels;
    const CrawlState &st = P.st;

    Cursor c;
    int status = DRAW ? st.status[tid] : 0;
    if (status == 2) return;
    if (status == 0) {
        long long k = (long long)GF_BLOCK * tid;
        c.blk_ilb = (int)(k / kmax);
        c.blk_k = (int)(k % kmax);
        c.pos = 0;
        c.ndraw = 0;
        c.cur_ilb = c.cur_im = c.cur_iM = 0;
        c.anc.D = c.anc.Am = c.anc.ms = 0.f;
    } else {
        c.blk_ilb = st.blk_ilb[tid]; c.blk_k = st.blk_k[tid]; c.pos = st.pos[tid];
        c.ndraw = st.ndraw[tid];
        c.cur_ilb = st.cur_ilb[tid]; c.cur_im = st.cur_im[tid]; c.cur_iM = st.cur_iM[tid];
        c.anc.D = st.D[tid]; c.anc.Am = st.Am[tid]; c.anc.ms = st.ms[tid];
    }

    uint32_t a = 0;
    uint64_t p = 0, v = 0, jlo = 0, jhi = 0;
    int64_t nstars = 0, limit = 0;
    gfr::Mwc r;
    if (DRAW) {
        const int NS = P.rng_nstreams;
        a = P.rng[tid];
        r.a = a; r.c = P.rng[NS + tid]; r.x = P.rng[2 * NS + tid];
        p = r.p();
        v = r.v();
        jlo = P.jt.lo[(size_t)tid * 32 + lane];
        jhi = P.jt.hi[(size_t)tid * 32 + lane];
        nstars = st.nstars[tid];
        limit = P.limits[tid];
        /* finish the draw that did not complete before the table filled (skygen.cu.h:497-502) */
        if (c.ndraw) {
            draw_stars(P, tid, lane, r, c.ndraw, nstars, limit, c.cur_ilb, c.cur_im, c.cur_iM, c.anc.Am);
            v = r.v();
        }
    }

    double cnt_sum = 0.0, cov_sum = 0.0;
    bool finished = false;
    int pp_ilb = -1;
    double pp_sum = 0.0;
    const long long step = (long long)GF_BLOCK * N;

    while (!(DRAW && c.ndraw)) {
        /* ---------- phase A: bins, anchors and mu of 32 blocks ---------- */
        long long kk = (long long)c.blk_k + (long long)lane * step;
        const int my_k = (int)(kk % kmax);
        const int my_q = (int)(kk / kmax);
        const int drift = gfc::block_drift(my_k, x, y);
        int dsum = drift;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, dsum, o);
            if (lane >= o) dsum += t;
        }
        const int dexcl = dsum - drift;
        const int dtot = __shfl_sync(0xffffffffu, dsum, 31);
        long long my_ilb_ll = (long long)c.blk_ilb + my_q + dexcl;
        const int my_ilb = my_ilb_ll > npix ? npix : (int)my_ilb_ll;
        const int s_begin = (lane == 0) ? c.pos : 0;
        const bool fast = my_k + GF_BLOCK - 1 < kmax;

        /* mu of bin s of this lane at mu_sm[s * 32 + lane] (conflict-free) */
#define MU(s_) mu_sm[(s_) * 32 + lane]
        gfc::Anchor anc = c.anc;       /* lane 0 inherits the carried anchor */
        bool lane_end = my_ilb >= npix;
        {
            int i = 0, j = 0, ilb = my_ilb;
            bool dead = lane_end;
            if (!dead) gfc::diag_to_ij(my_k, x, y, i, j);
#pragma unroll 1
            for (int s = 0; s < GF_BLOCK; s++) {
                bool moved = true;
                if (s > 0 && !dead) {
                    if (fast) {
                        int ni = i + 1, nj = j - 1;
                        if (nj < 0 || ni >= x) gfc::diag_to_ij(my_k + s, x, y, ni, nj);
                        i = ni; j = nj;
                        moved = (i == 0) || (j == y - 1);
                    } else {
                        bool inc;
                        moved = gfc::advance(i, j, x, y, inc);
                        if (inc) ilb++;
                        if (moved && ilb >= npix) dead = true;
                    }
                }
                float mus = gfc::cut_marker();
                if (dead) lane_end = true;
                if (!dead && s >= s_begin) {
                    const gf_pencil_beam pix = P.g.pixels[ilb];
                    if (moved || (s == s_begin && lane != 0)) anc = anchor(P, pix, i, j);
                    const float M = m.M1 - (float)j * m.dM;
                    mus = gfc::bin_mu(m, lf, anc, pix.dA, i, M);
                    if (!DRAW && !gfc::is_cut(mus)) {
                        cnt_sum += (double)mus;
                        float cov = mus * pix.coveredFraction;
                        cov_sum += (double)cov;
                        if (P.per_pixel) {
                            if (ilb != pp_ilb) {
                                if (pp_ilb >= 0) atomicAdd(&P.per_pixel[pp_ilb + P.pix_base], pp_sum);
                                pp_ilb = ilb;
                                pp_sum = 0.0;
                            }
                            pp_sum += (double)cov;
                        }
                    }
                }
                if (DRAW) MU(s) = mus;
            }
        }
        const unsigned end_mask = __ballot_sync(0xffffffffu, lane_end);
        __syncwarp();

        if (DRAW) {
            /* ---------- phase B: uniforms, restarted after each bin with stars ---------- */
            int lane_lo = s_begin;          /* first bin of the lane not yet consumed */
            for (;;) {
                int cnt = 0;
#pragma unroll
                for (int s = 0; s < GF_BLOCK; s++) cnt += (s >= lane_lo && !gfc::is_cut(MU(s))) ? 1 : 0;
                int csum = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int t = __shfl_up_sync(0xffffffffu, csum, o);
                    if (lane >= o) csum += t;
                }
                uint64_t w = jump(v, csum - cnt, jlo, jhi, a, p);
                int ev_s = -1;
                uint64_t w_before = w;
                float ev_mu = 0.f;
#pragma unroll
                for (int s = 0; s < GF_BLOCK; s++) {
                    const float mus = MU(s);
                    if (ev_s < 0 && s >= lane_lo && !gfc::is_cut(mus)) {
                        uint64_t wb = w;
                        float u = mwc_step(w, a);
                        if (!surely_empty(u, mus)) {
                            if (mus > 10.f || u > gfm::expf_(-mus)) { ev_s = s; w_before = wb; ev_mu = mus; }
                        }
                    }
                }
                const unsigned ev_mask = __ballot_sync(0xffffffffu, ev_s >= 0);
                if (ev_mask == 0) {
                    v = shfl64(w, 31);
                    break;
                }
                /* the first lane with stars: its bin goes through the reference's sampler */
                const int f = __ffs(ev_mask) - 1;
                const int es = __shfl_sync(0xffffffffu, ev_s, f);
                const uint64_t vb = shfl64(w_before, f);
                const float emu = __shfl_sync(0xffffffffu, ev_mu, f);
                const int f_ilb = __shfl_sync(0xffffffffu, my_ilb, f);
                const int f_k = __shfl_sync(0xffffffffu, my_k, f);
                const int f_sbeg = (f == 0) ? c.pos : 0;
                const BinPos eb = bin_at(f_ilb, f_k, es, f_sbeg, x, y, npix);
                if (!(emu < 3.0e38f)) {
                    /* an infinite expected count would never leave the sampler's gamma loop */
                    if (lane == 0) atomicOr(P.err, 1ull);
                    finished = true;
                    break;
                }
                r.a = a;
                r.set_v(vb);
                c.ndraw = (int)r.poisson(emu);
                c.cur_ilb = eb.ilb;
                c.cur_im = eb.im;
                c.cur_iM = eb.iM;
                const float AmMin = gfc::beam_extinction(P.g, P.g.pixels[eb.ilb]);
                draw_stars(P, tid, lane, r, c.ndraw, nstars, limit, c.cur_ilb, c.cur_im, c.cur_iM, AmMin);
                v = r.v();
                if (c.ndraw) {
                    /* the table is full: pause right after the event bin, with its anchor */
                    long long fk = (long long)c.blk_k + (long long)f * step;
                    const int fdrift = __shfl_sync(0xffffffffu, dexcl, f);
                    c.blk_ilb = (int)((long long)c.blk_ilb + fk / kmax + fdrift);
                    c.blk_k = (int)(fk % kmax);
                    if (eb.anchor_s >= 0) {
                        const BinPos ab = bin_at(f_ilb, f_k, eb.anchor_s, 0, x, y, npix);
                        c.anc = anchor(P, P.g.pixels[ab.ilb], ab.im, ab.iM);
                    }
                    c.pos = es + 1;
                    break;
                }
                /* continue with the bins after the event */
                if (lane < f) lane_lo = GF_BLOCK;
                else if (lane == f) lane_lo = es + 1;
            }
            if (finished || c.ndraw) break;
        }
#undef MU
        if (end_mask) { finished = true; break; }
        /* next window: 32 blocks further */
        long long nk = (long long)c.blk_k + 32LL * step;
        c.blk_ilb = (int)((long long)c.blk_ilb + nk / kmax + dtot);
        c.blk_k = (int)(nk % kmax);
        c.pos = 0;
    }

    if (!DRAW) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cnt_sum += __shfl_xor_sync(0xffffffffu, cnt_sum, o);
            cov_sum += __shfl_xor_sync(0xffffffffu, cov_sum, o);
        }
        if (P.per_pixel && pp_ilb >= 0) atomicAdd(&P.per_pixel[pp_ilb + P.pix_base], pp_sum);
        if (lane == 0) {
            P.counts[tid] += cnt_sum;
            P.countsCovered[tid] += cov_sum;
        }
        return;
    }

    if (lane == 0) {
        st.status[tid] = finished ? 2 : 1;
        st.blk_ilb[tid] = c.blk_ilb; st.blk_k[tid] = c.blk_k; st.pos[tid] = c.pos;
        st.ndraw[tid] = c.ndraw;
        st.cur_ilb[tid] = c.cur_ilb; st.cur_im[tid] = c.cur_im; st.cur_iM[tid] = c.cur_iM;
        st.D[tid] = c.anc.D; st.Am[tid] = c.anc.Am; st.ms[tid] = c.anc.ms;
        st.nstars[tid] = nstars;
        const int NS = P.rng_nstreams;
        P.rng[NS + tid] = (uint32_t)(v >> 32);
        P.rng[2 * NS + tid] = (uint32_t)v;
    }
}

template <int DRAW>
__global__ void __launch_bounds__(128) crawl_kernel(CrawlParams P)
{
    extern __shared__ float s_lf[];
    __shared__ float s_mu[128 / 32][GF_BLOCK * 32];
    for (int i = threadIdx.x; i < P.m.lf_n; i += blockDim.x) s_lf[i] = P.m.lf[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int tid = P.stream_begin + warp; tid < P.stream_end; tid += nwarps)
        crawl_stream<DRAW>(P, s_lf, s_mu[threadIdx.x >> 5], tid, lane);
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

__global__ void __launch_bounds__(256) place_kernel(PlaceParams P)
{
    const double r2d = 57.2957795130823208767981548;
    unsigned vis_local = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += (int64_t)gridDim.x * blockDim.x) {
        const StarRecord rec = P.rec[i];
        const SkyModel &m = P.m;
        const gf_pencil_beam pix = P.g.pixels[rec.ilb];
        const int64_t n = P.n;
        float M = m.M1 - (float)rec.iM * m.dM;
        float x = pix.X, y = pix.Y;
        x += pix.dx * (rec.u[0] - 0.5f);
        y += pix.dx * (rec.u[1] - 0.5f);
        if (x * x + y * y > 2.f) {
            P.hidden[i] = 1;
            P.key[i] = ~0ull;
            continue;
        }
        P.projIdx[i] = pix.projIdx;
        P.projXY[i] = x;
        P.projXY[n + i] = y;
        double l, b;
        deproject(P.g.proj[pix.projIdx], l, b, x, y);
        float cl = (float)gfm::cos_d(l), cb = (float)gfm::cos_d(b);
        float sl = (float)gfm::sin_d(l), sb = (float)gfm::sin_d(b);
        l *= r2d;
        if (l < 0.) l += 360.;
        if (l > 360.) l -= 360.;
        b *= r2d;
        P.lb[i] = l;
        P.lb[n + i] = b;
        float Mtmp = M + m.dM * (rec.u[2] - 0.5f);
        float mtmp = m.m0 + m.dm * ((float)rec.im + rec.u[3] - 0.5f);
        float DM = mtmp - Mtmp;
        P.absmag[i] = Mtmp;
        P.DM[i] = DM;
        float D = gfm::powf_(10.f, 0.2f * DM + 1.f);
        P.XYZ[i] = D * cl * cb;
        P.XYZ[n + i] = D * sl * cb;
        P.XYZ[2 * n + i] = D * sb;
        float Am0 = (P.g.ext_kind == GF_EXT_SCREEN_CSCB) ? P.g.A0 / fabsf(sb) : 0.f;
        float AmInf = Am0;
        int hid = (mtmp + Am0 > m.m1) ? 1 : 0;
        if (rec.AmMin > Am0) AmInf = -rec.AmMin;
        P.Am[i] = Am0;
        P.AmInf[i] = AmInf;
        P.hidden[i] = hid;
        /* l >= 0 here (-0.0 compares equal to 0.0 and maps to key 0) */
        P.key[i] = hid ? ~0ull : (l == 0.0 ? 0ull : (uint64_t)__double_as_longlong(l));
        vis_local += hid ? 0u : 1u;
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

static int sm_count_cached = 0;
int sm_count()
{
    if (!sm_count_cached) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sm_count_cached, cudaDevAttrMultiProcessorCount, dev);
        if (sm_count_cached <= 0) sm_count_cached = 148;
    }
    return sm_count_cached;
}

static CrawlParams make_params(const LaunchCrawl &L)
{
    CrawlParams P;
    P.m = L.m;
    P.g = L.g;
    P.st = L.st;
    P.rng = L.rng;
    P.rng_nstreams = L.rng_nstreams;
    P.jt = L.jt;
    P.stream_begin = L.stream_begin;
    P.stream_end = L.stream_end;
    P.limits = L.limits;
    P.rec = L.rec;
    P.rec_capacity = L.rec_capacity;
    P.rec_count = L.rec_count;
    P.err = L.err;
    P.counts = L.counts;
    P.countsCovered = L.countsCovered;
    P.per_pixel = L.per_pixel;
    P.pix_base = L.pix_base;
    P.Dtab = L.Dtab;
    return P;
}

cudaError_t launch_crawl(const LaunchCrawl &L, int draw, cudaStream_t s)
{
    CrawlParams P = make_params(L);
    int nstreams = L.stream_end - L.stream_begin;
    if (nstreams <= 0) return cudaSuccess;
    const int threads = 128;
    int warps_per_block = threads / 32;
    int blocks = (nstreams + warps_per_block - 1) / warps_per_block;
    size_t smem = (size_t)L.m.lf_n * sizeof(float);
    if (draw) crawl_kernel<1><<<blocks, threads, smem, s>>>(P);
    else crawl_kernel<0><<<blocks, threads, smem, s>>>(P);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_place(const LaunchPlace &L, cudaStream_t s)
{
    if (L.n <= 0) return cudaSuccess;
    PlaceParams P;
    P.m = L.m; P.g = L.g; P.rec = L.rec; P.n = L.n;
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
    for (int l = 0; l < 32; l++) {
        hi[(size_t)s * 32 + l] = h;                       /* a^(32 l - 3) */
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
