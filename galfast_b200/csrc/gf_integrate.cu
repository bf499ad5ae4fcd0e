/*
 * gf_integrate.cu -- the expected-count (integrate) pass of many requests,
 * pixel by pixel.
 *
 * The reference integrates with the same crawl as the draw pass: stream t
 * takes blocks of 10 consecutive bins, and evaluates the model at an anchor
 * bin at every block start and every diagonal start (skygen.cu.h:469-611);
 * each later bin of the block reuses its anchor.  When nm * nM is a multiple
 * of 10 the blocks of every pixel start at the local indices k = 0, 10, 20 ...,
 * so the anchors of a pixel are the same positions in every pixel and in
 * every stream decomposition.  This pass computes every bin's expected count
 * with the reference's anchor and float expression, without the streams:
 *
 *   plan    (per magnitude grid) the anchor positions of each diagonal and the
 *           anchor's distance D[im][iM].  Along a diagonal the distance
 *           modulus is the same number rounded in a few different ways, so
 *           the anchors of a diagonal take only 1-4 distinct D; the plan lists
 *           the distinct values (the slots) and maps every anchor to its slot.
 *   pixels  (one warp per pixel) the model density at each slot's distance
 *           along the pixel's direction (the only anchor quantity that depends
 *           on D and the pixel), then one lane per diagonal walks its bins:
 *           mu = (((LF(M) * ms) * norm) * D^3) * K, bins with m + Am > m1 cut.
 *           Per pixel the counts and covered counts are summed in FP64.
 *   totals  (one CTA per request) the pixel sums in a fixed order.
 *
 * Every bin's mu is bit-identical to the crawl's; the totals differ from a
 * per-stream summation only by the order of the FP64 additions.
 */
#include "gf_crawl.cuh"
#include "gf_launch.h"

namespace gfk {

namespace {

/* first local index of diagonal d (cells before it) and its length, for an x-by-y grid */
__device__ __forceinline__ long long diag_start(int d, int x, int y)
{
    const long long l = x < y ? x : y, m = x < y ? y : x, n = x + y - 1 - (long long)d;
    if (d < l) return (long long)d * (d + 1) / 2;
    if (d < m) return l * (l + 1) / 2 + ((long long)d - l) * l;
    return (long long)x * y - n * (n + 1) / 2;
}

__device__ __forceinline__ int diag_len(int d, int x, int y)
{
    const int l = x < y ? x : y;
    int n = d + 1;
    n = n < l ? n : l;
    const int r = x + y - 1 - d;
    return n < r ? n : r;
}

/* first anchor after position 0 on a diagonal that starts at local index k0 */
__device__ __forceinline__ int first_block_start(long long k0)
{
    const int r = (int)(k0 % GF_BLOCK);
    return r == 0 ? GF_BLOCK : GF_BLOCK - r;
}

#define GF_PLAN_REMEMBER 8          /* distinct distances remembered per diagonal */

constexpr int kIntegChunk = 8;      /* pixels per run a warp takes from the shared counter */

/* distinct anchor distances of diagonal d, in order of first appearance; calls
 * emit(anchor ordinal, slot ordinal on the diagonal, D, local index, i, j) for every anchor */
template <class F>
__device__ __forceinline__ int diag_anchors(const float *Dtab, int nM_tab, int d, int x, int y, F emit)
{
    const long long k0 = diag_start(d, x, y);
    const int len = diag_len(d, x, y);
    const int i0 = d - (y - 1) > 0 ? d - (y - 1) : 0;
    uint32_t seen[GF_PLAN_REMEMBER];
    int nseen = 0, nslot = 0, q = 0;
    for (int t = 0; t < len; t = (t == 0 ? first_block_start(k0) : t + GF_BLOCK), q++) {
        const int i = i0 + t, j = d - i;
        const float D = Dtab[(size_t)i * nM_tab + j];
        const uint32_t b = __float_as_uint(D);
        int s = -1;
        for (int r = 0; r < nseen; r++)
            if (seen[r] == b) s = r;
        if (s < 0) {
            s = nslot++;
            if (nseen < GF_PLAN_REMEMBER) seen[nseen++] = b;
        }
        emit(q, s, D, k0 + t, i, j);
    }
    return nslot;
}

/* block-wide exclusive scan of two counters (blockDim.x = 1024) */
__device__ __forceinline__ void scan2(int &a, int &b, int *sa, int *sb, int &tot_a, int &tot_b)
{
    const int t = threadIdx.x;
    sa[t] = a;
    sb[t] = b;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
        int va = 0, vb = 0;
        if (t >= o) { va = sa[t - o]; vb = sb[t - o]; }
        __syncthreads();
        sa[t] += va;
        sb[t] += vb;
        __syncthreads();
    }
    tot_a = sa[blockDim.x - 1];
    tot_b = sb[blockDim.x - 1];
    a = sa[t] - a;
    b = sb[t] - b;
    __syncthreads();
}

/* byte layout of a plan (the header's offsets) */
__host__ __device__ inline void plan_layout(int nm, int nM, int max_anchors, int max_slots, IntegPlanHdr &h)
{
    const long long nd = (long long)nm + nM - 1, nb = (long long)nm * nM / GF_BLOCK;
    long long off = (sizeof(IntegPlanHdr) + 15) & ~15ll;
    off += (8 * nd + 15) & ~15ll;
    h.off_slot = (int32_t)off;
    off += (4 * (long long)max_slots + 15) & ~15ll;
    h.off_anc = (int32_t)off;
    off += (2 * (long long)max_anchors + 15) & ~15ll;
    h.off_blk = (int32_t)off;
    off += (4 * nb + 15) & ~15ll;
    h.off_bslot = (int32_t)off;
    off += (2 * nb + 15) & ~15ll;
    h.off_dslot = (int32_t)off;
    off += (2 * nd + 15) & ~15ll;
    h.off_binfo = (int32_t)off;
    off += (4 * nb + 15) & ~15ll;
    h.nd = (int32_t)nd;
    h.nblocks = (int32_t)nb;
    h.max_anchors = max_anchors;
    h.max_slots = max_slots;
    h.bytes = (int32_t)off;
    h.nanchors = 0;
    h.nslots = 0;
    h.ok = 0;
    h.pad[0] = h.pad[1] = 0;
}

__global__ void __launch_bounds__(1024) plan_kernel(const IntegPlanDesc *desc)
{
    __shared__ int sa[1024], sb[1024];
    const IntegPlanDesc P = desc[blockIdx.x];
    const int x = P.nm, y = P.nM, nd = x + y - 1;
    unsigned char *plan = P.plan;
    IntegPlanHdr h;
    plan_layout(x, y, P.max_anchors, P.max_slots, h);
    int2 *diag = (int2 *)(plan + ((sizeof(IntegPlanHdr) + 15) & ~15));
    float *slotD = (float *)(plan + h.off_slot);
    uint16_t *anc = (uint16_t *)(plan + h.off_anc);
    uint32_t *blk = (uint32_t *)(plan + h.off_blk);
    uint16_t *bslot = (uint16_t *)(plan + h.off_bslot);
    uint16_t *dslot = (uint16_t *)(plan + h.off_dslot);
    int base_a = 0, base_s = 0;
    bool overflow = false;
    for (int c0 = 0; c0 < nd; c0 += blockDim.x) {
        const int d = c0 + threadIdx.x;
        int na = 0, ns = 0;
        if (d < nd) ns = diag_anchors(P.Dtab, P.nM_tab, d, x, y, [&](int q, int, float, long long, int, int) { na = q + 1; });
        int ea = na, es = ns, ta = 0, ts = 0;
        scan2(ea, es, sa, sb, ta, ts);
        const int abase = base_a + ea, sbase = base_s + es;
        if (d < nd) {
            diag[d] = make_int2(abase, first_block_start(diag_start(d, x, y)));
            if (abase + na <= P.max_anchors && sbase + ns <= P.max_slots && sbase + ns <= 65536)
                diag_anchors(P.Dtab, P.nM_tab, d, x, y, [&](int q, int s, float D, long long k, int i, int j) {
                    const int slot = sbase + s;
                    anc[abase + q] = (uint16_t)slot;
                    slotD[slot] = D;
                    if (q == 0) dslot[d] = (uint16_t)slot;
                    if (k % GF_BLOCK == 0) {
                        blk[k / GF_BLOCK] = (uint32_t)i | ((uint32_t)j << 16);
                        bslot[k / GF_BLOCK] = (uint16_t)slot;
                    }
                });
            else
                overflow = true;
        }
        base_a += ta;
        base_s += ts;
    }
    overflow = __syncthreads_or(overflow);
    /* per block: its largest m row and its diagonal starts, from the block-start bins above */
    if (!overflow) {
        uint32_t *binfo = (uint32_t *)(plan + h.off_binfo);
        for (int b = threadIdx.x; b < h.nblocks; b += blockDim.x) {
            const uint32_t bij = blk[b];
            int i = (int)(bij & 0xffffu), j = (int)(bij >> 16);
            int imax = i;
            uint32_t wm = 0;
            for (int s = 1; s < GF_BLOCK; s++) {
                if (gfc::step_in_pixel(i, j, x, y)) wm |= 1u << s;
                imax = i > imax ? i : imax;
            }
            binfo[b] = (uint32_t)imax | (wm << 16);
        }
    }
    if (threadIdx.x == 0) {
        h.nanchors = base_a;
        h.nslots = base_s;
        h.ok = overflow ? 0 : 1;
        *(IntegPlanHdr *)plan = h;
    }
}

/* The lane's diagonals d = lane, lane + 32, ... of one pixel: every uncut bin's mu
 * from its anchor slot, summed in FP64 (and, when COV, mu * cf as well). */
template <bool COV>
__device__ __forceinline__ void walk_diagonals(int lane, int nd, int x, int y, int icut, const int2 *diag,
                                               const uint16_t *anc, const float *LFM, const float2 *Q, float norm,
                                               float K, float cf, double &cnt, double &cov)
{
    /* two partial sums per quantity (even and odd bins of each run) halve the chain of
     * dependent FP64 additions; they are added at the end, in a fixed order */
    double c0 = 0.0, c1 = 0.0, v0 = 0.0, v1 = 0.0;
    for (int d = lane; d < nd; d += 32) {
        const int i0 = d - (y - 1) > 0 ? d - (y - 1) : 0;
        int i1 = d < x - 1 ? d : x - 1;
        i1 = i1 < icut - 1 ? i1 : icut - 1;
        if (i1 < i0) continue;
        const int2 dg = diag[d];
        const uint16_t *ap = anc + dg.x;
        const float *lf = LFM + (d - i0);           /* LF of bin t of the diagonal: lf[-t] */
        const int tl = i1 - i0 + 1;
        int t = 0, seg_end = dg.y < tl ? dg.y : tl;
        for (;;) {
            const float2 q = Q[*ap++];
            if (q.y >= 0.f) {
                /* One code path for whole and partial segments (no divergence between
                 * lanes whose segments differ in length): bins u >= len read no LF and
                 * add an exact +0.0, so the sums take the segment's bins in the order
                 * of the plain loop (even offsets to c0, odd ones to c1). */
                const int len = seg_end - t;
                float mv[GF_BLOCK];
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] = u < len ? lf[-(t + u)] : 0.f;
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] *= q.x;
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] *= norm;
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] *= q.y;
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] *= K;
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u++) mv[u] = u < len ? mv[u] : 0.f;    /* 0 * inf would be NaN */
#pragma unroll
                for (int u = 0; u < GF_BLOCK; u += 2) {
                    c0 += (double)mv[u];
                    c1 += (double)mv[u + 1];
                    if (COV) {
                        v0 += (double)(mv[u] * cf);
                        v1 += (double)(mv[u + 1] * cf);
                    }
                }
            }
            t = seg_end;
            if (t >= tl) break;
            seg_end = t + GF_BLOCK < tl ? t + GF_BLOCK : tl;
        }
    }
    cnt += c0 + c1;
    if (COV) cov += v0 + v1;
}

/* One warp per pixel.  Per-warp shared tables: the request's model, LF at every
 * absolute-magnitude row, m at every apparent-magnitude row, and (ms, D^3) of
 * every slot of the pixel (D^3 = -inf marks an anchor outside [dmin, dmax)). */
template <int MODEL>
__global__ void __launch_bounds__(256) integrate_pixels_kernel(IntegPixParams P)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *mine = smem + (size_t)wib * P.warp_bytes;
    SkyModel &m = *(SkyModel *)mine;
    float *LFM = (float *)(mine + P.off_lf);
    float *MMr = (float *)(mine + P.off_mr);
    float2 *Q = (float2 *)(mine + P.off_q);
    int job = -1;
    const unsigned char *plan = nullptr;
    const int2 *diag = nullptr;
    const float *slotD = nullptr;
    const uint16_t *anc = nullptr;
    int nslots = 0;
    const gf_pencil_beam *pixels = nullptr;
    SkyGeom g;
    g.ext_kind = GF_EXT_NONE;
    g.ammin = nullptr;
    /* runs of kIntegChunk consecutive pixels (mostly of one request) taken from a
     * shared counter: the request's tables are set up once per run, not per pixel */
    int p = 0, pend = 0, job_end = 0;
    for (;;) {
        if (p >= pend) {
            unsigned u0 = 0;
            if (lane == 0) u0 = atomicAdd(P.next, (unsigned)kIntegChunk);
            u0 = __shfl_sync(0xffffffffu, u0, 0);
            if (u0 >= (unsigned)P.total_pix) break;
            p = (int)u0;
            pend = p + kIntegChunk < P.total_pix ? p + kIntegChunk : P.total_pix;
        } else {
            p++;
            if (p >= pend) continue;
        }
        /* the request of flat pixel p: pix_off is increasing */
        int lo = job;
        if (job < 0 || p < P.pix_off[job] || p >= job_end) {
            lo = 0;
            int hi = P.njobs;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (P.pix_off[mid] <= p) lo = mid; else hi = mid;
            }
        }
        if (lo != job) {
            job_end = P.pix_off[lo + 1];
            job = lo;
            plan = P.plans[job];
            if (plan) {
                __syncwarp();
                const uint32_t *src = (const uint32_t *)&P.jobs[job].m;
                for (int w = lane; w < (int)(sizeof(SkyModel) / 4); w += 32) ((uint32_t *)&m)[w] = src[w];
                __syncwarp();
                for (int q = lane; q < m.nM; q += 32) LFM[q] = gfc::lf_sample(m, m.lf, m.M1 - (float)q * m.dM);
                for (int q = lane; q < m.nm; q += 32) MMr[q] = m.m0 + m.dm * (float)q;
                const IntegPlanHdr *h = (const IntegPlanHdr *)plan;
                nslots = h->nslots;
                diag = (const int2 *)(plan + ((sizeof(IntegPlanHdr) + 15) & ~15));
                slotD = (const float *)(plan + h->off_slot);
                anc = (const uint16_t *)(plan + h->off_anc);
                pixels = P.jobs[job].g.pixels;
                g.ext_kind = P.jobs[job].g.ext_kind;
                g.ammin = P.jobs[job].g.ammin;
                __syncwarp();
            }
        }
        if (!plan) continue;
        const int ilb = p - (int)P.pix_off[job];
        const gf_pencil_beam pix = pixels[ilb];
        const float Am = gfc::beam_extinction(g, pix);
        const float K = pix.dA * GF_POGSON * m.dm * m.dM;
        const float cf = pix.coveredFraction;
        const float norm = m.norm, m1 = m.m1;
        const int x = m.nm, y = m.nM, nd = x + y - 1;
        const bool dlim = m.dmin != 0.f || m.dmax != 0.f;
        /* model density of every slot along this pixel's direction (anchor_x) */
        for (int s = lane; s < nslots; s += 32) {
            const float D = slotD[s];
            const float px = D * pix.cl * pix.cb;
            const float py = D * pix.sl * pix.cb;
            const float pz = D * pix.sb;
            const float ms = gfc::model_rho<MODEL>(m, px, py, pz);
            const bool dcut = dlim && (m.dmin > D || m.dmax <= D);
            Q[s] = make_float2(ms, dcut ? -__int_as_float(0x7f800000) : D * D * D);
        }
        /* apparent-magnitude rows at and after icut are cut (m0 + dm im is increasing in im) */
        int icut = x;
        for (int i = lane; i < x; i += 32)
            if (MMr[i] + Am > m1) { icut = i; break; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int t = __shfl_xor_sync(0xffffffffu, icut, o);
            icut = t < icut ? t : icut;
        }
        __syncwarp();
        double cnt = 0.0, cov = 0.0;
        if (cf == 1.0f) {
            /* fully covered pixel: mu * cf == mu, so the covered sum is the sum */
            walk_diagonals<false>(lane, nd, x, y, icut, diag, anc, LFM, Q, norm, K, cf, cnt, cov);
            cov = cnt;
        } else {
            walk_diagonals<true>(lane, nd, x, y, icut, diag, anc, LFM, Q, norm, K, cf, cnt, cov);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            cov += __shfl_xor_sync(0xffffffffu, cov, o);
        }
        if (lane == 0) P.pix_sum[p] = make_double2(cnt, cov);
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) job_totals_kernel(const double2 *pix_sum, const int32_t *pix_off,
                                                          const unsigned char *const *plans, double2 *tot)
{
    __shared__ double sc[256], sv[256];
    const int j = blockIdx.x;
    double c = 0.0, v = 0.0;
    if (plans[j])
        for (int p = pix_off[j] + threadIdx.x; p < pix_off[j + 1]; p += blockDim.x) {
            const double2 s = pix_sum[p];
            c += s.x;
            v += s.y;
        }
    sc[threadIdx.x] = c;
    sv[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sc[threadIdx.x] += sc[threadIdx.x + o];
            sv[threadIdx.x] += sv[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) tot[j] = make_double2(sc[0], sv[0]);
}

}  // namespace

size_t integ_plan_bytes(int nm, int nM, int *max_anchors, int *max_slots)
{
    const long long nd = (long long)nm + nM - 1;
    const long long na = (long long)nm * nM / GF_BLOCK + nd;
    *max_anchors = (int)std::min<long long>(na, 1ll << 30);
    *max_slots = (int)std::min<long long>(na, 65536);
    IntegPlanHdr h;
    plan_layout(nm, nM, *max_anchors, *max_slots, h);
    return (size_t)h.bytes;
}

cudaError_t launch_integ_plans(const IntegPlanDesc *desc_dev, int nplans, cudaStream_t s)
{
    if (nplans <= 0) return cudaSuccess;
    plan_kernel<<<nplans, 1024, 0, s>>>(desc_dev);
    count_launches(1);
    return cudaGetLastError();
}

size_t integ_warp_bytes(int nm_max, int nM_max, int slots_max, IntegPixParams *P)
{
    size_t off = (sizeof(SkyModel) + 15) & ~(size_t)15;
    P->off_lf = (int32_t)off;
    off += ((size_t)4 * nM_max + 15) & ~(size_t)15;
    P->off_mr = (int32_t)off;
    off += ((size_t)4 * nm_max + 15) & ~(size_t)15;
    P->off_q = (int32_t)off;
    off += (size_t)8 * slots_max;
    off = (off + 15) & ~(size_t)15;
    P->warp_bytes = (int32_t)off;
    return off;
}

cudaError_t launch_integrate_pixels(const IntegPixParams &P, int model_type, double2 *tot, cudaStream_t s)
{
    if (P.total_pix <= 0) return cudaSuccess;
    if (!P.next) return cudaErrorInvalidValue;
    const size_t max_smem = 200 * 1024;
    int wpb = (int)std::min<size_t>(8, max_smem / (size_t)P.warp_bytes);
    if (wpb < 1) return cudaErrorInvalidValue;
    const size_t smem = (size_t)wpb * P.warp_bytes;
    const int threads = 32 * wpb;
    cudaError_t e;
    int per_sm = 0;
    if (model_type == GF_MODEL_EXP_DISK) {
        e = cudaFuncSetAttribute(integrate_pixels_kernel<GF_MODEL_EXP_DISK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, integrate_pixels_kernel<GF_MODEL_EXP_DISK>, threads, smem);
    } else {
        e = cudaFuncSetAttribute(integrate_pixels_kernel<GF_MODEL_POWER_LAW_ELLIPSOID>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, integrate_pixels_kernel<GF_MODEL_POWER_LAW_ELLIPSOID>, threads, smem);
    }
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    const long long need = ((long long)P.total_pix + wpb * kIntegChunk - 1) / (wpb * kIntegChunk);
    const int blocks = (int)std::min<long long>(need, (long long)sm_count() * per_sm);
    e = cudaMemsetAsync(P.next, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (model_type == GF_MODEL_EXP_DISK)
        integrate_pixels_kernel<GF_MODEL_EXP_DISK><<<blocks, threads, smem, s>>>(P);
    else
        integrate_pixels_kernel<GF_MODEL_POWER_LAW_ELLIPSOID><<<blocks, threads, smem, s>>>(P);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    job_totals_kernel<<<P.njobs, 256, 0, s>>>(P.pix_sum, P.pix_off, P.plans, tot);
    count_launches(1);
    return cudaGetLastError();
}

}  // namespace gfk
