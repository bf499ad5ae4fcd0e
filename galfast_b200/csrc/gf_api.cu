/*
 * gf_api.cu -- the C ABI (include/galfast_b200.h) and the host orchestration
 * of the catalog path on one B200.
 */
#include "gf_ctx.h"
#include "gf_host.h"
#include "gf_safeprimes.h"

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>

namespace gfa {

thread_local std::string g_err;

/* allocation failures arranged by gf_debug_fail_allocations: the allocations
 * after the next g_fail_after ones fail, g_fail_count of them (0: all) */
static std::atomic<long long> g_fail_after(-1), g_fail_count(0), g_alloc_seen(0);

void set_alloc_failures(long long after, long long count)
{
    g_fail_after.store(-1);
    g_alloc_seen.store(0);
    g_fail_count.store(count);
    g_fail_after.store(after < 0 ? -1 : after);
}

void release_caches(gf_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    gf_table_free(ctx, &ctx->plain_table);
    free_multi_ws(ctx);
    free_rec_cache(ctx);
}

cudaError_t device_malloc(void **p, size_t bytes)
{
    *p = nullptr;
    const long long after = g_fail_after.load();
    if (after >= 0) {
        const long long k = g_alloc_seen.fetch_add(1);
        const long long cnt = g_fail_count.load();
        if (k >= after && (cnt == 0 || k < after + cnt)) return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

gf_status fail(gf_status s, const std::string &msg)
{
    g_err = msg;
    return s;
}

gf_status zero_module_rows(gf_ctx *ctx, const gf_table *t, int64_t n)
{
    if (n <= 0) return GF_OK;
    const size_t P = (size_t)t->capacity, m = (size_t)n;
    cudaStream_t st = ctx->stream;
    auto z = [&](void *p, size_t elem, size_t ncomp) -> gf_status {
        if (!p || ncomp == 0) return GF_OK;
        GF_CUDA(cudaMemset2DAsync(p, P * elem, 0, m * elem, ncomp, st));
        return GF_OK;
    };
    GF_TRY(z(t->FeH, 4, 1));
    GF_TRY(z(t->vcyl, 4, 3));
    GF_TRY(z(t->mags, 4, (size_t)t->nbands));
    GF_TRY(z(t->photoflags, 4, 1));
    GF_TRY(z(t->obsmags, 4, (size_t)t->nbands));
    GF_TRY(z(t->pm, 4, 3));
    GF_TRY(z(t->radec, 8, 2));
    GF_TRY(z(t->FeH_comp, 4, 1));
    GF_TRY(z(t->absmagSys, 4, 2));
    GF_TRY(z(t->absmagSysNcomp, 4, 1));
    return GF_OK;
}

gf_status check_ctx(gf_ctx *ctx)
{
    if (!ctx) return fail(GF_E_INVALID, "null context");
    GF_CUDA(cudaSetDevice(ctx->device));
    return GF_OK;
}

gf_status ensure_multipliers(gf_ctx *ctx)
{
    if (ctx->d_mult) return GF_OK;
    const std::vector<uint32_t> &mult = gfh::multipliers();
    GF_TRY(dev_alloc(&ctx->d_mult, GF_MAX_STREAMS));
    GF_CUDA(cudaMemcpy(ctx->d_mult, mult.data(), 4 * (size_t)GF_MAX_STREAMS, cudaMemcpyHostToDevice));
    GF_TRY(dev_alloc(&ctx->jt.lo, (size_t)GF_MAX_STREAMS * 32));
    GF_TRY(dev_alloc(&ctx->jt.hi, (size_t)GF_MAX_STREAMS * GF_JUMP_HI));
    GF_CUDA(gfk::launch_jump_tables(ctx->d_mult, GF_MAX_STREAMS, ctx->jt.lo, ctx->jt.hi, ctx->stream));
    return GF_OK;
}

}  // namespace gfa

using gfa::fail;
using gfa::dev_alloc;
using gfa::dev_free;
using gfa::check_ctx;
using gfa::ProfScope;

namespace gfk {
void set_last_error(const std::string &msg) { gfa::g_err = msg; }
}

struct ModelState {
    gfh::HostModel hm;
    float *d_lf = nullptr;
    float *d_cube = nullptr;                 /* density cube (GF_MODEL_DENSITY_CUBE) */
    float *d_Dtab = nullptr;                 /* D[im][iM] */
    bool crawl_init = false;
    bool done = false;
    CrawlState st{};
    CrawlState snap{};
    void *st_mem = nullptr, *snap_mem = nullptr;
    double expected = 0, expected_covered = 0;
    int64_t drawn = 0;
    std::vector<double> stream_expected;     /* per-stream expected stars (integrate pass) */
    std::vector<int64_t> stream_drawn;       /* stars drawn per stream so far */
    int first_active = 0;                    /* streams before it have finished */
};

struct gf_skygen {
    gf_ctx *ctx = nullptr;
    gf_skygen_config cfg{};
    SkyGeom geom{};
    gf_pencil_beam *d_pixels = nullptr;
    float *d_ammin = nullptr;
    std::vector<ModelState> models;
    /* per-launch buffers */
    int64_t *d_limits = nullptr;
    int64_t *h_nstars = nullptr;         /* pinned [nthreads] */
    uint32_t *d_rng_snap = nullptr;      /* [3][nthreads] */
    StarRecord *d_rec = nullptr, *d_rec2 = nullptr;
    float *d_rec_am = nullptr, *d_rec_am2 = nullptr;   /* GF_EXT_MAPS: anchor extinction per record */
    bool maps = false;                                 /* GF_EXT_MAPS: the records carry their anchor's extinction */
    float *d_map[2] = {nullptr, nullptr};              /* device copies of the extinction maps */
    int64_t rec_cap = 0;
    /* placement + sort buffers (rec_cap rows) */
    double *d_lb = nullptr;
    int32_t *d_projIdx = nullptr, *d_hidden = nullptr;
    float *d_projXY = nullptr, *d_DM = nullptr, *d_absmag = nullptr, *d_XYZ = nullptr, *d_Am = nullptr, *d_AmInf = nullptr;
    uint64_t *d_key = nullptr, *d_key2 = nullptr;
    uint32_t *d_idx = nullptr, *d_idx2 = nullptr;
    void *d_sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    int nthreads = 0;
    /* checkpoints of the last speculative window (see gf_skygen_draw) */
    Checkpoint *d_ck = nullptr;
    int32_t ck_cap = 0;
    uint32_t *d_ck_count = nullptr;
    unsigned long long *d_ck_sel = nullptr;
    int64_t *d_keep = nullptr;
};

namespace {

/* CrawlState arrays carved from one allocation */
size_t crawl_state_bytes(int n) { return (size_t)n * (8 * 4 + 16 + 8) + 256; }

gf_status alloc_crawl_state(int n, CrawlState &st, void **mem)
{
    GF_CUDA(gfa::device_malloc(mem, crawl_state_bytes(n)));
    char *p = (char *)*mem;
    auto take = [&](size_t bytes) { char *r = p; p += (bytes + 15) & ~(size_t)15; return r; };
    st.anc = (AnchorX *)take(16 * (size_t)n);
    st.nstars = (int64_t *)take(8 * (size_t)n);
    st.status = (int32_t *)take(4 * (size_t)n);
    st.blk_ilb = (int32_t *)take(4 * (size_t)n);
    st.blk_k = (int32_t *)take(4 * (size_t)n);
    st.pos = (int32_t *)take(4 * (size_t)n);
    st.ndraw = (int32_t *)take(4 * (size_t)n);
    st.cur_ilb = (int32_t *)take(4 * (size_t)n);
    st.cur_im = (int32_t *)take(4 * (size_t)n);
    st.cur_iM = (int32_t *)take(4 * (size_t)n);
    return GF_OK;
}

/* The record and placement buffers of a finished generator, kept by its context:
 * every gf_catalog_run creates a generator, and allocating and freeing these
 * gigabytes per request costs device synchronisations and, now and then, much more. */
/* move the buffer set of src (a generator or a cached set) to dst */
template <class A, class B>
void move_recs(A &dst, B &src)
{
    dst.d_rec = src.d_rec; dst.d_rec2 = src.d_rec2; dst.d_rec_am = src.d_rec_am; dst.d_rec_am2 = src.d_rec_am2;
    dst.d_lb = src.d_lb; dst.d_projIdx = src.d_projIdx; dst.d_hidden = src.d_hidden; dst.d_projXY = src.d_projXY;
    dst.d_DM = src.d_DM; dst.d_absmag = src.d_absmag; dst.d_XYZ = src.d_XYZ; dst.d_Am = src.d_Am; dst.d_AmInf = src.d_AmInf;
    dst.d_key = src.d_key; dst.d_key2 = src.d_key2; dst.d_idx = src.d_idx; dst.d_idx2 = src.d_idx2;
    dst.d_sort_temp = src.d_sort_temp; dst.sort_temp_bytes = src.sort_temp_bytes; dst.rec_cap = src.rec_cap;
    src.d_rec = src.d_rec2 = nullptr; src.d_rec_am = src.d_rec_am2 = nullptr; src.d_lb = nullptr;
    src.d_projIdx = src.d_hidden = nullptr; src.d_projXY = src.d_DM = src.d_absmag = src.d_XYZ = src.d_Am = src.d_AmInf = nullptr;
    src.d_key = src.d_key2 = nullptr; src.d_idx = src.d_idx2 = nullptr; src.d_sort_temp = nullptr;
    src.sort_temp_bytes = 0; src.rec_cap = 0;
}

/* a cached buffer set, with the generator's field names */
struct RecView {
    StarRecord *d_rec = nullptr, *d_rec2 = nullptr;
    float *d_rec_am = nullptr, *d_rec_am2 = nullptr;
    double *d_lb = nullptr;
    int32_t *d_projIdx = nullptr, *d_hidden = nullptr;
    float *d_projXY = nullptr, *d_DM = nullptr, *d_absmag = nullptr, *d_XYZ = nullptr, *d_Am = nullptr, *d_AmInf = nullptr;
    uint64_t *d_key = nullptr, *d_key2 = nullptr;
    uint32_t *d_idx = nullptr, *d_idx2 = nullptr;
    void *d_sort_temp = nullptr;
    size_t sort_temp_bytes = 0;
    int64_t rec_cap = 0;
};

void free_recs(RecView &v)
{
    dev_free(v.d_rec); dev_free(v.d_rec2); dev_free(v.d_rec_am); dev_free(v.d_rec_am2);
    dev_free(v.d_lb); dev_free(v.d_projIdx); dev_free(v.d_hidden);
    dev_free(v.d_projXY); dev_free(v.d_DM); dev_free(v.d_absmag); dev_free(v.d_XYZ);
    dev_free(v.d_Am); dev_free(v.d_AmInf);
    dev_free(v.d_key); dev_free(v.d_key2); dev_free(v.d_idx); dev_free(v.d_idx2);
    if (v.d_sort_temp) cudaFree(v.d_sort_temp);
    v.d_sort_temp = nullptr;
    v.rec_cap = 0;
}

}  // namespace

namespace gfa {
void free_rec_cache(gf_ctx *ctx)
{
    if (!ctx || !ctx->rec_cache) return;
    RecView *c = (RecView *)ctx->rec_cache;
    free_recs(*c);
    delete c;
    ctx->rec_cache = nullptr;
}
}  // namespace gfa

namespace {

gf_status ensure_rec_capacity(gf_skygen *s, int64_t need, int64_t keep)
{
    if (need <= s->rec_cap) return GF_OK;
    if (s->rec_cap == 0 && !s->d_rec && keep == 0 && s->ctx->rec_cache) {
        /* a fresh generator adopts its context's buffers when they are large enough */
        RecView &c = *(RecView *)s->ctx->rec_cache;
        if (c.rec_cap >= need && (!s->maps || (c.d_rec_am && c.d_rec_am2))) {
            move_recs(*s, c);
            return GF_OK;
        }
    }
    int64_t cap = std::max<int64_t>(need, s->rec_cap * 3 / 2);
    cap = std::max<int64_t>(cap, 4096);
    StarRecord *old = s->d_rec;
    float *old_am = s->d_rec_am;
    s->d_rec = nullptr;
    s->d_rec_am = nullptr;
    if (keep > 0 && old) {
        StarRecord *nr = nullptr;
        GF_TRY(dev_alloc(&nr, cap));
        GF_CUDA(cudaMemcpyAsync(nr, old, sizeof(StarRecord) * (size_t)keep, cudaMemcpyDeviceToDevice, s->ctx->stream));
        if (s->maps && old_am) {
            float *na = nullptr;
            GF_TRY(dev_alloc(&na, cap));
            GF_CUDA(cudaMemcpyAsync(na, old_am, 4 * (size_t)keep, cudaMemcpyDeviceToDevice, s->ctx->stream));
            s->d_rec_am = na;
        }
        GF_CUDA(cudaStreamSynchronize(s->ctx->stream));
        dev_free(old);
        s->d_rec = nr;
    } else {
        dev_free(old);
    }
    dev_free(old_am);
    dev_free(s->d_rec2);
    dev_free(s->d_rec_am2);
    dev_free(s->d_lb); dev_free(s->d_projIdx); dev_free(s->d_hidden);
    dev_free(s->d_projXY); dev_free(s->d_DM); dev_free(s->d_absmag); dev_free(s->d_XYZ);
    dev_free(s->d_Am); dev_free(s->d_AmInf);
    dev_free(s->d_key); dev_free(s->d_key2); dev_free(s->d_idx); dev_free(s->d_idx2);
    if (s->d_sort_temp) cudaFree(s->d_sort_temp);
    s->d_sort_temp = nullptr;
    s->rec_cap = 0;
    if (!s->d_rec) GF_TRY(dev_alloc(&s->d_rec, cap));
    GF_TRY(dev_alloc(&s->d_rec2, cap));
    if (s->maps) {
        if (!s->d_rec_am) GF_TRY(dev_alloc(&s->d_rec_am, cap));
        GF_TRY(dev_alloc(&s->d_rec_am2, cap));
    }
    GF_TRY(dev_alloc(&s->d_lb, 2 * cap));
    GF_TRY(dev_alloc(&s->d_projIdx, cap));
    GF_TRY(dev_alloc(&s->d_hidden, cap));
    GF_TRY(dev_alloc(&s->d_projXY, 2 * cap));
    GF_TRY(dev_alloc(&s->d_DM, cap));
    GF_TRY(dev_alloc(&s->d_absmag, cap));
    GF_TRY(dev_alloc(&s->d_XYZ, 3 * cap));
    GF_TRY(dev_alloc(&s->d_Am, cap));
    GF_TRY(dev_alloc(&s->d_AmInf, cap));
    GF_TRY(dev_alloc(&s->d_key, cap));
    GF_TRY(dev_alloc(&s->d_key2, cap));
    GF_TRY(dev_alloc(&s->d_idx, cap));
    GF_TRY(dev_alloc(&s->d_idx2, cap));
    size_t tb = 0;
    GF_CUDA(gfk::sort_temp_bytes(cap, &tb));
    GF_CUDA(gfa::device_malloc(&s->d_sort_temp, tb + 256));
    s->sort_temp_bytes = tb + 256;
    s->rec_cap = cap;
    return GF_OK;
}

gfk::LaunchCrawl crawl_launch(gf_skygen *s, ModelState &ms)
{
    gfk::LaunchCrawl L;
    memset(&L, 0, sizeof(L));
    L.m = ms.hm.m;
    L.m.lf = ms.d_lf;
    L.g = s->geom;
    L.st = ms.st;
    L.rng = s->ctx->d_rng;
    L.rng_nstreams = s->ctx->rng_nstreams;
    L.jt = s->ctx->jt;
    L.stream_begin = 0;
    L.stream_end = s->nthreads;
    L.limits = s->d_limits;
    L.rec = s->d_rec;
    L.rec_am = s->d_rec_am;
    L.rec_capacity = s->rec_cap;
    L.rec_count = s->ctx->d_counters;
    L.err = s->ctx->d_counters + 2;
    L.Dtab = ms.d_Dtab;
    return L;
}

/* copy streams [a, b) of the crawl state and of the crawl streams between live and snapshot */
__global__ void copy_state_range(CrawlState dst, CrawlState src, uint32_t *rng_dst, int32_t dst_pitch,
                                 const uint32_t *rng_src, int32_t src_pitch, int32_t a, int32_t b)
{
    int i = a + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b) return;
    dst.status[i] = src.status[i]; dst.blk_ilb[i] = src.blk_ilb[i]; dst.blk_k[i] = src.blk_k[i]; dst.pos[i] = src.pos[i];
    dst.ndraw[i] = src.ndraw[i]; dst.cur_ilb[i] = src.cur_ilb[i]; dst.cur_im[i] = src.cur_im[i]; dst.cur_iM[i] = src.cur_iM[i];
    dst.anc[i] = src.anc[i]; dst.nstars[i] = 0;
    for (int k = 0; k < 3; k++) rng_dst[(size_t)k * dst_pitch + i] = rng_src[(size_t)k * src_pitch + i];
}

__global__ void fill_range(int64_t *p, int n, int a, int b, int64_t v)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && i >= a && i < b) p[i] = v;
}

gf_status snapshot_range(gf_skygen *s, ModelState &ms, int a, int b, bool restore)
{
    if (b <= a) return GF_OK;
    const int N = s->nthreads, NS = s->ctx->rng_nstreams;
    int blocks = (b - a + 255) / 256;
    if (restore)
        copy_state_range<<<blocks, 256, 0, s->ctx->stream>>>(ms.st, ms.snap, s->ctx->d_rng, NS, s->d_rng_snap, N, a, b);
    else
        copy_state_range<<<blocks, 256, 0, s->ctx->stream>>>(ms.snap, ms.st, s->d_rng_snap, N, s->ctx->d_rng, NS, a, b);
    GF_CUDA(cudaGetLastError());
    return GF_OK;
}

/* keep the records of streams before t, and the first keep_t[0] stars of stream t */
__global__ void filter_records(const StarRecord *in, const float *in_am, int64_t n, int32_t t, const int64_t *keep_t,
                               StarRecord *out, float *out_am, unsigned long long *count)
{
    const int64_t kt = *keep_t;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        StarRecord r = in[i];
        if (r.stream < t || (r.stream == t && (int64_t)r.seq < kt)) {
            unsigned long long k = atomicAdd(count, 1ull);
            out[k] = r;
            if (in_am) out_am[k] = in_am[i];
        }
    }
}

/* ---- checkpoints: resume a stream just before one of its bins with stars ---- */
__device__ void apply_checkpoint(const Checkpoint &ck, int s, CrawlState st, uint32_t *rng, int32_t NS)
{
    st.status[s] = 1;
    st.blk_ilb[s] = ck.blk_ilb;
    st.blk_k[s] = ck.blk_k;
    st.pos[s] = ck.pos;
    st.ndraw[s] = 0;
    st.anc[s] = ck.anc;
    st.nstars[s] = ck.nstars;
    rng[(size_t)NS + s] = (uint32_t)(ck.v >> 32);
    rng[2 * (size_t)NS + s] = (uint32_t)ck.v;
}

/* the latest checkpoint of stream t with at most Lt stars before it */
__global__ void select_checkpoint(const Checkpoint *ck, const uint32_t *count, int32_t cap, int32_t t, int64_t Lt,
                                  unsigned long long *sel)
{
    const uint32_t n = min(*count, (uint32_t)cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Checkpoint &c = ck[i];
        if (c.stream == t && (int64_t)c.nstars <= Lt)
            atomicMax(sel, ((unsigned long long)(c.nstars + 1) << 32) | i);
    }
}

/* stream t resumes from its selected checkpoint, or from the window snapshot if it has none;
 * keep[0] = the number of its stars that stay in the batch */
__global__ void resume_boundary_stream(const Checkpoint *ck, const unsigned long long *sel, int32_t t, CrawlState st,
                                       CrawlState snap, uint32_t *rng, int32_t NS, const uint32_t *rng_snap, int32_t N,
                                       int64_t *keep)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const unsigned long long sv = *sel;
    if (sv) {
        const Checkpoint c = ck[(uint32_t)sv];
        apply_checkpoint(c, t, st, rng, NS);
        *keep = c.nstars;
    } else {
        st.status[t] = snap.status[t]; st.blk_ilb[t] = snap.blk_ilb[t]; st.blk_k[t] = snap.blk_k[t]; st.pos[t] = snap.pos[t];
        st.ndraw[t] = snap.ndraw[t]; st.cur_ilb[t] = snap.cur_ilb[t]; st.cur_im[t] = snap.cur_im[t]; st.cur_iM[t] = snap.cur_iM[t];
        st.anc[t] = snap.anc[t]; st.nstars[t] = 0;
        for (int k = 0; k < 3; k++) rng[(size_t)k * NS + t] = rng_snap[(size_t)k * N + t];
        *keep = 0;
    }
}

/* first batch: streams in (t, w_hi) go back to their first bin with stars */
__global__ void resume_at_first_star(const Checkpoint *ck, const uint32_t *count, int32_t cap, int32_t t, int32_t w_hi,
                                     CrawlState st, uint32_t *rng, int32_t NS)
{
    const uint32_t n = min(*count, (uint32_t)cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Checkpoint c = ck[i];
        if (c.stream > t && c.stream < w_hi && c.nstars == 0) apply_checkpoint(c, c.stream, st, rng, NS);
    }
}

__global__ void set_limits(int64_t *lim, int n, int32_t t, int64_t Lt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    lim[i] = (i < t) ? 0 : (i == t ? Lt : 0);
}

}  // namespace

extern "C" {

const char *gf_last_error(void) { return gfa::g_err.c_str(); }

gf_status gf_ctx_create(int device, gf_ctx **out)
{
    if (!out) return fail(GF_E_INVALID, "null output");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return fail(GF_E_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) return fail(GF_E_INVALID, "device index out of range");
    GF_CUDA(cudaSetDevice(device));
    gf_ctx *c = new gf_ctx();
    c->device = device;
    cudaError_t ce = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = gfa::device_malloc((void **)&c->d_counters, 64);
    if (ce == cudaSuccess) ce = cudaMallocHost(&c->h_counters, 64);
    if (ce != cudaSuccess) {
        delete c;
        return fail(GF_E_CUDA, std::string("context setup: ") + cudaGetErrorString(ce));
    }
    *out = c;
    return GF_OK;
}

gf_status gf_ctx_destroy(gf_ctx *ctx)
{
    if (!ctx) return GF_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    gfa::free_multi_ws(ctx);
    gfa::free_rec_cache(ctx);
    gf_table_free(ctx, &ctx->plain_table);
    dev_free(ctx->d_rng);
    dev_free(ctx->d_mult);
    dev_free(ctx->jt.lo);
    dev_free(ctx->jt.hi);
    dev_free(ctx->d_counters);
    if (ctx->h_counters) cudaFreeHost(ctx->h_counters);
    for (auto &e : ctx->ev) if (e) cudaEventDestroy(e);
    for (auto &p : ctx->prof_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
    for (auto &e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return GF_OK;
}

gf_status gf_ctx_sync(gf_ctx *ctx)
{
    GF_TRY(check_ctx(ctx));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    return GF_OK;
}

gf_status gf_ctx_mark(gf_ctx *ctx, int32_t slot)
{
    GF_TRY(check_ctx(ctx));
    if (slot < 0 || slot >= 16) return fail(GF_E_INVALID, "event slot out of range");
    if (!ctx->ev[slot]) GF_CUDA(cudaEventCreate(&ctx->ev[slot]));
    GF_CUDA(cudaEventRecord(ctx->ev[slot], ctx->stream));
    return GF_OK;
}

gf_status gf_ctx_elapsed(gf_ctx *ctx, int32_t from, int32_t to, float *ms)
{
    GF_TRY(check_ctx(ctx));
    if (from < 0 || from >= 16 || to < 0 || to >= 16 || !ctx->ev[from] || !ctx->ev[to] || !ms)
        return fail(GF_E_INVALID, "event slots not recorded");
    GF_CUDA(cudaEventSynchronize(ctx->ev[to]));
    GF_CUDA(cudaEventElapsedTime(ms, ctx->ev[from], ctx->ev[to]));
    return GF_OK;
}

int64_t gf_launch_count(void) { return gfk::launches(); }

gf_status gf_profile_enable(gf_ctx *ctx, int32_t on)
{
    GF_TRY(check_ctx(ctx));
    ctx->prof = on != 0;
    return GF_OK;
}

gf_status gf_profile_read(gf_ctx *ctx, double *ms, int64_t *launches)
{
    GF_TRY(check_ctx(ctx));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    for (auto &p : ctx->prof_pending) {
        float t = 0.f;
        cudaEventElapsedTime(&t, p.second.first, p.second.second);
        ctx->prof_ms[p.first] += t;
        ctx->prof_n[p.first] += 1;
        ctx->ev_pool.push_back(p.second.first);
        ctx->ev_pool.push_back(p.second.second);
    }
    ctx->prof_pending.clear();
    for (int i = 0; i < GF_PROF_NPHASES; i++) {
        if (ms) ms[i] = ctx->prof_ms[i];
        if (launches) launches[i] = ctx->prof_n[i];
        ctx->prof_ms[i] = 0;
        ctx->prof_n[i] = 0;
    }
    return GF_OK;
}

gf_status gf_rng_init(gf_ctx *ctx, uint32_t seed48, int32_t nstreams)
{
    GF_TRY(check_ctx(ctx));
    if (nstreams <= 0 || nstreams > GF_MAX_STREAMS) return fail(GF_E_INVALID, "nstreams must be in [1, 65536]");
    if (nstreams % 64) nstreams += 64 - nstreams % 64;     /* roundUpModulo (cuda_rng.h:468) */
    const std::vector<uint32_t> &mult = gfh::multipliers();
    GF_TRY(gfa::ensure_multipliers(ctx));
    std::vector<uint32_t> h(3 * (size_t)nstreams);
    gfh::seed_streams(seed48, nstreams, mult.data(), h.data());
    if (ctx->rng_nstreams != nstreams) {
        dev_free(ctx->d_rng);
        GF_TRY(dev_alloc(&ctx->d_rng, 3 * (size_t)nstreams));
        ctx->rng_nstreams = nstreams;
    }
    GF_CUDA(cudaMemcpyAsync(ctx->d_rng, h.data(), 4 * h.size(), cudaMemcpyHostToDevice, ctx->stream));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    return GF_OK;
}

gf_status gf_rng_get_state(gf_ctx *ctx, uint32_t *host_state, int32_t nstreams)
{
    GF_TRY(check_ctx(ctx));
    if (nstreams != ctx->rng_nstreams) return fail(GF_E_INVALID, "stream count mismatch");
    GF_CUDA(cudaMemcpyAsync(host_state, ctx->d_rng, 12 * (size_t)nstreams, cudaMemcpyDeviceToHost, ctx->stream));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    return GF_OK;
}

gf_status gf_rng_set_state(gf_ctx *ctx, const uint32_t *host_state, int32_t nstreams)
{
    GF_TRY(check_ctx(ctx));
    if (nstreams != ctx->rng_nstreams) return fail(GF_E_INVALID, "stream count mismatch");
    GF_CUDA(cudaMemcpyAsync(ctx->d_rng, host_state, 12 * (size_t)nstreams, cudaMemcpyHostToDevice, ctx->stream));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    return GF_OK;
}

gf_status gf_rng_poisson(gf_ctx *ctx, uint32_t state[3], const float *mu, int32_t n, uint32_t *out)
{
    GF_TRY(check_ctx(ctx));
    if (!state || n < 0 || (n > 0 && (!mu || !out))) return fail(GF_E_INVALID, "invalid gf_rng_poisson arguments");
    if (state[0] == 0) return fail(GF_E_INVALID, "stream multiplier must be nonzero");
    for (int32_t i = 0; i < n; i++)
        if (!(mu[i] >= 0.f && mu[i] < 1e7f)) return fail(GF_E_INVALID, "Poisson means must be in [0, 1e7)");
    uint32_t *d_st = nullptr, *d_out = nullptr;
    float *d_mu = nullptr;
    gf_status st = dev_alloc(&d_st, 3);
    if (st == GF_OK) st = dev_alloc(&d_mu, (size_t)n + 1);
    if (st == GF_OK) st = dev_alloc(&d_out, (size_t)n + 1);
    if (st == GF_OK) {
        cudaError_t e = cudaMemcpyAsync(d_st, state, 12, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && n) e = cudaMemcpyAsync(d_mu, mu, 4 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = gfk::launch_poisson_stream(d_st, d_mu, n, d_out, ctx->stream);
        if (e == cudaSuccess && n) e = cudaMemcpyAsync(out, d_out, 4 * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(state, d_st, 12, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = fail(GF_E_CUDA, std::string("gf_rng_poisson: ") + cudaGetErrorString(e));
    }
    cudaStreamSynchronize(ctx->stream);
    dev_free(d_st);
    dev_free(d_mu);
    dev_free(d_out);
    return st;
}

gf_status gf_skygen_destroy(gf_skygen *s);

gf_status gf_skygen_create(gf_ctx *ctx, const gf_skygen_config *cfg, const gf_pencil_beam *pixels, int32_t npixels,
                           const float *beam_ammin, const gf_extinction *ext, const gf_model_config *models,
                           int32_t nmodels, gf_skygen **out)
{
    GF_TRY(check_ctx(ctx));
    if (!cfg || !pixels || npixels <= 0 || !models || nmodels <= 0 || !out) return fail(GF_E_INVALID, "invalid skygen arguments");
    for (int i = 0; i < npixels; i++) {
        if (pixels[i].projIdx < 0 || pixels[i].projIdx > 1) return fail(GF_E_INVALID, "pixel projIdx must be 0 or 1");
        if (beam_ammin && (pixels[i].extIdx < 0 || pixels[i].extIdx >= npixels)) return fail(GF_E_INVALID, "pixel extIdx out of range");
    }
    std::vector<gfh::HostModel> hms;
    std::string err;
    if (!gfh::setup_models(*cfg, npixels, models, nmodels, hms, err)) return fail(GF_E_INVALID, err);
    gf_skygen *s = new gf_skygen();
    s->ctx = ctx;
    s->cfg = *cfg;
    s->nthreads = cfg->nthreads;
    gf_status st = GF_OK;
    auto bail = [&](gf_status code) { gf_skygen_destroy(s); return code; };
    if ((st = dev_alloc(&s->d_pixels, npixels)) != GF_OK) return bail(st);
    cudaMemcpy(s->d_pixels, pixels, sizeof(gf_pencil_beam) * (size_t)npixels, cudaMemcpyHostToDevice);
    /* 3-D extinction maps: device copies and the per-beam rows of nz minima */
    size_t ammin_per_beam = 1;
    if (ext && ext->kind == GF_EXT_MAPS) {
        const gf_ext_map *mp[2] = {ext->north, ext->south};
        int nz = 0;
        for (int h = 0; h < 2; h++) {
            if (!mp[h]) continue;
            const gf_ext_map &e = *mp[h];
            if (!e.A || e.n[0] < 1 || e.n[1] < 1 || e.n[2] < 1 || (nz && e.n[2] != nz))
                return bail(fail(GF_E_INVALID, "invalid extinction map (or north/south depths differ)"));
            nz = e.n[2];
            const size_t n = (size_t)e.n[0] * e.n[1] * e.n[2];
            if ((st = dev_alloc(&s->d_map[h], n)) != GF_OK) return bail(st);
            cudaMemcpy(s->d_map[h], e.A, 4 * n, cudaMemcpyHostToDevice);
            s->geom.map[h] = s->d_map[h];
            for (int a = 0; a < 3; a++) {
                s->geom.map_n[h][a] = e.n[a];
                s->geom.map_tc[h][a][0] = e.tc[a][0];
                s->geom.map_tc[h][a][1] = e.tc[a][1];
            }
            s->geom.ext_tcz[0] = e.tc[2][0];
            s->geom.ext_tcz[1] = e.tc[2][1];
        }
        if (nz == 0) {                 /* no map: zero extinction, one texel of minima */
            nz = 1;
            s->geom.ext_tcz[0] = 0.f;
            s->geom.ext_tcz[1] = 1.f;
        }
        s->geom.ext_nz = nz;
        s->maps = true;
        ammin_per_beam = (size_t)nz;
    }
    if (beam_ammin) {
        if ((st = dev_alloc(&s->d_ammin, ammin_per_beam * (size_t)npixels)) != GF_OK) return bail(st);
        cudaMemcpy(s->d_ammin, beam_ammin, 4 * ammin_per_beam * (size_t)npixels, cudaMemcpyHostToDevice);
    }
    s->geom.pixels = s->d_pixels;
    s->geom.npixels = npixels;
    s->geom.ammin = s->d_ammin;
    s->geom.ext_kind = ext ? ext->kind : GF_EXT_NONE;
    s->geom.A0 = ext ? ext->A0 : 0.f;
    s->geom.proj[0] = cfg->proj[0];
    s->geom.proj[1] = cfg->proj[1];
    s->models.resize(nmodels);
    for (int i = 0; i < nmodels; i++) {
        ModelState &ms = s->models[i];
        ms.hm = hms[i];
        if ((st = dev_alloc(&ms.d_lf, ms.hm.lf.size())) != GF_OK) return bail(st);
        cudaMemcpy(ms.d_lf, ms.hm.lf.data(), 4 * ms.hm.lf.size(), cudaMemcpyHostToDevice);
        if (ms.hm.cube) {
            if ((st = dev_alloc(&ms.d_cube, ms.hm.cube_size)) != GF_OK) return bail(st);
            cudaMemcpy(ms.d_cube, ms.hm.cube, 4 * ms.hm.cube_size, cudaMemcpyHostToDevice);
            ms.hm.m.cube = ms.d_cube;
        }
        if ((st = dev_alloc(&ms.d_Dtab, (size_t)ms.hm.m.nm * ms.hm.m.nM)) != GF_OK) return bail(st);
        if (gfk::launch_dtab(ms.hm.m, ms.d_Dtab, ctx->stream) != cudaSuccess) return bail(fail(GF_E_CUDA, "distance table"));
        if ((st = alloc_crawl_state(s->nthreads, ms.st, &ms.st_mem)) != GF_OK) return bail(st);
        if ((st = alloc_crawl_state(s->nthreads, ms.snap, &ms.snap_mem)) != GF_OK) return bail(st);
    }
    if ((st = dev_alloc(&s->d_limits, s->nthreads)) != GF_OK) return bail(st);
    if ((st = dev_alloc(&s->d_rng_snap, 3 * (size_t)s->nthreads)) != GF_OK) return bail(st);
    if (cudaMallocHost(&s->h_nstars, 8 * (size_t)s->nthreads) != cudaSuccess) return bail(fail(GF_E_OOM, "pinned allocation"));
    cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return bail(fail(GF_E_CUDA, cudaGetErrorString(ce)));
    *out = s;
    return GF_OK;
}

gf_status gf_skygen_destroy(gf_skygen *s)
{
    if (!s) return GF_OK;
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    for (auto &ms : s->models) {
        dev_free(ms.d_lf);
        dev_free(ms.d_cube);
        dev_free(ms.d_Dtab);
        if (ms.st_mem) cudaFree(ms.st_mem);
        if (ms.snap_mem) cudaFree(ms.snap_mem);
    }
    dev_free(s->d_pixels); dev_free(s->d_ammin); dev_free(s->d_limits); dev_free(s->d_rng_snap);
    if (s->h_nstars) cudaFreeHost(s->h_nstars);
    dev_free(s->d_map[0]); dev_free(s->d_map[1]);
    /* the record and placement buffers go to the context for its next generator
     * (the larger set is kept) */
    if (!s->ctx->rec_cache) s->ctx->rec_cache = new RecView();
    RecView &c = *(RecView *)s->ctx->rec_cache;
    RecView mine;
    move_recs(mine, *s);
    if (mine.rec_cap > c.rec_cap) std::swap(mine, c);
    free_recs(mine);
    dev_free(s->d_ck); dev_free(s->d_ck_count); dev_free(s->d_ck_sel); dev_free(s->d_keep);
    delete s;
    return GF_OK;
}

gf_status gf_skygen_model_info_get(gf_skygen *s, int32_t model, gf_skygen_model_info *info)
{
    if (!s || model < 0 || model >= (int)s->models.size() || !info) return fail(GF_E_INVALID, "invalid model");
    const SkyModel &m = s->models[model].hm.m;
    info->m0 = m.m0; info->m1 = m.m1; info->dm = m.dm; info->M0 = m.M0; info->M1 = m.M1; info->dM = m.dM;
    info->nm = m.nm; info->nM = m.nM; info->npixels = m.npixels; info->nthreads = m.nthreads;
    info->f = m.f; info->lf_x0 = m.lf_x0; info->lf_inv_dx = m.lf_inv_dx; info->lf_n = m.lf_n;
    info->norm = m.norm;
    return GF_OK;
}

gf_status gf_skygen_model_lf_get(gf_skygen *s, int32_t model, float *lf)
{
    if (!s || model < 0 || model >= (int)s->models.size() || !lf) return fail(GF_E_INVALID, "invalid model");
    const std::vector<float> &v = s->models[model].hm.lf;
    std::copy(v.begin(), v.end(), lf);
    return GF_OK;
}

gf_status gf_skygen_set_norm(gf_skygen *s, int32_t model, float norm)
{
    if (!s || model < 0 || model >= (int)s->models.size()) return fail(GF_E_INVALID, "invalid model");
    ModelState &ms = s->models[model];
    ms.hm.m.norm = norm;
    ms.expected *= norm;
    ms.expected_covered *= norm;
    return GF_OK;
}

gf_status gf_skygen_integrate(gf_skygen *s, int32_t model, double *expected, double *expected_covered, double *per_pixel)
{
    if (!s || model < 0 || model >= (int)s->models.size()) return fail(GF_E_INVALID, "invalid model");
    GF_TRY(check_ctx(s->ctx));
    ModelState &ms = s->models[model];
    cudaStream_t st = s->ctx->stream;
    const int N = s->nthreads;
    const int npix = s->geom.npixels;
    double *d_counts = nullptr, *d_cov = nullptr, *d_pp = nullptr;
    GF_TRY(dev_alloc(&d_counts, N));
    GF_TRY(dev_alloc(&d_cov, N));
    if (per_pixel) GF_TRY(dev_alloc(&d_pp, npix));
    GF_CUDA(cudaMemsetAsync(d_counts, 0, 8 * (size_t)N, st));
    GF_CUDA(cudaMemsetAsync(d_cov, 0, 8 * (size_t)N, st));
    if (d_pp) GF_CUDA(cudaMemsetAsync(d_pp, 0, 8 * (size_t)npix, st));
    gfk::LaunchCrawl L = crawl_launch(s, ms);
    L.counts = d_counts;
    L.countsCovered = d_cov;
    L.per_pixel = d_pp;
    const SkyModel &m = ms.hm.m;
    const long long kmax = (long long)m.nm * m.nM;
    if (kmax % GF_BLOCK == 0) {
        /* blocks never straddle pixels: one crawl over all pixels visits the same
         * bins with the same anchors as the reference's pixel-block launches */
        L.pix_base = 0;
        ProfScope ps(s->ctx, GF_PROF_INTEGRATE);
        GF_CUDA(gfk::launch_crawl(L, 0, st));
    } else {
        /* pixel blocks of 2^21 / nthreads pixels (skyconfig_impl.h:344-387) */
        const int PIXBLOCK = 1024 * 1024 * 2 / N;
        if (PIXBLOCK < 1) return fail(GF_E_UNSUPPORTED, "nthreads too large for pixel blocking");
        for (int p0 = 0; p0 < npix; p0 += PIXBLOCK) {
            int p1 = std::min(p0 + PIXBLOCK, npix);
            L.g.pixels = s->d_pixels + p0;
            L.g.npixels = p1 - p0;
            L.pix_base = p0;
            ProfScope ps(s->ctx, GF_PROF_INTEGRATE);
            GF_CUDA(gfk::launch_crawl(L, 0, st));
        }
    }
    std::vector<double> hc(N), hv(N);
    GF_CUDA(cudaMemcpyAsync(hc.data(), d_counts, 8 * (size_t)N, cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaMemcpyAsync(hv.data(), d_cov, 8 * (size_t)N, cudaMemcpyDeviceToHost, st));
    if (per_pixel) GF_CUDA(cudaMemcpyAsync(per_pixel, d_pp, 8 * (size_t)npix, cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    dev_free(d_counts); dev_free(d_cov); dev_free(d_pp);
    double e = 0, ec = 0;
    for (int i = 0; i < N; i++) { e += hc[i]; ec += hv[i]; }
    if (kmax % GF_BLOCK == 0) ms.stream_expected = hc;   /* the draw crawl assigns the same bins to the same streams */
    ms.expected = e;
    ms.expected_covered = ec;
    if (expected) *expected = e;
    if (expected_covered) *expected_covered = ec;
    return GF_OK;
}

gf_status gf_skygen_precision(gf_skygen *s, int32_t model, gf_precision_report *rep, double *per_pixel32,
                              double *per_pixel64, double *dm_hist64)
{
    if (!s || model < 0 || model >= (int)s->models.size() || !rep) return fail(GF_E_INVALID, "invalid arguments");
    GF_TRY(check_ctx(s->ctx));
    ModelState &ms = s->models[model];
    SkyModel m = ms.hm.m;
    m.lf = ms.d_lf;
    if (((long long)m.nm * m.nM) % GF_BLOCK) return fail(GF_E_UNSUPPORTED, "nm*nM must be a multiple of 10");
    cudaStream_t st = s->ctx->stream;
    const int npix = s->geom.npixels, nd = m.nm + m.nM - 1;
    double *d = nullptr;
    GF_TRY(dev_alloc(&d, 2 * (size_t)npix + nd + 4));
    double *pix32 = d, *pix64 = d + npix, *hist = d + 2 * (size_t)npix, *acc = hist + nd;
    GF_CUDA(cudaMemsetAsync(d, 0, 8 * (2 * (size_t)npix + nd + 4), st));
    cudaError_t e = gfk::launch_precision(m, s->geom, ms.d_Dtab, pix32, pix64, hist, (unsigned long long *)acc, acc + 1,
                                          (unsigned long long *)(acc + 2), st);
    if (e != cudaSuccess) { dev_free(d); return fail(GF_E_CUDA, cudaGetErrorString(e)); }
    std::vector<double> h(2 * (size_t)npix + nd + 4);
    GF_CUDA(cudaMemcpyAsync(h.data(), d, 8 * h.size(), cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    dev_free(d);
    double e32 = 0, e64 = 0, pmax = 0, psum = 0;
    int64_t pn = 0;
    for (int i = 0; i < npix; i++) {
        const double a = h[i], b = h[npix + i];
        e32 += a;
        e64 += b;
        if (b != 0.0) {
            const double r = fabs(a - b) / fabs(b);
            pmax = std::max(pmax, r);
            psum += r;
            pn++;
        }
    }
    const double *hacc = h.data() + 2 * (size_t)npix + nd;
    uint64_t mbits;
    memcpy(&mbits, hacc, 8);
    double bmax;
    memcpy(&bmax, &mbits, 8);
    uint64_t nb;
    memcpy(&nb, hacc + 2, 8);
    rep->expected32 = e32;
    rep->expected64 = e64;
    rep->total_rel_err = e64 != 0 ? fabs(e32 - e64) / fabs(e64) : 0.0;
    rep->bin_max_rel_err = bmax;
    rep->bin_mean_rel_err = nb ? hacc[1] / (double)nb : 0.0;
    rep->pixel_max_rel_err = pmax;
    rep->pixel_mean_rel_err = pn ? psum / (double)pn : 0.0;
    rep->bins = (int64_t)nb;
    if (per_pixel32) memcpy(per_pixel32, h.data(), 8 * (size_t)npix);
    if (per_pixel64) memcpy(per_pixel64, h.data() + npix, 8 * (size_t)npix);
    if (dm_hist64) memcpy(dm_hist64, h.data() + 2 * (size_t)npix, 8 * (size_t)nd);
    return GF_OK;
}

gf_status gf_skygen_draw(gf_skygen *s, int32_t model, gf_table *out, int64_t *n_generated, int32_t *done)
{
    if (!s || model < 0 || model >= (int)s->models.size() || !out || !n_generated || !done) return fail(GF_E_INVALID, "invalid arguments");
    GF_TRY(check_ctx(s->ctx));
    if (s->ctx->rng_nstreams < s->nthreads) return fail(GF_E_STATE, "gf_rng_init with at least nthreads streams must precede gf_skygen_draw");
    if (out->capacity <= 0) return fail(GF_E_INVALID, "output table has no capacity");
    ModelState &ms = s->models[model];
    cudaStream_t st = s->ctx->stream;
    const int N = s->nthreads;
    const int64_t C = out->capacity;
    if (ms.done) { out->size = 0; *n_generated = 0; *done = 1; return GF_OK; }
    const bool first_batch = !ms.crawl_init;
    if (first_batch) {
        GF_CUDA(cudaMemsetAsync(ms.st_mem, 0, crawl_state_bytes(N), st));
        ms.crawl_init = true;
        ms.stream_drawn.assign(N, 0);
    }
    GF_CUDA(cudaMemsetAsync(ms.st.nstars, 0, 8 * (size_t)N, st));
    GF_CUDA(cudaMemsetAsync(s->ctx->d_counters, 0, 24, st));
    GF_TRY(ensure_rec_capacity(s, C + C / 2 + 65536, 0));
    const int fb = (N + 255) / 256;
    /* checkpoints: one at each stream's first bin with stars and one every kCkEvery stars */
    const int kCkEvery = 64;
    {
        const int64_t want = (int64_t)N + (C + C / 2 + 65536) / kCkEvery + 4096;
        if (want > s->ck_cap) {
            dev_free(s->d_ck);
            GF_TRY(dev_alloc(&s->d_ck, (size_t)want));
            s->ck_cap = (int32_t)want;
        }
        if (!s->d_ck_count) {
            GF_TRY(dev_alloc(&s->d_ck_count, 4));
            GF_TRY(dev_alloc(&s->d_ck_sel, 1));
            GF_TRY(dev_alloc(&s->d_keep, 1));
        }
    }

    /* The batch is filled by streams in stream order (the CPU path runs the
     * emulated threads one after another).  Streams run speculatively in
     * windows predicted from their expected counts; the window that reaches
     * the capacity fixes the boundary stream t. */
    const bool have_pred = (int)ms.stream_expected.size() == N;
    int64_t cum = 0;          /* stars of streams before the current window position */
    int t = -1;
    int w_lo = ms.first_active, w_hi = w_lo;
    while (w_lo < N) {
        /* window end: enough expected stars to fill the remaining capacity with margin */
        int64_t room = C - cum;
        if (have_pred) {
            double need = (double)room + 6.0 * sqrt((double)room) + 256.0, acc = 0.0;
            w_hi = w_lo;
            while (w_hi < N && acc < need) {
                double rem = ms.stream_expected[w_hi] * (double)ms.hm.m.norm - (double)ms.stream_drawn[w_hi];
                acc += rem > 0 ? rem : 0.0;
                w_hi++;
            }
            w_hi = std::min(N, std::max(w_hi + 16, w_lo + 32));
        } else {
            w_hi = N;
        }
        unsigned long long rec_before = 0;
        GF_CUDA(cudaMemcpyAsync(&s->ctx->h_counters[0], s->ctx->d_counters, 8, cudaMemcpyDeviceToHost, st));
        GF_CUDA(cudaStreamSynchronize(st));
        rec_before = s->ctx->h_counters[0];
        GF_TRY(snapshot_range(s, ms, w_lo, w_hi, false));
        for (;;) {
            fill_range<<<fb, 256, 0, st>>>(s->d_limits, N, w_lo, w_hi, room);
            GF_CUDA(cudaMemsetAsync(s->d_ck_count, 0, 4, st));
            gfk::LaunchCrawl L = crawl_launch(s, ms);
            L.stream_begin = w_lo;
            L.stream_end = w_hi;
            L.ck = s->d_ck;
            L.ck_count = s->d_ck_count;
            L.ck_capacity = s->ck_cap;
            L.ck_every = kCkEvery;
            {
                ProfScope ps(s->ctx, GF_PROF_DRAW_WINDOW);
                GF_CUDA(gfk::launch_crawl(L, 1, st));
            }
            GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters, s->ctx->d_counters, 8, cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters + 4, s->d_ck_count, 4, cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaMemcpyAsync(s->h_nstars + w_lo, ms.st.nstars + w_lo, 8 * (size_t)(w_hi - w_lo), cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaStreamSynchronize(st));
            int64_t total = (int64_t)s->ctx->h_counters[0];
            if (total <= s->rec_cap) break;
            /* the window drew more stars than the record buffer holds: grow it and redo the window */
            GF_TRY(snapshot_range(s, ms, w_lo, w_hi, true));
            GF_TRY(ensure_rec_capacity(s, total + total / 4, (int64_t)rec_before));
            unsigned long long rb = rec_before;
            GF_CUDA(cudaMemcpyAsync(s->ctx->d_counters, &rb, 8, cudaMemcpyHostToDevice, st));
        }
        for (int i = w_lo; i < w_hi; i++) {
            if (cum + s->h_nstars[i] >= C) { t = i; break; }
            cum += s->h_nstars[i];
        }
        if (t >= 0) break;
        w_lo = w_hi;
    }
    int64_t nbatch;
    bool generated_all;
    if (t < 0) {
        GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters, s->ctx->d_counters, 8, cudaMemcpyDeviceToHost, st));
        GF_CUDA(cudaStreamSynchronize(st));
        nbatch = (int64_t)s->ctx->h_counters[0];
        generated_all = true;
        for (int i = ms.first_active; i < N; i++) ms.stream_drawn[i] += s->h_nstars[i];
        ms.first_active = N;
    } else {
        /* The batch ends inside stream t: it keeps the stars of the streams before
         * t and the first C - cum stars of t, and every later stream stops at its
         * first star (skygen.cu.h:366-373).  Stream t resumes from its latest
         * checkpoint at or below that count and re-draws only the stars after it;
         * in the first batch, the later streams of the window resume at their
         * first bin with stars and the streams after the window run up to theirs. */
        GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters, s->ctx->d_counters, 8, cudaMemcpyDeviceToHost, st));
        GF_CUDA(cudaStreamSynchronize(st));
        const int64_t total = (int64_t)s->ctx->h_counters[0];
        const bool ck_ok = (int64_t)(uint32_t)s->ctx->h_counters[4] <= (int64_t)s->ck_cap;
        const int64_t Lt = C - cum;
        const uint32_t NS = (uint32_t)s->ctx->rng_nstreams;
        GF_CUDA(cudaMemsetAsync(s->ctx->d_counters, 0, 8, st));
        int r_lo = t, r_hi;
        if (ck_ok) {
            GF_CUDA(cudaMemsetAsync(s->d_ck_sel, 0, 8, st));
            select_checkpoint<<<gfk::sm_count() * 4, 256, 0, st>>>(s->d_ck, s->d_ck_count, s->ck_cap, t, Lt, s->d_ck_sel);
            resume_boundary_stream<<<1, 32, 0, st>>>(s->d_ck, s->d_ck_sel, t, ms.st, ms.snap, s->ctx->d_rng, (int32_t)NS,
                                                      s->d_rng_snap, N, s->d_keep);
            if (first_batch) {
                resume_at_first_star<<<gfk::sm_count() * 4, 256, 0, st>>>(s->d_ck, s->d_ck_count, s->ck_cap, t, w_hi,
                                                                        ms.st, s->ctx->d_rng, (int32_t)NS);
                r_hi = N;
            } else {
                GF_TRY(snapshot_range(s, ms, t + 1, w_hi, true));
                r_hi = t + 1;
            }
            gfk::count_launches(first_batch ? 3 : 2);
        } else {
            GF_TRY(snapshot_range(s, ms, t, w_hi, true));
            GF_CUDA(cudaMemsetAsync(s->d_keep, 0, 8, st));
            r_hi = first_batch ? N : w_hi;
        }
        int blocks = (int)std::min<int64_t>((total + 255) / 256, (int64_t)gfk::sm_count() * 16);
        if (total > 0)
            filter_records<<<std::max(blocks, 1), 256, 0, st>>>(s->d_rec, s->d_rec_am, total, t, s->d_keep, s->d_rec2,
                                                                s->d_rec_am2, s->ctx->d_counters);
        std::swap(s->d_rec, s->d_rec2);
        std::swap(s->d_rec_am, s->d_rec_am2);
        set_limits<<<fb, 256, 0, st>>>(s->d_limits, N, t, Lt);
        gfk::LaunchCrawl L = crawl_launch(s, ms);
        L.stream_begin = r_lo;
        L.stream_end = r_hi;
        {
            ProfScope ps(s->ctx, GF_PROF_DRAW_RERUN);
            GF_CUDA(gfk::launch_crawl(L, 1, st));
        }
        GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters, s->ctx->d_counters, 8, cudaMemcpyDeviceToHost, st));
        GF_CUDA(cudaStreamSynchronize(st));
        nbatch = (int64_t)s->ctx->h_counters[0];
        if (nbatch != C) return fail(GF_E_CUDA, "batch rerun produced an unexpected star count");
        generated_all = false;
        for (int i = ms.first_active; i < t; i++) ms.stream_drawn[i] += s->h_nstars[i];
        ms.stream_drawn[t] += Lt;
        ms.first_active = t;
    }
    GF_CUDA(cudaMemcpy(s->ctx->h_counters + 2, s->ctx->d_counters + 2, 8, cudaMemcpyDeviceToHost));
    if (s->ctx->h_counters[2]) return fail(GF_E_INVALID, "a bin has an infinite expected star count");
    /* placement, sort by (hidden, l, b, DM, M, Am), truncation at the first hidden row */
    GF_CUDA(cudaMemsetAsync(s->ctx->d_counters + 1, 0, 8, st));
    gfk::LaunchPlace P;
    P.m = ms.hm.m;
    P.m.lf = ms.d_lf;
    P.g = s->geom;
    P.rec = s->d_rec;
    P.rec_am = s->d_rec_am;
    P.n = nbatch;
    P.lb = s->d_lb; P.projIdx = s->d_projIdx; P.projXY = s->d_projXY; P.DM = s->d_DM; P.absmag = s->d_absmag;
    P.XYZ = s->d_XYZ; P.Am = s->d_Am; P.AmInf = s->d_AmInf; P.hidden = s->d_hidden; P.key = s->d_key;
    P.nvis = s->ctx->d_counters + 1;
    {
        ProfScope ps(s->ctx, GF_PROF_PLACE);
        GF_CUDA(gfk::launch_place(P, st));
    }
    GF_CUDA(cudaMemcpyAsync(s->ctx->h_counters + 1, s->ctx->d_counters + 1, 8, cudaMemcpyDeviceToHost, st));
    GF_CUDA(cudaStreamSynchronize(st));
    int64_t nvis = (int64_t)s->ctx->h_counters[1];
    gfk::LaunchSort S;
    S.n = nbatch;
    S.nvisible = nvis;
    S.key_in = s->d_key; S.key_out = s->d_key2; S.idx_in = s->d_idx; S.idx_out = s->d_idx2;
    S.temp = s->d_sort_temp; S.temp_bytes = s->sort_temp_bytes;
    S.lb = s->d_lb; S.projIdx = s->d_projIdx; S.projXY = s->d_projXY; S.DM = s->d_DM; S.absmag = s->d_absmag;
    S.XYZ = s->d_XYZ; S.Am = s->d_Am; S.AmInf = s->d_AmInf; S.comp = ms.hm.m.comp;
    S.out = *out;
    {
        ProfScope ps(s->ctx, GF_PROF_SORT);
        GF_CUDA(gfk::launch_sort_gather(S, st));
    }
    GF_CUDA(cudaStreamSynchronize(st));
    out->size = nvis;
    ms.drawn += nbatch;
    *n_generated = nbatch;
    *done = generated_all ? 1 : 0;
    if (generated_all) ms.done = true;
    return GF_OK;
}

/* ---------------- tables ---------------- */

/* module columns start at zero so that rows a module skips are defined */
static gf_status zero_module_columns(gf_ctx *ctx, gf_table *t)
{
    return gfa::zero_module_rows(ctx, t, t->capacity);
}

/* the columns of a table of n rows (any that fail leave the others allocated) */
static gf_status table_alloc_columns(gf_table *t, size_t n, int32_t nbands)
{
    GF_TRY(dev_alloc(&t->lb, 2 * n));
    GF_TRY(dev_alloc(&t->projIdx, n));
    GF_TRY(dev_alloc(&t->projXY, 2 * n));
    GF_TRY(dev_alloc(&t->DM, n));
    GF_TRY(dev_alloc(&t->absmag, n));
    GF_TRY(dev_alloc(&t->XYZ, 3 * n));
    GF_TRY(dev_alloc(&t->comp, n));
    GF_TRY(dev_alloc(&t->Am, n));
    GF_TRY(dev_alloc(&t->AmInf, n));
    GF_TRY(dev_alloc(&t->hidden, n));
    GF_TRY(dev_alloc(&t->FeH, n));
    GF_TRY(dev_alloc(&t->vcyl, 3 * n));
    if (nbands) {
        GF_TRY(dev_alloc(&t->mags, (size_t)nbands * n));
        GF_TRY(dev_alloc(&t->obsmags, (size_t)nbands * n));
    }
    GF_TRY(dev_alloc(&t->photoflags, n));
    GF_TRY(dev_alloc(&t->pm, 3 * n));
    GF_TRY(dev_alloc(&t->radec, 2 * n));
    GF_TRY(dev_alloc(&t->FeH_comp, n));
    GF_TRY(dev_alloc(&t->absmagSys, 2 * n));
    GF_TRY(dev_alloc(&t->absmagSysNcomp, n));
    return GF_OK;
}

gf_status gf_table_alloc(gf_ctx *ctx, int64_t capacity, int32_t nbands, gf_table *t)
{
    GF_TRY(check_ctx(ctx));
    if (!t || capacity <= 0 || nbands < 0 || nbands > GF_MAX_BANDS) return fail(GF_E_INVALID, "invalid table arguments");
    memset(t, 0, sizeof(*t));
    t->capacity = capacity;
    t->nbands = nbands;
    gf_status st = table_alloc_columns(t, (size_t)capacity, nbands);
    if (st != GF_OK) {
        const std::string msg = gfa::g_err;
        gf_table_free(ctx, t);         /* no partial table is left behind */
        return fail(st, msg);
    }
    GF_TRY(zero_module_columns(ctx, t));
    GF_CUDA(cudaStreamSynchronize(ctx->stream));
    return GF_OK;
}

gf_status gf_table_free(gf_ctx *ctx, gf_table *t)
{
    if (!ctx || !t) return GF_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    dev_free(t->lb); dev_free(t->projIdx); dev_free(t->projXY); dev_free(t->DM); dev_free(t->absmag);
    dev_free(t->XYZ); dev_free(t->comp); dev_free(t->Am); dev_free(t->AmInf); dev_free(t->hidden);
    dev_free(t->FeH); dev_free(t->vcyl); dev_free(t->mags); dev_free(t->photoflags); dev_free(t->obsmags);
    dev_free(t->pm); dev_free(t->radec); dev_free(t->FeH_comp); dev_free(t->absmagSys); dev_free(t->absmagSysNcomp);
    memset(t, 0, sizeof(*t));
    return GF_OK;
}

gf_status gf_table_download_rows(gf_ctx *ctx, const gf_table *dev, int64_t begin, int64_t end, gf_table *host)
{
    GF_TRY(check_ctx(ctx));
    if (!dev || !host) return fail(GF_E_INVALID, "null table");
    if (begin < 0 || end < begin || end > dev->capacity) return fail(GF_E_INVALID, "invalid row range");
    if (host->capacity < end - begin) return fail(GF_E_INVALID, "host table too small");
    if (host->nbands < dev->nbands && (host->mags || host->obsmags)) return fail(GF_E_INVALID, "host table has fewer bands");
    const size_t n = (size_t)(end - begin), P = (size_t)dev->capacity, H = (size_t)host->capacity, b0 = (size_t)begin;
    cudaStream_t st = ctx->stream;
    auto cp = [&](void *h, const void *d, size_t elem, int ncomp) -> gf_status {
        if (!h || !d || n == 0) return GF_OK;
        for (int k = 0; k < ncomp; k++)
            GF_CUDA(cudaMemcpyAsync((char *)h + k * H * elem, (const char *)d + (k * P + b0) * elem, n * elem,
                                    cudaMemcpyDeviceToHost, st));
        return GF_OK;
    };
    GF_TRY(cp(host->lb, dev->lb, 8, 2));
    GF_TRY(cp(host->projIdx, dev->projIdx, 4, 1));
    GF_TRY(cp(host->projXY, dev->projXY, 4, 2));
    GF_TRY(cp(host->DM, dev->DM, 4, 1));
    GF_TRY(cp(host->absmag, dev->absmag, 4, 1));
    GF_TRY(cp(host->XYZ, dev->XYZ, 4, 3));
    GF_TRY(cp(host->comp, dev->comp, 4, 1));
    GF_TRY(cp(host->Am, dev->Am, 4, 1));
    GF_TRY(cp(host->AmInf, dev->AmInf, 4, 1));
    GF_TRY(cp(host->hidden, dev->hidden, 4, 1));
    GF_TRY(cp(host->FeH, dev->FeH, 4, 1));
    GF_TRY(cp(host->vcyl, dev->vcyl, 4, 3));
    GF_TRY(cp(host->mags, dev->mags, 4, dev->nbands));
    GF_TRY(cp(host->photoflags, dev->photoflags, 4, 1));
    GF_TRY(cp(host->obsmags, dev->obsmags, 4, dev->nbands));
    GF_TRY(cp(host->pm, dev->pm, 4, 3));
    GF_TRY(cp(host->radec, dev->radec, 8, 2));
    GF_TRY(cp(host->FeH_comp, dev->FeH_comp, 4, 1));
    GF_TRY(cp(host->absmagSys, dev->absmagSys, 4, 2));
    GF_TRY(cp(host->absmagSysNcomp, dev->absmagSysNcomp, 4, 1));
    GF_CUDA(cudaStreamSynchronize(st));
    host->size = end - begin;
    host->systems = dev->systems;
    return GF_OK;
}

gf_status gf_table_download(gf_ctx *ctx, const gf_table *dev, gf_table *host)
{
    if (!dev) return fail(GF_E_INVALID, "null table");
    return gf_table_download_rows(ctx, dev, 0, dev->size, host);
}

/* ---------------- modules ---------------- */

static gf_status row_range(const gf_table *t, int64_t begin, int64_t end)
{
    if (!t || begin < 0 || end < begin || end > t->capacity) return fail(GF_E_INVALID, "invalid row range");
    return GF_OK;
}

gf_status gf_module_clipper(gf_ctx *ctx, const gf_footprint *foot, const gf_lambert proj[2], gf_table *t, int64_t begin, int64_t end)
{
    (void)proj;
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!foot) return fail(GF_E_INVALID, "null footprint");
    ProfScope ps(ctx, GF_PROF_CLIPPER);
    GF_CUDA(gfk::launch_clipper(*foot, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_module_fixedfeh(gf_ctx *ctx, const gf_fixedfeh_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!cfg) return fail(GF_E_INVALID, "null config");
    ProfScope ps(ctx, GF_PROF_FEH);
    GF_CUDA(gfk::launch_fixedfeh(*cfg, *t, begin, end, ctx->stream));
    return GF_OK;
}

static gf_status module_feh(gf_ctx *ctx, const gf_feh_config *fp, const gf_gaussfeh_config *gp, gf_table *t,
                            int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!fp && !gp) return fail(GF_E_INVALID, "null config");
    if (gp && (gp->ncomp < 1 || gp->ncomp >= GF_GAUSSFEH_MAXCOMP || !(gp->pcum[gp->ncomp - 1] > 0.f)))
        return fail(GF_E_INVALID, "GaussianFeH needs 1 <= ncomp < 10 and positive cumulative weights");
    if (gp && !t->FeH_comp) return fail(GF_E_INVALID, "table without the FeH_comp column");
    if (!ctx->d_rng) return fail(GF_E_STATE, "gf_rng_init must precede the metallicity modules");
    const int64_t n = end - begin;
    if ((n + 255) / 256 > ctx->rng_nstreams) return fail(GF_E_INVALID, "more than 256 rows per stream");
    ProfScope ps(ctx, GF_PROF_FEH);
    GF_CUDA(gfk::launch_feh(fp, gp, ctx->d_rng, ctx->rng_nstreams, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_module_multiples(gf_ctx *ctx, const gf_multiples_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!cfg) return fail(GF_E_INVALID, "null config");
    if (cfg->algo < GF_MULT_LF_M2_GT_M1 || cfg->algo > GF_MULT_EQUAL_MASS || cfg->nsec < 1 || cfg->nsec > 64 ||
        cfg->ncum < 1 || cfg->ncum > GF_MULT_TEX || cfg->ninv < 1 || cfg->ninv > GF_MULT_TEX)
        return fail(GF_E_INVALID, "invalid unresolved-multiples configuration");
    if (!t->absmagSys || !t->absmagSysNcomp) return fail(GF_E_INVALID, "table without the absmagSys columns");
    if (!ctx->d_rng) return fail(GF_E_STATE, "gf_rng_init must precede gf_module_multiples");
    const int64_t n = end - begin;
    if ((n + 255) / 256 > ctx->rng_nstreams) return fail(GF_E_INVALID, "more than 256 rows per stream");
    ProfScope ps(ctx, GF_PROF_FEH);
    GF_CUDA(gfk::launch_multiples(*cfg, ctx->d_rng, ctx->rng_nstreams, *t, begin, end, ctx->stream));
    t->systems = 1;
    return GF_OK;
}

gf_status gf_module_feh(gf_ctx *ctx, const gf_feh_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    if (!cfg) return fail(GF_E_INVALID, "null config");
    return module_feh(ctx, cfg, nullptr, t, begin, end);
}

gf_status gf_module_gaussfeh(gf_ctx *ctx, const gf_gaussfeh_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    if (!cfg) return fail(GF_E_INVALID, "null config");
    return module_feh(ctx, nullptr, cfg, t, begin, end);
}

gf_status gf_module_bond2010(gf_ctx *ctx, const gf_bond2010_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!cfg) return fail(GF_E_INVALID, "null config");
    if (!ctx->d_rng) return fail(GF_E_STATE, "gf_rng_init must precede gf_module_bond2010");
    int64_t n = end - begin;
    if ((n + 255) / 256 > ctx->rng_nstreams) return fail(GF_E_INVALID, "more than 256 rows per stream");
    ProfScope ps(ctx, GF_PROF_BOND2010);
    GF_CUDA(gfk::launch_bond2010(*cfg, ctx->d_rng, ctx->rng_nstreams, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_photometry_create(gf_ctx *ctx, const gf_photometry_config *cfg, gf_photometry **out)
{
    GF_TRY(check_ctx(ctx));
    if (!cfg || !out || cfg->nbands < 2 || cfg->nbands > GF_MAX_BANDS || cfg->bidx < 0 || cfg->bidx >= cfg->nbands ||
        cfg->nFeH < 1 || cfg->nMr < 1 || !cfg->colors || !cfg->eflags)
        return fail(GF_E_INVALID, "invalid photometry configuration");
    gf_photometry *p = new gf_photometry();
    size_t n = (size_t)(cfg->nbands - 1) * cfg->nMr * cfg->nFeH;
    if (dev_alloc(&p->d_colors, n) != GF_OK || dev_alloc(&p->d_eflags, n) != GF_OK) {
        dev_free(p->d_colors); dev_free(p->d_eflags); delete p;
        return fail(GF_E_OOM, "photometry tables");
    }
    cudaMemcpy(p->d_colors, cfg->colors, 4 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(p->d_eflags, cfg->eflags, n, cudaMemcpyHostToDevice);
    gfk::PhotTables &T = p->tab;
    T.nbands = cfg->nbands; T.bidx = cfg->bidx; T.nFeH = cfg->nFeH; T.nMr = cfg->nMr;
    for (int i = 0; i < GF_MAX_BANDS; i++) T.reddening[i] = cfg->reddening[i];
    T.tcFeH[0] = cfg->tcFeH[0]; T.tcFeH[1] = cfg->tcFeH[1]; T.tcMr[0] = cfg->tcMr[0]; T.tcMr[1] = cfg->tcMr[1];
    T.colors = p->d_colors; T.eflags = p->d_eflags; T.comp_mask = cfg->comp_mask;
    *out = p;
    return GF_OK;
}

gf_status gf_photometry_destroy(gf_photometry *p)
{
    if (!p) return GF_OK;
    dev_free(p->d_colors); dev_free(p->d_eflags);
    delete p;
    return GF_OK;
}

gf_status gf_module_photometry(gf_ctx *ctx, const gf_photometry *p, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!p) return fail(GF_E_INVALID, "null photometry");
    if (t->nbands < p->tab.nbands) return fail(GF_E_INVALID, "table has fewer bands than the photometric system");
    ProfScope ps(ctx, GF_PROF_PHOTOMETRY);
    GF_CUDA(gfk::launch_photometry(p->tab, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_photoerr_create(gf_ctx *ctx, const gf_photoerr_config *cfg, gf_photoerr **out)
{
    GF_TRY(check_ctx(ctx));
    if (!cfg || !out || cfg->nbands < 1 || cfg->nbands > GF_MAX_BANDS || cfg->nknots < 2 || !cfg->mag || !cfg->sigma)
        return fail(GF_E_INVALID, "invalid photometric error configuration");
    gf_photoerr *p = new gf_photoerr();
    size_t n = (size_t)cfg->nbands * cfg->nknots;
    if (dev_alloc(&p->d_mag, n) != GF_OK || dev_alloc(&p->d_sigma, n) != GF_OK) {
        dev_free(p->d_mag); dev_free(p->d_sigma); delete p;
        return fail(GF_E_OOM, "photometric error tables");
    }
    cudaMemcpy(p->d_mag, cfg->mag, 8 * n, cudaMemcpyHostToDevice);
    cudaMemcpy(p->d_sigma, cfg->sigma, 8 * n, cudaMemcpyHostToDevice);
    p->tab.nbands = cfg->nbands; p->tab.nknots = cfg->nknots; p->tab.mag = p->d_mag; p->tab.sigma = p->d_sigma;
    p->tab.seed = cfg->seed;
    p->tab.guide = nullptr;
    p->tab.nguide = 0;
    /* bracket guide: one cell per knot over each band's knot range, when every band's
     * knots are finite and strictly increasing */
    const int nk = cfg->nknots;
    bool mono = true;
    for (int b = 0; b < cfg->nbands && mono; b++) {
        const double *xa = cfg->mag + (size_t)b * nk;
        for (int i = 0; i < nk && mono; i++) mono = std::isfinite(xa[i]) && (i == 0 || xa[i] > xa[i - 1]);
    }
    if (mono) {
        const int G = nk;
        std::vector<int32_t> guide((size_t)cfg->nbands * G);
        for (int b = 0; b < cfg->nbands; b++) {
            const double *xa = cfg->mag + (size_t)b * nk;
            const double x0 = xa[0], inv = (double)G / (xa[nk - 1] - xa[0]);
            p->tab.gx0[b] = x0;
            p->tab.ginv[b] = inv;
            int last = 0, i = 0;
            for (int g = 0; g < G; g++) {
                while (i <= nk - 2 && gfk::perr_cell(xa[i], x0, inv, G) < g) last = i++;
                guide[(size_t)b * G + g] = last;
            }
        }
        if (dev_alloc(&p->d_guide, guide.size()) != GF_OK) {
            dev_free(p->d_mag); dev_free(p->d_sigma); delete p;
            return fail(GF_E_OOM, "photometric error tables");
        }
        cudaMemcpy(p->d_guide, guide.data(), 4 * guide.size(), cudaMemcpyHostToDevice);
        p->tab.guide = p->d_guide;
        p->tab.nguide = G;
    }
    *out = p;
    return GF_OK;
}

gf_status gf_photoerr_destroy(gf_photoerr *p)
{
    if (!p) return GF_OK;
    dev_free(p->d_mag); dev_free(p->d_sigma); dev_free(p->d_guide);
    delete p;
    return GF_OK;
}

gf_status gf_module_photoerrors(gf_ctx *ctx, const gf_photoerr *p, int64_t row_offset, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!p) return fail(GF_E_INVALID, "null photometric errors");
    if (t->nbands < p->tab.nbands) return fail(GF_E_INVALID, "table has fewer bands than the error model");
    ProfScope ps(ctx, GF_PROF_PHOTOERR);
    GF_CUDA(gfk::launch_photoerrors(p->tab, row_offset, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_module_vel2pm(gf_ctx *ctx, const gf_vel2pm_config *cfg, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    if (!cfg) return fail(GF_E_INVALID, "null config");
    ProfScope ps(ctx, GF_PROF_VEL2PM);
    GF_CUDA(gfk::launch_vel2pm(*cfg, *t, begin, end, ctx->stream));
    return GF_OK;
}

gf_status gf_module_gal2other(gf_ctx *ctx, int32_t coordsys, gf_table *t, int64_t begin, int64_t end)
{
    GF_TRY(check_ctx(ctx));
    GF_TRY(row_range(t, begin, end));
    ProfScope ps(ctx, GF_PROF_GAL2OTHER);
    GF_CUDA(gfk::launch_gal2other(coordsys, *t, begin, end, ctx->stream));
    return GF_OK;
}

/* ---------------- the catalog path ---------------- */

static gf_status catalog_run_once(gf_ctx *ctx, const gf_job *job, gf_batch_callback cb, void *user, gf_catalog_stats *stats)
{
    GF_TRY(check_ctx(ctx));
    if (!job || job->nmodels <= 0 || job->nmodels > GF_MAX_MODELS || job->capacity <= 0) return fail(GF_E_INVALID, "invalid job");
    if (job->capacity > (int64_t)256 * GF_MAX_STREAMS) return fail(GF_E_INVALID, "capacity above 256 rows x 65536 streams");
    gf_catalog_stats local;
    gf_catalog_stats &S = stats ? *stats : local;
    memset(&S, 0, sizeof(S));
    S.norm = 1.f;
    if (job->nstreams > 0) GF_TRY(gf_rng_init(ctx, job->seed48, job->nstreams));
    if (!ctx->d_rng) return fail(GF_E_STATE, "no random streams: set nstreams or call gf_rng_init");
    /* models in component order (os_skygen.cpp:392-399) */
    std::vector<gf_model_config> models(job->models, job->models + job->nmodels);
    std::stable_sort(models.begin(), models.end(), [](const gf_model_config &a, const gf_model_config &b) { return a.comp < b.comp; });
    gf_skygen *sky = nullptr;
    GF_TRY(gf_skygen_create(ctx, &job->sky, job->pixels, job->npixels, job->beam_ammin, &job->ext, models.data(),
                            (int32_t)models.size(), &sky));
    struct Guard {
        gf_ctx *ctx; gf_skygen *sky; gf_table t; gf_photometry *ph; gf_photoerr *pe;
        ~Guard()
        {
            /* the output table stays with the context for the next request of the same shape */
            gf_table_free(ctx, &ctx->plain_table);
            ctx->plain_table = t;
            gf_photometry_destroy(ph); gf_photoerr_destroy(pe); gf_skygen_destroy(sky);
        }
    } g{ctx, sky, gf_table(), nullptr, nullptr};
    memset(&g.t, 0, sizeof(g.t));
    /* integrate every model first (os_skygen.cpp:875-880) */
    double total = 0;
    for (int i = 0; i < (int)models.size(); i++) {
        GF_TRY(gf_skygen_integrate(sky, i, &S.expected[i], &S.expected_covered[i], nullptr));
        total += S.expected_covered[i];
    }
    if (job->sky.nstars != 0.f) {
        /* forced normalisation (os_skygen.cpp:886-901) */
        double norm = job->sky.nstars / total;
        S.norm = (float)norm;
        for (int i = 0; i < (int)models.size(); i++) GF_TRY(gf_skygen_set_norm(sky, i, (float)norm));
    }
    if (ctx->plain_table.capacity == job->capacity && ctx->plain_table.nbands == job->nbands) {
        g.t = ctx->plain_table;
        memset(&ctx->plain_table, 0, sizeof(gf_table));
        g.t.size = 0;
        GF_TRY(zero_module_columns(ctx, &g.t));
    } else {
        GF_TRY(gf_table_alloc(ctx, job->capacity, job->nbands, &g.t));
    }
    if (job->phot) GF_TRY(gf_photometry_create(ctx, job->phot, &g.ph));
    if (job->perr) GF_TRY(gf_photoerr_create(ctx, job->perr, &g.pe));
    int64_t row_offset = 0;
    for (int i = 0; i < (int)models.size(); i++) {
        int32_t done = 0;
        while (!done) {
            int64_t ngen = 0;
            GF_TRY(gf_skygen_draw(sky, i, &g.t, &ngen, &done));
            S.generated[i] += ngen;
            const int64_t n = g.t.size;
            if (n == 0) continue;
            S.batches++;
            GF_TRY(gfa::zero_module_rows(ctx, &g.t, n));
            g.t.systems = 0;
            /* the module chain in pipeline order (pipeline.h:75-88) */
            if (job->foot) GF_TRY(gf_module_clipper(ctx, job->foot, job->sky.proj, &g.t, 0, n));
            if (job->feh) GF_TRY(gf_module_fixedfeh(ctx, job->feh, &g.t, 0, n));
            if (job->feh_ivezic) GF_TRY(gf_module_feh(ctx, job->feh_ivezic, &g.t, 0, n));
            if (job->feh_gauss) GF_TRY(gf_module_gaussfeh(ctx, job->feh_gauss, &g.t, 0, n));
            if (job->multiples) GF_TRY(gf_module_multiples(ctx, job->multiples, &g.t, 0, n));
            if (job->kin) GF_TRY(gf_module_bond2010(ctx, job->kin, &g.t, 0, n));
            if (g.ph) GF_TRY(gf_module_photometry(ctx, g.ph, &g.t, 0, n));
            if (g.pe) GF_TRY(gf_module_photoerrors(ctx, g.pe, row_offset, &g.t, 0, n));
            if (job->v2pm) GF_TRY(gf_module_vel2pm(ctx, job->v2pm, &g.t, 0, n));
            if (job->gal2other) GF_TRY(gf_module_gal2other(ctx, job->gal2other, &g.t, 0, n));
            GF_CUDA(cudaStreamSynchronize(ctx->stream));
            S.stored[i] += n;
            if (cb && cb(user, models[i].comp, &g.t, row_offset) != 0) return fail(GF_E_STATE, "stopped by the batch callback");
            row_offset += n;
        }
    }
    return GF_OK;
}

namespace {
struct CountingBatch {
    gf_batch_callback cb;
    void *user;
    long long calls;
};
int counting_batch(void *u, int32_t model, const gf_table *t, int64_t off)
{
    CountingBatch *c = (CountingBatch *)u;
    c->calls++;
    return c->cb ? c->cb(c->user, model, t, off) : 0;
}
}  // namespace

/* os_skygen::run + the module chain.  An out-of-memory failure before any batch
 * was delivered frees the context's cached buffers and runs the request once
 * more, as the reference collects garbage and retries a failed allocation
 * (cux.cpp:189-198); the streams are seeded again, so the retry is the same run. */
gf_status gf_catalog_run(gf_ctx *ctx, const gf_job *job, gf_batch_callback cb, void *user, gf_catalog_stats *stats)
{
    CountingBatch c = {cb, user, 0};
    gf_status st = catalog_run_once(ctx, job, counting_batch, &c, stats);
    if (st == GF_E_OOM && c.calls == 0 && job && job->nstreams > 0) {
        gfa::release_caches(ctx);
        st = catalog_run_once(ctx, job, counting_batch, &c, stats);
    }
    return st;
}

}  /* extern "C" */

namespace gfa {
gf_status catalog_run_in_multi(gf_ctx *ctx, const gf_job *job, gf_batch_callback cb, void *user, gf_catalog_stats *stats)
{
    CountingBatch c = {cb, user, 0};
    gf_status st = catalog_run_once(ctx, job, counting_batch, &c, stats);
    if (st == GF_E_OOM && c.calls == 0 && job && job->nstreams > 0) {
        cudaStreamSynchronize(ctx->stream);
        gf_table_free(ctx, &ctx->plain_table);
        free_rec_cache(ctx);
        st = catalog_run_once(ctx, job, counting_batch, &c, stats);
    }
    return st;
}
}  // namespace gfa

extern "C" {

gf_status gf_debug_fail_allocations(int64_t after, int64_t count)
{
    if (count < 0) return fail(GF_E_INVALID, "negative failure count");
    gfa::set_alloc_failures(after, count);
    return GF_OK;
}

}  /* extern "C" */
