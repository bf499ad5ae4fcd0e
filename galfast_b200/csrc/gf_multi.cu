/*
 * gf_multi.cu -- many catalog requests per pass: gf_catalog_run_multi.
 *
 * The plain path (gf_catalog_run) generates one request at a time.  A small
 * request -- a pencil beam of a few hundred pixels -- keeps only a fraction of
 * the GPU busy: its crawl has 7680 short streams, and every launch, sort and
 * module pass has fixed costs.  Here every pass runs over all requests at
 * once:
 *
 *   seeding     the 65536 streams of every request, on the GPU (seed_streams_kernel)
 *   integrate   one persistent crawl per model over the (request, stream) work queue
 *   draw        one persistent crawl per model over the same queue, requests in
 *               decreasing size so that the queue ends on small work
 *   place/sort  all records at once, sorted by (request, star_comp order)
 *   modules     one launch per module over the rows of all requests; Bond2010 and
 *               the photometric errors use each row's own request (its streams,
 *               its seed and catalog row numbers)
 *
 * Each request's catalog is the one gf_catalog_run produces for it alone, bit
 * for bit, as long as every model's stars fit one output batch (the batch
 * boundary rules of the plain path do not arise).  Requests whose expected
 * counts come near their batch capacity, or whose grid makes crawl blocks
 * straddle pixels (nm*nM not a multiple of 10), run through gf_catalog_run
 * after the batched passes.
 */
#include "gf_ctx.h"
#include "gf_host.h"
#include "gf_safeprimes.h"

#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstring>
#include <deque>
#include <thread>
#include <map>
#include <tuple>
#include <vector>

using gfa::dev_alloc;
using gfa::dev_free;
using gfa::fail;
using gfa::ProfScope;

namespace {

/* device allocations released together */
struct Pool {
    std::vector<void *> ptrs;
    template <typename T>
    gf_status alloc(T **p, size_t n)
    {
        GF_TRY(dev_alloc(p, n));
        if (*p) ptrs.push_back((void *)*p);
        return GF_OK;
    }
    ~Pool()
    {
        for (void *p : ptrs) cudaFree(p);
    }
};

/* fn(0) .. fn(n - 1) on up to 32 host threads (items taken in order from a shared counter) */
template <class F>
void parallel_for(int n, F fn)
{
    const int nt = std::max(1, std::min<int>({n / 16 + 1, (int)std::thread::hardware_concurrency(), 32}));
    if (nt <= 1) {
        for (int i = 0; i < n; i++) fn(i);
        return;
    }
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (int k = 0; k < nt; k++)
        th.emplace_back([&] {
            for (int i = next++; i < n; i = next++) fn(i);
        });
    for (auto &t : th) t.join();
}

/* a buffer that only grows */
template <typename T>
struct Grow {
    T *p = nullptr;
    size_t n = 0;
    gf_status need(size_t m)
    {
        if (m <= n) return GF_OK;
        dev_free(p);
        n = 0;
        GF_TRY(dev_alloc(&p, m));
        n = m;
        return GF_OK;
    }
    ~Grow() { dev_free(p); }
};

/* a page-locked host buffer that only grows */
template <typename T>
struct HostGrow {
    T *p = nullptr;
    size_t n = 0;
    gf_status need(size_t m)
    {
        if (m <= n) return GF_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        GF_CUDA(cudaMallocHost((void **)&p, m * sizeof(T)));
        n = m;
        return GF_OK;
    }
    ~HostGrow()
    {
        if (p) cudaFreeHost(p);
    }
};

/* module-group key of a request (the error seed is per request and not part of it) */
std::string module_signature(const gf_job &J)
{
    /* the configuration bytes, table pointers included: requests built from one
     * photometric system share its tables and land in one group */
    std::string sig;
    if (J.phot) {
        sig += "P";
        sig.append((const char *)J.phot, sizeof(gf_photometry_config));
    }
    if (J.perr) {
        gf_photoerr_config c = *J.perr;
        c.seed = 0;
        sig += "E";
        sig.append((const char *)&c, sizeof(c));
    }
    return sig;
}

bool same_cfg(const void *a, const void *b, size_t n)
{
    if (!a || !b) return a == b;
    return memcmp(a, b, n) == 0;
}

/* the kernel template a model type runs in: GF_MODEL_EXP_DISK or GF_MODEL_POWER_LAW_ELLIPSOID */
int model_kind(int type) { return type == GF_MODEL_EXP_DISK ? GF_MODEL_EXP_DISK : GF_MODEL_POWER_LAW_ELLIPSOID; }

struct ReqInfo {
    std::vector<gfh::HostModel> hm;    /* models in component order */
    std::vector<gf_model_config> mc;
    int64_t pix_off = 0;
    bool plain = false;
    /* batched, but one model's stars filled a whole output batch: its rows of that
     * pass on are withheld and the request runs alone at the end, delivering only
     * the components it had not delivered yet */
    bool overflow = false;
    std::vector<int32_t> delivered;    /* components delivered by batched passes */
    bool deferred = false;             /* left for a later call by the admission hook */
    int group = 0;
    int slot = -1;
    double cost = 0;
};

/* CrawlState slices of one request inside the arrays of all requests */
CrawlState slice(const CrawlState &a, size_t off)
{
    CrawlState s;
    s.status = a.status + off; s.blk_ilb = a.blk_ilb + off; s.blk_k = a.blk_k + off; s.pos = a.pos + off;
    s.ndraw = a.ndraw + off; s.cur_ilb = a.cur_ilb + off; s.cur_im = a.cur_im + off; s.cur_iM = a.cur_iM + off;
    s.anc = a.anc + off; s.nstars = a.nstars + off;
    return s;
}

}  // namespace

/* Device buffers of gf_catalog_run_multi, kept by the context between calls
 * (they only grow), so that repeated runs do not allocate. */
struct MultiWS {
    Grow<float> ammin;
    Grow<int64_t> catoff;
    Grow<int64_t> chunk_begin;
    Grow<uint32_t> counter;
    Grow<double> counts;
    Grow<char> cs;
    Grow<gf_footprint> foot;
    Grow<uint32_t> items;
    Grow<int32_t> job_slot;
    Grow<CrawlJob> jobs;
    Grow<float> lf;
    Grow<gf_pencil_beam> pix;
    Grow<uint64_t> pseed;
    Grow<uint32_t> rng;
    Grow<uint32_t> rng_snap;
    Grow<int64_t> row_begin;
    Grow<uint32_t> seeds;
    Grow<int64_t> seg;
    Grow<int32_t> slot_comp;
    Grow<int32_t> slot_job;
    Grow<int64_t> slot_rows;
    Grow<StarRecord> rec;
    Grow<int32_t> row_slot;
    Grow<uint64_t> key, key_b;
    Grow<uint32_t> idx_a, idx_b;
    Grow<char> temp;
    Grow<double2> pixsum, tot;              /* pixel-by-pixel integrate: per pixel, per request */
    Grow<const unsigned char *> plans;
    Grow<int32_t> pixoff;
    Grow<gfk::IntegPlanDesc> pdesc;
    Grow<float2> msbuf;                     /* batched draw: slot densities of the chunk's pixels */
    Grow<float2 *> msptr;
    Grow<int32_t> joblist, chunkoff;
    Grow<EventRecord> ev;
    Grow<int64_t> k64, off64;
    Grow<uint32_t> gitems;                  /* batched draw: (request << 16) | first of 32 streams */
    Grow<uint4> brec;                       /* batched draw: per request and block, the bound walk's record */
    Grow<uint4 *> brecptr;
    Grow<int64_t> blkoff;
    gf_table out;
    gf_table out2;                          /* host delivery: passes alternate between out and out2 */
    HostGrow<char> h_stage;              /* page-locked staging of uploads and downloads */
    /* host delivery: copy stream, per-table events, page-locked ring of host tables */
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_pass[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    bool free_recorded[2] = {false, false};
    HostGrow<char> ring;
    /* host delivery of plain-path batches: two device staging tables of the delivered
     * columns only, each free again once its copy-stream event has passed */
    Grow<char> stage;
    cudaEvent_t ev_stage[2] = {nullptr, nullptr}, ev_stage_free[2] = {nullptr, nullptr};
    bool stage_recorded[2] = {false, false};
    MultiWS()
    {
        memset(&out, 0, sizeof(out));
        memset(&out2, 0, sizeof(out2));
    }
    ~MultiWS()
    {
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        for (int b = 0; b < 2; b++) {
            if (ev_pass[b]) cudaEventDestroy(ev_pass[b]);
            if (ev_free[b]) cudaEventDestroy(ev_free[b]);
            if (ev_stage[b]) cudaEventDestroy(ev_stage[b]);
            if (ev_stage_free[b]) cudaEventDestroy(ev_stage_free[b]);
        }
        if (copy_stream) cudaStreamDestroy(copy_stream);
    }
};

namespace gfa {
void free_multi_ws(gf_ctx *ctx)
{
    if (!ctx->multi_ws) return;
    gf_table_free(ctx, &ctx->multi_ws->out);
    gf_table_free(ctx, &ctx->multi_ws->out2);
    delete ctx->multi_ws;
    ctx->multi_ws = nullptr;
}
}  // namespace gfa

namespace {
struct PlainForward {
    gf_multi_callback cb;
    void *user;
    int32_t njobs, job;
    std::vector<int64_t> begin, count;
    std::vector<int32_t> skip;         /* components already delivered by batched passes */
};

bool skipped(const std::vector<int32_t> &skip, int32_t comp)
{
    return std::find(skip.begin(), skip.end(), comp) != skip.end();
}

int forward_plain_batch(void *u, int32_t model, const gf_table *dev, int64_t row_offset)
{
    (void)row_offset;
    PlainForward *f = (PlainForward *)u;
    if (!f->cb || skipped(f->skip, model)) return 0;
    std::fill(f->begin.begin(), f->begin.end(), 0);
    std::fill(f->count.begin(), f->count.end(), 0);
    f->count[f->job] = dev->size;
    return f->cb(f->user, model, dev, f->begin.data(), f->count.data());
}

}  // namespace

namespace {

/* ---- host delivery: rows copied to a page-locked ring while the device works on ---- */
#define GF_RING 3

/* bytes of one row of a table with nb bands, counting the columns in mask (GF_COL_*) */
size_t row_bytes(int nb, uint32_t mask)
{
    const size_t w[20] = {16, 4, 8, 4, 4, 12, 4, 4, 4, 4, 4, 12, 4 * (size_t)nb, 4, 4 * (size_t)nb, 12, 16, 4, 8, 4};
    size_t b = 0;
    for (int i = 0; i < 20; i++)
        if (mask & (1u << i)) b += w[i];
    return b;
}

/* host table of `cap` rows and nb bands over page-locked memory at p (column by
 * column; the columns outside mask stay NULL and are not copied) */
gf_table carve_table(char *p, int64_t cap, int nb, uint32_t mask)
{
    gf_table t;
    memset(&t, 0, sizeof(t));
    t.capacity = cap;
    t.nbands = nb;
    const size_t n = (size_t)cap;
    auto take = [&](uint32_t col, size_t bytes) -> void * {
        if (!(mask & col) || bytes == 0) return nullptr;
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    t.lb = (double *)take(GF_COL_LB, 16 * n); t.projIdx = (int32_t *)take(GF_COL_PROJIDX, 4 * n);
    t.projXY = (float *)take(GF_COL_PROJXY, 8 * n); t.DM = (float *)take(GF_COL_DM, 4 * n);
    t.absmag = (float *)take(GF_COL_ABSMAG, 4 * n); t.XYZ = (float *)take(GF_COL_XYZ, 12 * n);
    t.comp = (int32_t *)take(GF_COL_COMP, 4 * n); t.Am = (float *)take(GF_COL_AM, 4 * n);
    t.AmInf = (float *)take(GF_COL_AMINF, 4 * n); t.hidden = (int32_t *)take(GF_COL_HIDDEN, 4 * n);
    t.FeH = (float *)take(GF_COL_FEH, 4 * n); t.vcyl = (float *)take(GF_COL_VCYL, 12 * n);
    t.mags = (float *)take(GF_COL_MAGS, 4 * n * nb); t.photoflags = (int32_t *)take(GF_COL_PHOTOFLAGS, 4 * n);
    t.obsmags = (float *)take(GF_COL_OBSMAGS, 4 * n * nb); t.pm = (float *)take(GF_COL_PM, 12 * n);
    t.radec = (double *)take(GF_COL_RADEC, 16 * n);
    t.FeH_comp = (int32_t *)take(GF_COL_FEHCOMP, 4 * n);
    t.absmagSys = (float *)take(GF_COL_ABSMAGSYS, 8 * n);
    t.absmagSysNcomp = (int32_t *)take(GF_COL_SYSNCOMP, 4 * n);
    return t;
}

size_t carved_bytes(int64_t cap, int nb, uint32_t mask) { return row_bytes(nb, mask) * (size_t)cap + 23 * 256; }

/* rows [r0, r1) of the device table d into the table h (host memory, or device
 * memory with kind = cudaMemcpyDeviceToDevice) at its row 0, on stream cs; the
 * columns that either table lacks are not copied */
gf_status copy_rows_async(const gf_table &d, int64_t r0, int64_t r1, gf_table &h, cudaStream_t cs,
                          cudaMemcpyKind kind = cudaMemcpyDeviceToHost)
{
    const size_t n = (size_t)(r1 - r0), P = (size_t)d.capacity, H = (size_t)h.capacity;
    auto cp = [&](void *hp, const void *dp, size_t elem, int ncomp) -> gf_status {
        if (!hp || !dp || n == 0 || ncomp <= 0) return GF_OK;
        GF_CUDA(cudaMemcpy2DAsync(hp, H * elem, (const char *)dp + (size_t)r0 * elem, P * elem, n * elem, (size_t)ncomp,
                                  kind, cs));
        return GF_OK;
    };
    GF_TRY(cp(h.lb, d.lb, 8, 2)); GF_TRY(cp(h.projIdx, d.projIdx, 4, 1)); GF_TRY(cp(h.projXY, d.projXY, 4, 2));
    GF_TRY(cp(h.DM, d.DM, 4, 1)); GF_TRY(cp(h.absmag, d.absmag, 4, 1)); GF_TRY(cp(h.XYZ, d.XYZ, 4, 3));
    GF_TRY(cp(h.comp, d.comp, 4, 1)); GF_TRY(cp(h.Am, d.Am, 4, 1)); GF_TRY(cp(h.AmInf, d.AmInf, 4, 1));
    GF_TRY(cp(h.hidden, d.hidden, 4, 1)); GF_TRY(cp(h.FeH, d.FeH, 4, 1)); GF_TRY(cp(h.vcyl, d.vcyl, 4, 3));
    GF_TRY(cp(h.mags, d.mags, 4, d.nbands)); GF_TRY(cp(h.photoflags, d.photoflags, 4, 1));
    GF_TRY(cp(h.obsmags, d.obsmags, 4, d.nbands)); GF_TRY(cp(h.pm, d.pm, 4, 3)); GF_TRY(cp(h.radec, d.radec, 8, 2));
    GF_TRY(cp(h.FeH_comp, d.FeH_comp, 4, 1));
    GF_TRY(cp(h.absmagSys, d.absmagSys, 4, 2)); GF_TRY(cp(h.absmagSysNcomp, d.absmagSysNcomp, 4, 1));
    h.systems = d.systems;
    return GF_OK;
}

/* one delivered piece: run by the copy stream after its rows have arrived */
struct Piece {
    gf_multi_host_callback cb;
    void *user;
    int32_t model;
    gf_table host;
    std::vector<int64_t> begin, count;
    std::atomic<int> *stop;
};

void CUDART_CB deliver_piece(void *arg)
{
    Piece *p = (Piece *)arg;
    if (p->stop->load() || !p->cb) return;
    if (p->cb(p->user, p->model, &p->host, p->begin.data(), p->count.data()) != 0) p->stop->store(1);
}

struct HostDelivery {
    gf_multi_host_callback cb = nullptr;
    void *user = nullptr;
    int64_t piece_rows = 0;
    int nbands = 0;
    int64_t next = 0;                    /* pieces enqueued */
    std::deque<Piece> pieces;
    std::atomic<int> stop{0};
    gf_table ring[GF_RING];
};

/* Enqueue the delivery of rows [0, total) of the device table d, whose slot s holds
 * request slot_job[s] at rows [row_begin[s], row_begin[s] + rows[s]). */
gf_status deliver_rows(MultiWS &ws, HostDelivery &hd, cudaEvent_t ev_ready, cudaEvent_t ev_done, cudaStream_t st,
                       const gf_table &d, int32_t model, const std::vector<int> &slot_job,
                       const std::vector<int64_t> &row_begin, const std::vector<int64_t> &rows, int njobs)
{
    cudaStream_t cs = ws.copy_stream;
    GF_CUDA(cudaEventRecord(ev_ready, st));
    GF_CUDA(cudaStreamWaitEvent(cs, ev_ready, 0));
    const int64_t total = row_begin[slot_job.size()];
    for (int64_t r0 = 0; r0 < total; r0 += hd.piece_rows) {
        const int64_t r1 = std::min(total, r0 + hd.piece_rows);
        gf_table &h = hd.ring[hd.next % GF_RING];
        hd.next++;
        GF_TRY(copy_rows_async(d, r0, r1, h, cs));
        hd.pieces.emplace_back();
        Piece &p = hd.pieces.back();
        p.cb = hd.cb; p.user = hd.user; p.model = model; p.stop = &hd.stop;
        p.host = h;
        p.host.size = r1 - r0;
        p.host.nbands = d.nbands;
        p.begin.assign(njobs, 0);
        p.count.assign(njobs, 0);
        for (size_t q = 0; q < slot_job.size(); q++) {
            const int64_t a = std::max(r0, row_begin[q]), e = std::min(r1, row_begin[q] + rows[q]);
            if (e > a) { p.begin[slot_job[q]] = a - r0; p.count[slot_job[q]] = e - a; }
        }
        GF_CUDA(cudaLaunchHostFunc(cs, deliver_piece, &p));
    }
    GF_CUDA(cudaEventRecord(ev_done, cs));
    return GF_OK;
}

gf_status deliver_pass(MultiWS &ws, HostDelivery &hd, int b, cudaStream_t st, const gf_table &d, int32_t model,
                       const std::vector<int> &slot_job, const std::vector<int64_t> &row_begin,
                       const std::vector<int64_t> &rows, int njobs)
{
    GF_TRY(deliver_rows(ws, hd, ws.ev_pass[b], ws.ev_free[b], st, d, model, slot_job, row_begin, rows, njobs));
    ws.free_recorded[b] = true;
    return GF_OK;
}

struct PlainHostForward {
    HostDelivery *hd;
    MultiWS *ws;
    int *pass;                         /* model passes delivered so far (selects the staging table) */
    gf_ctx *ctx;
    int32_t njobs, job;
    int64_t capacity;                  /* the request's batch capacity */
    std::vector<int32_t> skip;         /* components already delivered by batched passes */
    gf_status err = GF_OK;             /* a failure inside the callback, and its message */
    std::string msg;
};

/* A plain-path batch of a request run inside the multi call.  Its delivered
 * columns are staged on the device, in two alternating staging tables of their
 * own, and leave through the copy stream behind the batched passes' rows, so the
 * plain path generates its next batch while the copies drain; it waits only for
 * the copy of the batch before last. */
int forward_plain_host(void *u, int32_t model, const gf_table *dev, int64_t row_offset)
{
    (void)row_offset;
    PlainHostForward *f = (PlainHostForward *)u;
    HostDelivery &hd = *f->hd;
    MultiWS &ws = *f->ws;
    auto failed = [&](gf_status e, const char *what) {
        f->err = e;
        f->msg = std::string(what) + ": " + gf_last_error();
        return 1;
    };
    if (hd.stop.load()) return 1;
    if (skipped(f->skip, model) || dev->size <= 0) return 0;
    cudaStream_t st = f->ctx->stream;
    const int b = *f->pass & 1;
    /* staging table b: the delivered columns of up to `capacity` rows */
    const int64_t cap = std::max(dev->size, f->capacity);
    const size_t bytes = (carved_bytes(cap, dev->nbands, f->ctx->host_cols) + 255) & ~(size_t)255;
    cudaError_t ce = cudaSuccess;
    if (ws.stage.n < 2 * bytes) {
        ce = cudaStreamSynchronize(ws.copy_stream);            /* nothing reads the old staging tables */
        if (ce == cudaSuccess) {
            const gf_status as = ws.stage.need(2 * bytes);
            if (as != GF_OK) return failed(as, "staging tables");
            ws.stage_recorded[0] = ws.stage_recorded[1] = false;
        }
    }
    /* its previous rows have been copied out */
    if (ce == cudaSuccess && ws.stage_recorded[b]) ce = cudaStreamWaitEvent(st, ws.ev_stage_free[b], 0);
    if (ce != cudaSuccess) return failed(GF_E_CUDA, cudaGetErrorString(ce));
    /* each half of the staging buffer holds at least `bytes`, the carving of cap rows */
    const size_t half = (ws.stage.n / 2) & ~(size_t)255;
    gf_table V = carve_table(ws.stage.p + (size_t)b * half, cap, dev->nbands, f->ctx->host_cols);
    gf_status cs = copy_rows_async(*dev, 0, dev->size, V, st, cudaMemcpyDeviceToDevice);
    if (cs != GF_OK) return failed(cs, "staging copy");
    V.size = dev->size;
    V.systems = dev->systems;
    const std::vector<int> slot_job(1, f->job);
    const std::vector<int64_t> row_begin = {0, dev->size}, rows(1, dev->size);
    cs = deliver_rows(ws, hd, ws.ev_stage[b], ws.ev_stage_free[b], st, V, model, slot_job, row_begin, rows, f->njobs);
    if (cs != GF_OK) return failed(cs, "host delivery");
    ws.stage_recorded[b] = true;
    (*f->pass)++;
    return 0;
}

gf_status run_multi(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, gf_multi_host_callback hcb,
                    int64_t piece_rows, void *user, gf_catalog_stats *stats, gfa::Admission *adm)
{
    GF_TRY(gfa::check_ctx(ctx));
    gfa::HostScope setup_time(ctx, GF_PROF_SETUP);
    if (!jobs || njobs <= 0 || njobs > 32767) return fail(GF_E_INVALID, "njobs must be in [1, 32767]");
    const gf_job &J0 = jobs[0];
    const int N = J0.sky.nthreads;
    const int nmod = J0.nmodels;
    if (N <= 0 || N > GF_MAX_STREAMS) return fail(GF_E_INVALID, "nthreads must be in [1, 65536]");
    if (nmod <= 0 || nmod > GF_MAX_MODELS) return fail(GF_E_INVALID, "invalid model count");
    int NS = 0, nbands = 0;
    for (int j = 0; j < njobs; j++) {
        const gf_job &J = jobs[j];
        if (J.sky.nthreads != N || J.nmodels != nmod)
            return fail(GF_E_INVALID, "all requests of a multi-request run need the same nthreads and model count");
        if (!J.pixels || J.npixels <= 0 || !J.models) return fail(GF_E_INVALID, "request without pixels or models");
        if (J.sky.nstars != 0.f) return fail(GF_E_UNSUPPORTED, "forced star counts (nstars) need gf_catalog_run");
        if (J.nstreams <= 0) return fail(GF_E_INVALID, "every request of a multi-request run seeds its own streams (nstreams > 0)");
        if (J.capacity <= 0 || J.capacity > (int64_t)256 * GF_MAX_STREAMS) return fail(GF_E_INVALID, "invalid capacity");
        int ns = J.nstreams > GF_MAX_STREAMS ? GF_MAX_STREAMS : J.nstreams;
        if (ns % 64) ns += 64 - ns % 64;
        if (ns < N) return fail(GF_E_INVALID, "nstreams below nthreads");
        if ((J.kin || J.feh_ivezic || J.feh_gauss || J.multiples) && (J.capacity + 255) / 256 > ns)
            return fail(GF_E_INVALID, "capacity above 256 rows per stream (the stream-drawing modules)");
        NS = std::max(NS, ns);
        nbands = std::max(nbands, (int)J.nbands);
        if (!!J.feh != !!J0.feh || !!J.kin != !!J0.kin || !!J.v2pm != !!J0.v2pm || J.gal2other != J0.gal2other ||
            !!J.phot != !!J0.phot || !!J.perr != !!J0.perr || !!J.feh_ivezic != !!J0.feh_ivezic ||
            !!J.feh_gauss != !!J0.feh_gauss || !!J.multiples != !!J0.multiples)
            return fail(GF_E_INVALID, "all requests of a multi-request run need the same modules");
        if (!same_cfg(J.feh, J0.feh, sizeof(gf_fixedfeh_config)) || !same_cfg(J.kin, J0.kin, sizeof(gf_bond2010_config)) ||
            !same_cfg(J.v2pm, J0.v2pm, sizeof(gf_vel2pm_config)) ||
            !same_cfg(J.feh_ivezic, J0.feh_ivezic, sizeof(gf_feh_config)) ||
            !same_cfg(J.feh_gauss, J0.feh_gauss, sizeof(gf_gaussfeh_config)) ||
            !same_cfg(J.multiples, J0.multiples, sizeof(gf_multiples_config)))
            return fail(GF_E_INVALID, "the metallicity, multiples, Bond2010 and vel2pm configurations must agree across requests");
        if (J.feh_gauss && (J.feh_gauss->ncomp < 1 || J.feh_gauss->ncomp >= GF_GAUSSFEH_MAXCOMP))
            return fail(GF_E_INVALID, "GaussianFeH needs 1 <= ncomp < 10");
    }
    GF_TRY(gfa::ensure_multipliers(ctx));
    cudaStream_t st = ctx->stream;

    std::vector<gf_catalog_stats> local(njobs);
    gf_catalog_stats *S = stats ? stats : local.data();
    for (int j = 0; j < njobs; j++) {
        memset(&S[j], 0, sizeof(gf_catalog_stats));
        S[j].norm = 1.f;
    }

    /* ---- host set-up of every request (models and module signatures on host threads) ---- */
    std::vector<ReqInfo> R(njobs);
    int64_t pix_total = 0;
    std::map<std::string, int> groups;          /* module-table signature -> group */
    std::vector<int> group_rep;                 /* a request of each group */
    std::vector<std::string> errs(njobs), sigs(njobs);
    parallel_for(njobs, [&](int j) {
        const gf_job &J = jobs[j];
        ReqInfo &q = R[j];
        q.mc.assign(J.models, J.models + nmod);
        std::stable_sort(q.mc.begin(), q.mc.end(), [](const gf_model_config &a, const gf_model_config &b) { return a.comp < b.comp; });
        if (!gfh::setup_models(J.sky, J.npixels, q.mc.data(), nmod, q.hm, errs[j]) && errs[j].empty()) errs[j] = "invalid model";
        sigs[j] = module_signature(J);
    });
    for (int j = 0; j < njobs; j++) {
        const gf_job &J = jobs[j];
        ReqInfo &q = R[j];
        if (!errs[j].empty()) return fail(GF_E_INVALID, errs[j]);
        for (int i = 0; i < nmod; i++) {
            if (model_kind(q.hm[i].m.type) != model_kind(R[0].hm[i].m.type))
                return fail(GF_E_INVALID, "model kinds must agree across requests (in component order)");
            const long long kmax = (long long)q.hm[i].m.nm * q.hm[i].m.nM;
            if (kmax % GF_BLOCK) q.plain = true;
            if (q.hm[i].m.type == GF_MODEL_DENSITY_CUBE) q.plain = true;    /* its grid is uploaded by the plain path */
            if (q.hm[i].m.nm + q.hm[i].m.nM > 16384) q.plain = true;
        }
        /* 3-D extinction maps: the anchors' extinction depends on their distance,
         * which the slot tables do not carry; such a request takes the plain path */
        if (J.ext.kind == GF_EXT_MAPS) q.plain = true;
        q.pix_off = pix_total;
        pix_total += J.npixels;
        q.cost = (double)J.npixels * q.hm[0].m.nm;
        const std::string &key = sigs[j];
        auto it = groups.find(key);
        if (it == groups.end()) {
            it = groups.insert({key, (int)groups.size()}).first;
            group_rep.push_back(j);
        }
        q.group = it->second;
    }

    Pool pool;
    if (!ctx->multi_ws) ctx->multi_ws = new MultiWS();
    MultiWS &ws = *ctx->multi_ws;
    gf_pencil_beam *d_pix = nullptr;
    float *d_ammin = nullptr, *d_lf = nullptr;
    GF_TRY(ws.pix.need((size_t)pix_total));
    d_pix = ws.pix.p;
    GF_TRY(ws.ammin.need((size_t)pix_total));
    d_ammin = ws.ammin.p;
    GF_TRY(ws.lf.need((size_t)njobs * nmod * 1024));
    d_lf = ws.lf.p;
    {
        /* one page-locked staging area: all pixels, then the per-beam extinction, then the LFs */
        const size_t pb = sizeof(gf_pencil_beam) * (size_t)pix_total, ab = 4 * (size_t)pix_total;
        const size_t lb_ = 4 * (size_t)njobs * nmod * 1024;
        GF_TRY(ws.h_stage.need(pb + ab + lb_));
        char *h = ws.h_stage.p;
        gf_pencil_beam *hp = (gf_pencil_beam *)h;
        float *ha = (float *)(h + pb), *hl = (float *)(h + pb + ab);
        memset(hl, 0, lb_);
        parallel_for(njobs, [&](int j) {
            memcpy(hp + R[j].pix_off, jobs[j].pixels, sizeof(gf_pencil_beam) * (size_t)jobs[j].npixels);
            if (jobs[j].beam_ammin) memcpy(ha + R[j].pix_off, jobs[j].beam_ammin, 4 * (size_t)jobs[j].npixels);
            else memset(ha + R[j].pix_off, 0, 4 * (size_t)jobs[j].npixels);
            for (int i = 0; i < nmod; i++)
                std::copy(R[j].hm[i].lf.begin(), R[j].hm[i].lf.end(), hl + ((size_t)j * nmod + i) * 1024);
        });
        GF_CUDA(cudaMemcpyAsync(d_pix, hp, pb, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaMemcpyAsync(d_ammin, ha, ab, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaMemcpyAsync(d_lf, hl, lb_, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaStreamSynchronize(st));
    }
    /* distance tables D[im][iM], shared by the requests with the same magnitude grid */
    std::map<std::tuple<float, float, float, float, int>, std::pair<int, float *>> dtabs;
    for (int j = 0; j < njobs; j++)
        for (int i = 0; i < nmod; i++) {
            const SkyModel &m = R[j].hm[i].m;
            auto k = std::make_tuple(m.m0, m.dm, m.M1, m.dM, m.nM);
            auto &e = dtabs[k];
            e.first = std::max(e.first, m.nm);
        }
    for (auto &kv : dtabs) {
        SkyModel m;
        memset(&m, 0, sizeof(m));
        m.m0 = std::get<0>(kv.first); m.dm = std::get<1>(kv.first); m.M1 = std::get<2>(kv.first); m.dM = std::get<3>(kv.first);
        m.nM = std::get<4>(kv.first);
        m.nm = kv.second.first;
        GF_TRY(pool.alloc(&kv.second.second, (size_t)m.nm * m.nM));
        GF_CUDA(gfk::launch_dtab(m, kv.second.second, st));
    }
    auto dtab_of = [&](const SkyModel &m) { return dtabs[std::make_tuple(m.m0, m.dm, m.M1, m.dM, m.nM)].second; };

    /* ---- streams of every request ---- */
    uint32_t *d_rng = nullptr, *d_rng_snap = nullptr, *d_seeds = nullptr;
    GF_TRY(ws.rng.need((size_t)njobs * 3 * NS));
    d_rng = ws.rng.p;
    GF_TRY(ws.rng_snap.need((size_t)njobs * 3 * NS));
    d_rng_snap = ws.rng_snap.p;
    GF_TRY(ws.seeds.need((size_t)njobs));
    d_seeds = ws.seeds.p;
    {
        std::vector<uint32_t> seeds(njobs);
        for (int j = 0; j < njobs; j++) seeds[j] = jobs[j].seed48;
        GF_CUDA(cudaMemcpyAsync(d_seeds, seeds.data(), 4 * (size_t)njobs, cudaMemcpyHostToDevice, st));
        GF_CUDA(gfk::launch_seed_streams(d_seeds, njobs, ctx->d_mult, NS, d_rng, st));
    }

    /* ---- per-(request, stream) state ---- */
    const size_t nall = (size_t)njobs * N;
    CrawlState cs;
    {
        char *base = nullptr;
        const size_t bytes = nall * (8 * 4 + 16 + 8) + 256;
        GF_TRY(ws.cs.need(bytes));
    base = ws.cs.p;
        char *p = base;
        auto take = [&](size_t b) { char *r = p; p += (b + 15) & ~(size_t)15; return r; };
        cs.anc = (AnchorX *)take(16 * nall);
        cs.nstars = (int64_t *)take(8 * nall);
        cs.status = (int32_t *)take(4 * nall); cs.blk_ilb = (int32_t *)take(4 * nall); cs.blk_k = (int32_t *)take(4 * nall);
        cs.pos = (int32_t *)take(4 * nall); cs.ndraw = (int32_t *)take(4 * nall); cs.cur_ilb = (int32_t *)take(4 * nall);
        cs.cur_im = (int32_t *)take(4 * nall); cs.cur_iM = (int32_t *)take(4 * nall);
    }
    const size_t cs_bytes = nall * (8 * 4 + 16 + 8) + 256;
    char *cs_base = (char *)cs.anc;
    double *d_counts = nullptr;
    CrawlJob *d_jobs = nullptr;
    uint32_t *d_items = nullptr, *d_counter = nullptr;
    GF_TRY(ws.counts.need(2 * nall));
    d_counts = ws.counts.p;
    GF_TRY(ws.jobs.need((size_t)njobs));
    d_jobs = ws.jobs.p;
    GF_TRY(ws.items.need(nall));
    d_items = ws.items.p;
    GF_TRY(ws.counter.need(1));
    d_counter = ws.counter.p;

    auto crawl_job = [&](int j, int i) {
        CrawlJob c;
        memset(&c, 0, sizeof(c));
        c.m = R[j].hm[i].m;
        c.m.lf = d_lf + ((size_t)j * nmod + i) * 1024;
        c.g.pixels = d_pix + R[j].pix_off;
        c.g.npixels = jobs[j].npixels;
        c.g.ammin = jobs[j].beam_ammin ? d_ammin + R[j].pix_off : nullptr;
        c.g.ext_kind = jobs[j].ext.kind;
        c.g.A0 = jobs[j].ext.A0;
        c.g.proj[0] = jobs[j].sky.proj[0];
        c.g.proj[1] = jobs[j].sky.proj[1];
        c.st = slice(cs, (size_t)j * N);
        c.rng = d_rng + (size_t)j * 3 * NS;
        c.rng_nstreams = NS;
        c.counts = d_counts + (size_t)j * N;
        c.countsCovered = d_counts + nall + (size_t)j * N;
        c.Dtab = dtab_of(c.m);
        c.fx = make_fastdiv((uint32_t)c.m.nm);
        c.fy = make_fastdiv((uint32_t)c.m.nM);
        c.job_id = j;
        c.limit_all = jobs[j].capacity;
        return c;
    };
    /* work items: requests in decreasing size, all streams of each */
    auto upload_items = [&](const std::vector<int> &order, int32_t *nitems) -> gf_status {
        const size_t cnt = order.size() * (size_t)N;
        GF_TRY(ws.h_stage.need(4 * cnt));
        uint32_t *items = (uint32_t *)ws.h_stage.p;
        size_t k = 0;
        for (int j : order)
            for (int t = 0; t < N; t++) items[k++] = ((uint32_t)j << 16) | (uint32_t)t;
        GF_CUDA(cudaMemcpyAsync(d_items, items, 4 * cnt, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaStreamSynchronize(st));
        *nitems = (int32_t)cnt;
        return GF_OK;
    };
    std::vector<int> order_all(njobs);
    for (int j = 0; j < njobs; j++) order_all[j] = j;
    std::stable_sort(order_all.begin(), order_all.end(), [&](int a, int b) { return R[a].cost > R[b].cost; });
    auto max_tab = [&](int i, const std::vector<int> &js) {
        int mt = 0;
        for (int j : js) mt = std::max(mt, R[j].hm[i].m.nm + R[j].hm[i].m.nM);
        return mt;
    };

    /* ---- integrate every model of every request (os_skygen.cpp:875-880) ---- */
    std::vector<CrawlJob> hj(njobs);
    std::vector<int> integ;
    for (int j : order_all)
        if (!R[j].plain) integ.push_back(j);
    int32_t nitems = 0;
    bool items_integ = false;          /* per-stream items of the crawl integrate, uploaded when needed */
    /* pixel-by-pixel integrate: anchor plans per magnitude grid (nm * nM is a
     * multiple of 10 for every batched request) */
    std::map<std::tuple<float, float, float, float, int, int>, unsigned char *> plans;
    std::map<const unsigned char *, int> plan_nslots;
    std::vector<char> plan_used(nmod, 0);
    auto plan_of = [&](int j, int i) -> unsigned char * {
        const SkyModel &m = R[j].hm[i].m;
        auto it = plans.find(std::make_tuple(m.m0, m.dm, m.M1, m.dM, m.nM, m.nm));
        return it == plans.end() ? nullptr : it->second;
    };
    std::vector<double2> htot(njobs);
    const bool pixel_integrate = pix_total < (int64_t)INT32_MAX;
    if (pixel_integrate && !integ.empty()) {
        std::vector<int32_t> off(njobs + 1);
        for (int j = 0; j < njobs; j++) off[j] = (int32_t)R[j].pix_off;
        off[njobs] = (int32_t)pix_total;
        GF_TRY(ws.pixoff.need((size_t)njobs + 1));
        GF_CUDA(cudaMemcpyAsync(ws.pixoff.p, off.data(), 4 * ((size_t)njobs + 1), cudaMemcpyHostToDevice, st));
        GF_TRY(ws.pixsum.need((size_t)std::max<int64_t>(pix_total, 1)));
        GF_TRY(ws.tot.need((size_t)njobs));
        GF_TRY(ws.plans.need((size_t)njobs));
    }
    setup_time.stop();
    for (int i = 0; i < nmod && !integ.empty(); i++) {
        for (int j = 0; j < njobs; j++) hj[j] = crawl_job(j, i);
        GF_CUDA(cudaMemcpyAsync(d_jobs, hj.data(), sizeof(CrawlJob) * (size_t)njobs, cudaMemcpyHostToDevice, st));
        bool done = false;
        if (pixel_integrate) {
            /* plans of the grids not seen yet */
            std::vector<gfk::IntegPlanDesc> nd;
            std::vector<unsigned char *> job_plan(njobs, nullptr);
            for (int j : integ) {
                const SkyModel &m = R[j].hm[i].m;
                auto key = std::make_tuple(m.m0, m.dm, m.M1, m.dM, m.nM, m.nm);
                auto it = plans.find(key);
                if (it == plans.end()) {
                    gfk::IntegPlanDesc d;
                    memset(&d, 0, sizeof(d));
                    const size_t bytes = gfk::integ_plan_bytes(m.nm, m.nM, &d.max_anchors, &d.max_slots);
                    GF_TRY(pool.alloc(&d.plan, bytes));
                    d.Dtab = hj[j].Dtab;
                    d.nm = m.nm; d.nM = m.nM; d.nM_tab = m.nM;
                    nd.push_back(d);
                    it = plans.insert({key, d.plan}).first;
                }
                job_plan[j] = it->second;
            }
            if (!nd.empty()) {
                GF_TRY(ws.pdesc.need(nd.size()));
                GF_CUDA(cudaMemcpyAsync(ws.pdesc.p, nd.data(), sizeof(gfk::IntegPlanDesc) * nd.size(), cudaMemcpyHostToDevice, st));
                GF_CUDA(gfk::launch_integ_plans(ws.pdesc.p, (int)nd.size(), st));
            }
            /* every plan's header: slot count, and whether it fitted */
            std::vector<unsigned char *> uniq;
            for (auto &kv : plans) uniq.push_back(kv.second);
            GF_TRY(ws.h_stage.need(sizeof(gfk::IntegPlanHdr) * uniq.size()));
            gfk::IntegPlanHdr *hh = (gfk::IntegPlanHdr *)ws.h_stage.p;
            for (size_t q = 0; q < uniq.size(); q++)
                GF_CUDA(cudaMemcpyAsync(hh + q, uniq[q], sizeof(gfk::IntegPlanHdr), cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaStreamSynchronize(st));
            bool ok = true;
            int slots_max = 1, nm_max = 1, nM_max = 1;
            for (size_t q = 0; q < uniq.size(); q++) {
                ok = ok && hh[q].ok;
                slots_max = std::max(slots_max, hh[q].nslots);
                plan_nslots[uniq[q]] = hh[q].nslots;
            }
            for (int j : integ) {
                nm_max = std::max(nm_max, R[j].hm[i].m.nm);
                nM_max = std::max(nM_max, R[j].hm[i].m.nM);
            }
            gfk::IntegPixParams P;
            memset(&P, 0, sizeof(P));
            if (ok && gfk::integ_warp_bytes(nm_max, nM_max, slots_max, &P) <= 200 * 1024) {
                GF_CUDA(cudaMemcpyAsync(ws.plans.p, job_plan.data(), sizeof(unsigned char *) * (size_t)njobs, cudaMemcpyHostToDevice, st));
                P.jobs = d_jobs;
                P.plans = ws.plans.p;
                P.pix_off = ws.pixoff.p;
                P.njobs = njobs;
                P.total_pix = (int32_t)pix_total;
                P.pix_sum = ws.pixsum.p;
                P.next = d_counter;
                {
                    ProfScope ps(ctx, GF_PROF_INTEGRATE);
                    GF_CUDA(gfk::launch_integrate_pixels(P, model_kind(R[integ[0]].hm[i].m.type), ws.tot.p, st));
                }
                GF_CUDA(cudaMemcpyAsync(htot.data(), ws.tot.p, sizeof(double2) * (size_t)njobs, cudaMemcpyDeviceToHost, st));
                GF_CUDA(cudaStreamSynchronize(st));
                for (int j : integ) {
                    S[j].expected[i] = htot[j].x;
                    S[j].expected_covered[i] = htot[j].y;
                }
                done = true;
                plan_used[i] = 1;
            }
        }
        if (!done) {
            /* the stream crawl (a grid whose plan does not fit) */
            if (!items_integ) {
                GF_TRY(upload_items(integ, &nitems));
                items_integ = true;
            }
            GF_CUDA(cudaMemsetAsync(d_counts, 0, 16 * nall, st));
            gfk::LaunchCrawlMulti L;
            memset(&L, 0, sizeof(L));
            L.jobs = d_jobs; L.items = d_items; L.nitems = nitems; L.counter = d_counter;
            L.model_type = model_kind(R[integ[0]].hm[i].m.type);
            L.max_tab = max_tab(i, integ);
            L.jt = ctx->jt;
            {
                ProfScope ps(ctx, GF_PROF_INTEGRATE);
                GF_CUDA(gfk::launch_crawl_multi(L, 0, st));
            }
            GF_TRY(ws.h_stage.need(16 * nall));
            GF_CUDA(cudaMemcpyAsync(ws.h_stage.p, d_counts, 16 * nall, cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaStreamSynchronize(st));
            /* the per-stream sums, read in place from the page-locked staging area */
            const double *hc = (const double *)ws.h_stage.p;
            for (int j : integ) {
                double e = 0, ec = 0;
                for (int t = 0; t < N; t++) {
                    e += hc[(size_t)j * N + t];
                    ec += hc[nall + (size_t)j * N + t];
                }
                S[j].expected[i] = e;
                S[j].expected_covered[i] = ec;
            }
        }
        for (int j : integ) {
            /* room for the Poisson spread of the model's stars in one batch */
            const double e = S[j].expected[i];
            if (e + ctx->admit_sigma * sqrt(e) + 1024.0 >= (double)jobs[j].capacity) R[j].plain = true;
        }
    }

    /* ---- requests generated together ---- */
    /* device memory of a batched request's draw passes: records, sort keys and
     * output columns take about kStarBytes per star of its largest model, events 48
     * bytes per star at most, and the slot densities of its pixels */
    const double kStarBytes = 256.0;
    auto need_of = [&](int j) {
        double mx = 0;
        for (int i = 0; i < nmod; i++) mx = std::max(mx, S[j].expected[i] + 8.0 * sqrt(S[j].expected[i]) + 1024.0);
        int ns = 0;
        for (int i = 0; i < nmod; i++)
            if (plan_used[i] && plan_of(j, i)) ns = std::max(ns, plan_nslots[plan_of(j, i)]);
        return mx * (kStarBytes + 48.0) + 8.0 * (double)jobs[j].npixels * (ns + 1) +
               16.0 * (double)R[j].hm[0].m.nm * R[j].hm[0].m.nM / GF_BLOCK;
    };
    int64_t budget = ctx->multi_budget;
    if (adm && adm->admit) {
        /* the caller admits the leading batched requests (in submission order) whose
         * memory it can grant now; the others are left for a later call */
        adm->deferred.assign(njobs, 0);
        std::vector<int> cand;
        for (int j = 0; j < njobs; j++)
            if (!R[j].plain) cand.push_back(j);
        if (!cand.empty()) {
            std::vector<double> need(cand.size());
            for (size_t k = 0; k < cand.size(); k++) need[k] = need_of(cand[k]);
            int64_t granted = 0;
            int32_t take = adm->admit(adm->user, need.data(), (int32_t)cand.size(), &granted);
            take = std::max<int32_t>(1, std::min<int32_t>(take, (int32_t)cand.size()));
            for (size_t k = (size_t)take; k < cand.size(); k++) {
                R[cand[k]].deferred = true;
                adm->deferred[cand[k]] = 1;
            }
            if (granted > 0) budget = granted;
        }
    }
    std::vector<int> batched_all;
    for (int j : order_all)
        if (!R[j].plain && !R[j].deferred) batched_all.push_back(j);
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        GF_CUDA(cudaMemGetInfo(&fr, &tot));
        budget = (int64_t)(0.6 * (double)fr);
    }
    /* chunks of requests whose draw passes fit the memory budget */
    std::vector<std::vector<int>> chunks;
    {
        double used = 0;
        for (int j : batched_all) {
            const double need = need_of(j);
            if (chunks.empty() || (used + need > (double)budget && !chunks.back().empty())) {
                chunks.emplace_back();
                used = 0;
            }
            chunks.back().push_back(j);
            used += need;
        }
    }

    std::vector<int32_t> job_slot(njobs, 0);
    int32_t *d_job_slot = nullptr, *d_slot_job = nullptr, *d_slot_comp = nullptr;
    int64_t *d_seg = nullptr, *d_row_begin = nullptr, *d_slot_rows = nullptr, *d_chunk_begin = nullptr, *d_catoff = nullptr;
    uint64_t *d_pseed = nullptr;
    gf_footprint *d_foot = nullptr;
    GF_TRY(ws.job_slot.need((size_t)njobs));
    d_job_slot = ws.job_slot.p;
    GF_TRY(ws.slot_job.need((size_t)njobs));
    d_slot_job = ws.slot_job.p;
    GF_TRY(ws.slot_comp.need((size_t)njobs));
    d_slot_comp = ws.slot_comp.p;
    GF_TRY(ws.seg.need(3 * (size_t)njobs));
    d_seg = ws.seg.p;
    GF_TRY(ws.row_begin.need((size_t)njobs + 1));
    d_row_begin = ws.row_begin.p;
    GF_TRY(ws.slot_rows.need((size_t)njobs));
    d_slot_rows = ws.slot_rows.p;
    GF_TRY(ws.chunk_begin.need((size_t)njobs));
    d_chunk_begin = ws.chunk_begin.p;
    GF_TRY(ws.catoff.need((size_t)njobs));
    d_catoff = ws.catoff.p;
    GF_TRY(ws.pseed.need((size_t)njobs));
    d_pseed = ws.pseed.p;
    GF_TRY(ws.foot.need((size_t)njobs));
    d_foot = ws.foot.p;
    bool any_foot = false;
    {
        std::vector<gf_footprint> foot(njobs);
        std::vector<uint64_t> pseed(njobs, 0);
        for (int j = 0; j < njobs; j++) {
            memset(&foot[j], 0, sizeof(gf_footprint));
            if (jobs[j].foot) { foot[j] = *jobs[j].foot; any_foot = any_foot || foot[j].kind != GF_FOOT_ALL; }
            if (jobs[j].perr) pseed[j] = jobs[j].perr->seed;
        }
        GF_CUDA(cudaMemcpyAsync(d_foot, foot.data(), sizeof(gf_footprint) * (size_t)njobs, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaMemcpyAsync(d_pseed, pseed.data(), 8 * (size_t)njobs, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaStreamSynchronize(st));
    }
    /* photometry and photometric-error tables of each module group */
    struct GroupMods { gf_photometry *ph = nullptr; gf_photoerr *pe = nullptr; };
    std::vector<GroupMods> gm(groups.size());
    struct ModGuard {
        std::vector<GroupMods> *g;
        ~ModGuard() { for (auto &x : *g) { gf_photometry_destroy(x.ph); gf_photoerr_destroy(x.pe); } }
    } mod_guard{&gm};
    if (!batched_all.empty())
        for (int g = 0; g < (int)group_rep.size(); g++) {
            const gf_job &J = jobs[group_rep[g]];
            if (J.phot) GF_TRY(gf_photometry_create(ctx, J.phot, &gm[g].ph));
            if (J.perr) GF_TRY(gf_photoerr_create(ctx, J.perr, &gm[g].pe));
        }

    /* growing buffers of the draw passes */
    auto &rec = ws.rec;
    auto &row_slot = ws.row_slot;
    auto &key = ws.key, &key_b = ws.key_b;
    auto &idx_a = ws.idx_a, &idx_b = ws.idx_b;
    auto &temp = ws.temp;
    std::vector<int64_t> catoff(njobs, 0);
    /* host delivery: copy stream, events and the page-locked ring */
    HostDelivery hd;
    const bool to_host = hcb != nullptr;
    if (to_host) {
        if (!ws.copy_stream) {
            GF_CUDA(cudaStreamCreateWithFlags(&ws.copy_stream, cudaStreamNonBlocking));
            for (int b = 0; b < 2; b++) {
                GF_CUDA(cudaEventCreateWithFlags(&ws.ev_pass[b], cudaEventDisableTiming));
                GF_CUDA(cudaEventCreateWithFlags(&ws.ev_free[b], cudaEventDisableTiming));
                GF_CUDA(cudaEventCreateWithFlags(&ws.ev_stage[b], cudaEventDisableTiming));
                GF_CUDA(cudaEventCreateWithFlags(&ws.ev_stage_free[b], cudaEventDisableTiming));
            }
        }
        ws.free_recorded[0] = ws.free_recorded[1] = false;
        ws.stage_recorded[0] = ws.stage_recorded[1] = false;
        hd.cb = hcb;
        hd.user = user;
        hd.piece_rows = piece_rows > 0 ? piece_rows : (int64_t)16 << 20;
        hd.nbands = nbands;
        const size_t slot_bytes = carved_bytes(hd.piece_rows, nbands, ctx->host_cols);
        GF_TRY(ws.ring.need(slot_bytes * GF_RING));
        for (int r = 0; r < GF_RING; r++)
            hd.ring[r] = carve_table(ws.ring.p + (size_t)r * slot_bytes, hd.piece_rows, nbands, ctx->host_cols);
    }
    /* the copy stream finishes (and stops calling back) before this function returns */
    struct CopyDrain {
        MultiWS *ws;
        bool on;
        ~CopyDrain() { if (on && ws->copy_stream) cudaStreamSynchronize(ws->copy_stream); }
    } copy_drain{&ws, to_host};
    int pass = 0;

    for (const std::vector<int> &batched : chunks) {
        /* output order of the chunk: by module group, then request */
        std::vector<int> slot_job = batched;
        std::stable_sort(slot_job.begin(), slot_job.end(), [&](int a, int b) { return R[a].group != R[b].group ? R[a].group < R[b].group : a < b; });
        const int nslots = (int)slot_job.size();
        for (int sl = 0; sl < nslots; sl++) job_slot[slot_job[sl]] = sl;
        GF_CUDA(cudaMemcpyAsync(d_job_slot, job_slot.data(), 4 * (size_t)njobs, cudaMemcpyHostToDevice, st));
        GF_CUDA(cudaMemcpyAsync(d_slot_job, slot_job.data(), 4 * (size_t)nslots, cudaMemcpyHostToDevice, st));
        bool items_chunk = false;      /* per-stream items of the crawl draw, uploaded when needed */
        int slot_bits = 1;
        while ((1 << slot_bits) < nslots) slot_bits++;

        for (int i = 0; i < nmod; i++) {
            for (int j = 0; j < njobs; j++) hj[j] = crawl_job(j, i);
            GF_CUDA(cudaMemcpyAsync(d_jobs, hj.data(), sizeof(CrawlJob) * (size_t)njobs, cudaMemcpyHostToDevice, st));
            double want = 65536;
            for (int j : batched) want += S[j].expected[i] + 8.0 * sqrt(S[j].expected[i]) + 1024.0;
            int64_t cap = (int64_t)want;
            GF_CUDA(cudaMemcpyAsync(d_rng_snap, d_rng, 12 * (size_t)njobs * NS, cudaMemcpyDeviceToDevice, st));
            /* the kernels' model kind: exponential disks, or the ellipsoids (power laws,
             * broken power laws, LC bulges: their density is chosen per request) */
            const int mtype = model_kind(R[batched[0]].hm[i].m.type);
            GF_TRY(rec.need((size_t)cap));
            int64_t nrec = 0;
            if (plan_used[i]) {
                /* slot densities of the chunk's pixels */
                std::vector<const unsigned char *> jp(njobs, nullptr);
                std::vector<float2 *> jm(njobs, nullptr);
                std::vector<int32_t> jl, poff;
                std::vector<int64_t> moff(njobs, 0);
                int64_t ms_total = 0;
                int32_t tp = 0;
                for (int j : batched) {
                    jp[j] = plan_of(j, i);
                    moff[j] = ms_total;
                    ms_total += (int64_t)jobs[j].npixels * (plan_nslots[jp[j]] + 1);
                    jl.push_back(j);
                    poff.push_back(tp);
                    tp += jobs[j].npixels;
                }
                poff.push_back(tp);
                GF_TRY(ws.msbuf.need((size_t)std::max<int64_t>(ms_total, 1)));
                for (int j : batched) jm[j] = ws.msbuf.p + moff[j];
                GF_TRY(ws.msptr.need((size_t)njobs));
                GF_TRY(ws.joblist.need(jl.size()));
                GF_TRY(ws.chunkoff.need(poff.size()));
                GF_CUDA(cudaMemcpyAsync(ws.plans.p, jp.data(), sizeof(void *) * (size_t)njobs, cudaMemcpyHostToDevice, st));
                GF_CUDA(cudaMemcpyAsync(ws.msptr.p, jm.data(), sizeof(void *) * (size_t)njobs, cudaMemcpyHostToDevice, st));
                GF_CUDA(cudaMemcpyAsync(ws.joblist.p, jl.data(), 4 * jl.size(), cudaMemcpyHostToDevice, st));
                GF_CUDA(cudaMemcpyAsync(ws.chunkoff.p, poff.data(), 4 * poff.size(), cudaMemcpyHostToDevice, st));
                gfk::SlotDensityParams SD;
                SD.jobs = d_jobs; SD.plans = ws.plans.p; SD.ms = ws.msptr.p;
                SD.job_list = ws.joblist.p; SD.pix_off = ws.chunkoff.p;
                SD.njobs = (int32_t)jl.size(); SD.total_pix = tp;
                {
                    ProfScope ps(ctx, GF_PROF_SLOTS);
                    GF_CUDA(gfk::launch_slot_density(SD, mtype, st));
                }
                /* the record of every block of every request (the draw's bound walk) */
                {
                    std::vector<uint4 *> lp(njobs, nullptr);
                    std::vector<int64_t> boff;
                    int64_t nb_total = 0;
                    for (int j : batched) {
                        boff.push_back(nb_total);
                        nb_total += (int64_t)R[j].hm[i].m.nm * R[j].hm[i].m.nM / GF_BLOCK;
                    }
                    boff.push_back(nb_total);
                    GF_TRY(ws.brec.need((size_t)std::max<int64_t>(nb_total, 1)));
                    for (size_t q = 0; q < batched.size(); q++) lp[batched[q]] = ws.brec.p + boff[q];
                    GF_TRY(ws.brecptr.need((size_t)njobs));
                    GF_TRY(ws.blkoff.need(boff.size()));
                    GF_CUDA(cudaMemcpyAsync(ws.brecptr.p, lp.data(), sizeof(void *) * (size_t)njobs, cudaMemcpyHostToDevice, st));
                    GF_CUDA(cudaMemcpyAsync(ws.blkoff.p, boff.data(), 8 * boff.size(), cudaMemcpyHostToDevice, st));
                    gfk::BlockLfParams BL;
                    BL.jobs = d_jobs; BL.plans = ws.plans.p; BL.brec = ws.brecptr.p;
                    BL.job_list = ws.joblist.p; BL.blk_off = ws.blkoff.p;
                    BL.njobs = (int32_t)batched.size(); BL.total = nb_total;
                    ProfScope ps(ctx, GF_PROF_SLOTS);
                    GF_CUDA(gfk::launch_block_records(BL, st));
                    /* the host vectors are read by the copies above before they go out of scope */
                    GF_CUDA(cudaStreamSynchronize(st));
                }
                gfk::BatchDrawParams B;
                memset(&B, 0, sizeof(B));
                B.brec = ws.brecptr.p;
                if (gfk::batch_draw_warp_bytes(max_tab(i, batched), &B) > 200 * 1024)
                    return fail(GF_E_UNSUPPORTED, "magnitude grid too large for the batched draw");
                B.jobs = d_jobs; B.plans = ws.plans.p; B.ms = ws.msptr.p;
                /* work items: 32 consecutive streams of a request, requests in decreasing size;
                 * first the requests that take the block bound of their expected counts
                 * (non-negative densities, no distance limits), then the others */
                const int ngroups = (N + 31) / 32;
                GF_TRY(ws.gitems.need((size_t)batched.size() * ngroups));
                int32_t nbound = 0;
                {
                    GF_TRY(ws.h_stage.need(4 * batched.size() * (size_t)ngroups));
                    uint32_t *gi = (uint32_t *)ws.h_stage.p;
                    size_t q = 0;
                    for (int pass_bound = 1; pass_bound >= 0; pass_bound--) {
                        for (int j : batched) {
                            const SkyModel &mj = R[j].hm[i].m;
                            const bool bj = mj.dmin == 0.f && mj.dmax == 0.f && mj.f >= 0.f && mj.norm >= 0.f;
                            if (bj != (pass_bound == 1)) continue;
                            for (int g = 0; g < ngroups; g++) gi[q++] = ((uint32_t)j << 16) | (uint32_t)(32 * g);
                        }
                        if (pass_bound == 1) nbound = (int32_t)q;
                    }
                    GF_CUDA(cudaMemcpyAsync(ws.gitems.p, gi, 4 * q, cudaMemcpyHostToDevice, st));
                    GF_CUDA(cudaStreamSynchronize(st));
                }
                const int32_t ngitems = (int32_t)(batched.size() * (size_t)ngroups);
                B.items = ws.gitems.p; B.nitems = ngitems; B.next_item = d_counter;
                B.ev_count = ctx->d_counters; B.err = ctx->d_counters + 2;
                GF_TRY(ws.ev.need((size_t)cap));
                B.ev = ws.ev.p; B.ev_capacity = (int64_t)ws.ev.n;
                /* the two launches of a draw pass: bound requests, then exact ones */
                auto draw_all = [&](const gfk::BatchDrawParams &BB, int wpc) -> gf_status {
                    gfk::BatchDrawParams X = BB;
                    X.nitems = nbound;
                    GF_CUDA(gfk::launch_batch_draw(X, mtype, wpc, true, st));
                    X.items = BB.items + nbound;
                    X.nitems = ngitems - nbound;
                    GF_CUDA(gfk::launch_batch_draw(X, mtype, wpc, false, st));
                    return GF_OK;
                };
                if (ctx->draw_wpc[mtype] == 0) {
                    /* autotuner: time 8, 4, 2 and 1 warps per CTA on the head of the work queue
                     * (the largest requests), from the same stream states, and keep the fastest */
                    const bool tb = nbound > 0;
                    gfk::BatchDrawParams T = B;
                    const int32_t avail = tb ? nbound : ngitems;
                    T.items = B.items + (tb ? 0 : nbound);
                    T.nitems = std::min<int32_t>(avail, std::max<int32_t>(avail / 16, 148 * 8));
                    float best_ms = 0.f;
                    int best = 4;
                    cudaEvent_t e0, e1;
                    GF_CUDA(cudaEventCreate(&e0));
                    GF_CUDA(cudaEventCreate(&e1));
                    for (int wpc : {8, 4, 2, 1}) {
                        GF_CUDA(cudaMemcpyAsync(d_rng, d_rng_snap, 12 * (size_t)njobs * NS, cudaMemcpyDeviceToDevice, st));
                        GF_CUDA(cudaMemsetAsync(ctx->d_counters, 0, 24, st));
                        GF_CUDA(cudaEventRecord(e0, st));
                        GF_CUDA(gfk::launch_batch_draw(T, mtype, wpc, tb, st));
                        GF_CUDA(cudaEventRecord(e1, st));
                        GF_CUDA(cudaEventSynchronize(e1));
                        float ms = 0.f;
                        GF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                        if (wpc == 8 || ms < best_ms) { best_ms = ms; best = wpc; }
                    }
                    cudaEventDestroy(e0);
                    cudaEventDestroy(e1);
                    ctx->draw_wpc[mtype] = best;
                    GF_CUDA(cudaMemcpyAsync(d_rng, d_rng_snap, 12 * (size_t)njobs * NS, cudaMemcpyDeviceToDevice, st));
                }
                int64_t nev = 0;
                for (;;) {
                    GF_CUDA(cudaMemsetAsync(ctx->d_counters, 0, 24, st));
                    {
                        ProfScope ps(ctx, GF_PROF_BATCH_DRAW);
                        GF_TRY(draw_all(B, ctx->draw_wpc[mtype]));
                    }
                    GF_CUDA(cudaMemcpyAsync(ctx->h_counters, ctx->d_counters, 24, cudaMemcpyDeviceToHost, st));
                    GF_CUDA(cudaStreamSynchronize(st));
                    nev = (int64_t)ctx->h_counters[0];
                    if (ctx->h_counters[2] & 2ull) return fail(GF_E_STATE, "internal: a request without the block bound in the bound draw");
                    if (ctx->h_counters[2]) return fail(GF_E_INVALID, "a bin has an infinite expected star count");
                    if (nev <= B.ev_capacity) break;
                    /* more bins with stars than the event list holds: restore the streams and draw again */
                    GF_CUDA(cudaMemcpyAsync(d_rng, d_rng_snap, 12 * (size_t)njobs * NS, cudaMemcpyDeviceToDevice, st));
                    GF_TRY(ws.ev.need((size_t)(nev + nev / 8 + 65536)));
                    B.ev = ws.ev.p; B.ev_capacity = (int64_t)ws.ev.n;
                }
                /* the star records of the events */
                GF_TRY(ws.k64.need((size_t)std::max<int64_t>(nev, 1)));
                GF_TRY(ws.off64.need((size_t)std::max<int64_t>(nev, 1)));
                size_t tb = 0;
                GF_CUDA(gfk::expand_temp_bytes(nev, &tb));
                GF_TRY(temp.need(tb + 256));
                int64_t *d_total = (int64_t *)(ctx->d_counters + 1);
                for (;;) {
                    {
                        ProfScope ps(ctx, GF_PROF_EXPAND);
                        GF_CUDA(gfk::launch_expand_events(ws.ev.p, nev, d_jobs, ws.k64.p, ws.off64.p, temp.p, temp.n, rec.p,
                                                          (int64_t)rec.n, d_total, st));
                    }
                    GF_CUDA(cudaMemcpyAsync(ctx->h_counters + 1, ctx->d_counters + 1, 8, cudaMemcpyDeviceToHost, st));
                    GF_CUDA(cudaStreamSynchronize(st));
                    nrec = (int64_t)ctx->h_counters[1];
                    if (nrec <= (int64_t)rec.n) break;
                    GF_TRY(rec.need((size_t)(nrec + nrec / 8 + 65536)));
                }
            } else {
                if (!items_chunk) {
                    GF_TRY(upload_items(batched, &nitems));
                    items_chunk = true;
                }
                for (;;) {
                    GF_TRY(rec.need((size_t)cap));
                    GF_CUDA(cudaMemsetAsync(cs_base, 0, cs_bytes, st));
                    GF_CUDA(cudaMemsetAsync(ctx->d_counters, 0, 24, st));
                    gfk::LaunchCrawlMulti L;
                    memset(&L, 0, sizeof(L));
                    L.jobs = d_jobs; L.items = d_items; L.nitems = nitems; L.counter = d_counter;
                    L.model_type = mtype;
                    L.max_tab = max_tab(i, batched);
                    L.jt = ctx->jt;
                    L.rec = rec.p; L.rec_capacity = (int64_t)rec.n;
                    L.rec_count = ctx->d_counters; L.err = ctx->d_counters + 2;
                    L.cw = 1;
                    {
                        ProfScope ps(ctx, GF_PROF_DRAW_WINDOW);
                        GF_CUDA(gfk::launch_crawl_multi(L, 1, st));
                    }
                    GF_CUDA(cudaMemcpyAsync(ctx->h_counters, ctx->d_counters, 24, cudaMemcpyDeviceToHost, st));
                    GF_CUDA(cudaStreamSynchronize(st));
                    nrec = (int64_t)ctx->h_counters[0];
                    if (ctx->h_counters[2]) return fail(GF_E_INVALID, "a bin has an infinite expected star count");
                    if (nrec <= (int64_t)rec.n) break;
                    /* more stars than the buffer holds: restore the streams and draw again */
                    GF_CUDA(cudaMemcpyAsync(d_rng, d_rng_snap, 12 * (size_t)njobs * NS, cudaMemcpyDeviceToDevice, st));
                    cap = nrec + nrec / 8 + 65536;
                }
            }
            /* the (request, star_comp) sort of the records; placement follows in sorted order */
            const size_t n = (size_t)std::max<int64_t>(nrec, 1);
            GF_TRY(key.need(n)); GF_TRY(key_b.need(n)); GF_TRY(idx_a.need(n)); GF_TRY(idx_b.need(n));
            size_t tb = 0;
            GF_CUDA(gfk::sort_temp_bytes_multi((int64_t)n, &tb));
            GF_TRY(temp.need(tb + 256));
            GF_CUDA(cudaMemsetAsync(d_seg, 0, 24 * (size_t)nslots, st));
            gfk::LaunchPlaceMulti PL;
            memset(&PL, 0, sizeof(PL));
            PL.jobs = d_jobs; PL.job_slot = d_job_slot; PL.rec = rec.p; PL.n = nrec;
            PL.key = key.p; PL.key_b = key_b.p;
            PL.idx_a = idx_a.p; PL.idx_b = idx_b.p; PL.slot_bits = slot_bits;
            PL.temp = temp.p; PL.temp_bytes = temp.n;
            PL.seg_begin = d_seg; PL.vis_end = d_seg + nslots; PL.seg_end = d_seg + 2 * nslots;
            {
                ProfScope ps(ctx, GF_PROF_SORT);
                GF_CUDA(gfk::launch_place_sort_multi(PL, st));
            }
            std::vector<int64_t> seg(3 * (size_t)nslots);
            GF_CUDA(cudaMemcpyAsync(seg.data(), d_seg, 24 * (size_t)nslots, cudaMemcpyDeviceToHost, st));
            GF_CUDA(cudaStreamSynchronize(st));
            std::vector<int64_t> row_begin(nslots + 1, 0), slot_rows(nslots), chunk_begin(nslots);
            std::vector<int32_t> slot_comp(nslots);
            int64_t nchunks = 0;
            for (int s = 0; s < nslots; s++) {
                const int j = slot_job[s];
                const int64_t gen = seg[2 * nslots + s] - seg[s];
                const int64_t vis = gen > 0 ? seg[nslots + s] - seg[s] : 0;
                if (gen >= jobs[j].capacity && !R[j].overflow) {
                    /* the batch rules of the plain path apply: withhold this request's rows
                     * from here on and run it alone after the batched passes */
                    R[j].overflow = true;
                    R[j].plain = true;
                }
                if (R[j].overflow) {
                    /* no rows of this slot in the output: its visible range ends where it begins */
                    seg[nslots + s] = seg[s];
                    GF_CUDA(cudaMemcpyAsync(d_seg + nslots + s, &seg[nslots + s], 8, cudaMemcpyHostToDevice, st));
                    slot_rows[s] = 0;
                    row_begin[s + 1] = row_begin[s];
                    chunk_begin[s] = nchunks;
                    slot_comp[s] = R[j].hm[i].m.comp;
                    continue;
                }
                R[j].delivered.push_back(R[j].hm[i].m.comp);
                S[j].generated[i] = gen;
                S[j].stored[i] = vis;
                if (vis > 0) S[j].batches++;
                slot_rows[s] = vis;
                row_begin[s + 1] = row_begin[s] + vis;
                chunk_begin[s] = nchunks;
                nchunks += (vis + 255) / 256;
                slot_comp[s] = R[j].hm[i].m.comp;
            }
            const int64_t total = row_begin[nslots];
            /* host delivery: this pass's table must have been copied out by its previous user */
            const int ob = to_host ? (pass & 1) : 0;
            gf_table &out = ob ? ws.out2 : ws.out;
            if (to_host && ws.free_recorded[ob]) GF_CUDA(cudaStreamWaitEvent(st, ws.ev_free[ob], 0));
            if (out.capacity < std::max<int64_t>(total, 1) || out.nbands < nbands) {
                if (to_host) GF_CUDA(cudaStreamSynchronize(ws.copy_stream));
                gf_table_free(ctx, &out);
                GF_TRY(gf_table_alloc(ctx, std::max<int64_t>(total + total / 8, 1024), nbands, &out));
            }
            GF_TRY(row_slot.need((size_t)out.capacity));
            GF_CUDA(cudaMemcpyAsync(d_row_begin, row_begin.data(), 8 * (size_t)(nslots + 1), cudaMemcpyHostToDevice, st));
            GF_CUDA(cudaMemcpyAsync(d_slot_rows, slot_rows.data(), 8 * (size_t)nslots, cudaMemcpyHostToDevice, st));
            GF_CUDA(cudaMemcpyAsync(d_chunk_begin, chunk_begin.data(), 8 * (size_t)nslots, cudaMemcpyHostToDevice, st));
            GF_CUDA(cudaMemcpyAsync(d_slot_comp, slot_comp.data(), 4 * (size_t)nslots, cudaMemcpyHostToDevice, st));
            GF_CUDA(cudaMemcpyAsync(d_catoff, catoff.data(), 8 * (size_t)njobs, cudaMemcpyHostToDevice, st));
            {
                ProfScope ps(ctx, GF_PROF_PLACE);
                GF_CUDA(gfk::launch_tie_place_multi(PL, d_row_begin, d_slot_comp, out, row_slot.p, st));
            }
            out.size = total;
            GF_TRY(gfa::zero_module_rows(ctx, &out, total));
            out.systems = J0.multiples ? 1 : 0;
            /* the module chain in pipeline order (pipeline.h:75-88) over every request's rows */
            gfk::MultiRows MR;
            MR.row_slot = row_slot.p; MR.slot_row_begin = d_row_begin; MR.slot_job = d_slot_job;
            if (total > 0) {
                if (any_foot) {
                    ProfScope ps(ctx, GF_PROF_CLIPPER);
                    GF_CUDA(gfk::launch_clipper_multi(d_foot, MR, out, 0, total, st));
                }
                if (J0.feh) GF_TRY(gf_module_fixedfeh(ctx, J0.feh, &out, 0, total));
                if (J0.feh_ivezic || J0.feh_gauss) {
                    ProfScope ps(ctx, GF_PROF_FEH);
                    if (J0.feh_ivezic)
                        GF_CUDA(gfk::launch_feh_multi(J0.feh_ivezic, nullptr, d_rng, NS, MR, d_chunk_begin, nslots, nchunks,
                                                      d_slot_rows, out, st));
                    if (J0.feh_gauss)
                        GF_CUDA(gfk::launch_feh_multi(nullptr, J0.feh_gauss, d_rng, NS, MR, d_chunk_begin, nslots, nchunks,
                                                      d_slot_rows, out, st));
                }
                if (J0.multiples) {
                    ProfScope ps(ctx, GF_PROF_FEH);
                    GF_CUDA(gfk::launch_multiples_multi(*J0.multiples, d_rng, NS, MR, d_chunk_begin, nslots, nchunks, d_slot_rows,
                                                        out, st));
                }
                if (J0.kin) {
                    ProfScope ps(ctx, GF_PROF_BOND2010);
                    GF_CUDA(gfk::launch_bond2010_multi(*J0.kin, d_rng, NS, MR, d_chunk_begin, nslots, nchunks, d_slot_rows, out, st));
                }
                int s0 = 0;
                while (s0 < nslots) {
                    const int g = R[slot_job[s0]].group;
                    int s1 = s0;
                    while (s1 < nslots && R[slot_job[s1]].group == g) s1++;
                    const int64_t b = row_begin[s0], e = row_begin[s1];
                    if (gm[g].ph) GF_TRY(gf_module_photometry(ctx, gm[g].ph, &out, b, e));
                    if (gm[g].pe) {
                        ProfScope ps(ctx, GF_PROF_PHOTOERR);
                        GF_CUDA(gfk::launch_photoerrors_multi(gm[g].pe->tab, d_pseed, d_catoff, MR, out, b, e, st));
                    }
                    s0 = s1;
                }
                if (J0.v2pm) GF_TRY(gf_module_vel2pm(ctx, J0.v2pm, &out, 0, total));
                if (J0.gal2other) GF_TRY(gf_module_gal2other(ctx, J0.gal2other, &out, 0, total));
            }
            if (to_host) {
                GF_TRY(deliver_pass(ws, hd, ob, st, out, R[batched[0]].hm[i].m.comp, slot_job, row_begin, slot_rows, njobs));
                if (hd.stop.load()) return fail(GF_E_STATE, "stopped by the host callback");
            } else {
                GF_CUDA(cudaStreamSynchronize(st));
                if (cb) {
                    std::vector<int64_t> rb(njobs, 0), rc(njobs, 0);
                    for (int s = 0; s < nslots; s++) { rb[slot_job[s]] = row_begin[s]; rc[slot_job[s]] = slot_rows[s]; }
                    if (cb(user, R[batched[0]].hm[i].m.comp, &out, rb.data(), rc.data()) != 0)
                        return fail(GF_E_STATE, "stopped by the batch callback");
                }
            }
            pass++;
            for (int s = 0; s < nslots; s++) catoff[slot_job[s]] += slot_rows[s];
        }
    }

    /* ---- requests that need the batch rules of the plain path ----
     * With host delivery their rows follow the batched passes' rows through the copy
     * stream (deliveries stay in order) while the device generates them. */
    {
        gfa::ProfScope plain_time(ctx, GF_PROF_PLAIN);
        for (int j = 0; j < njobs; j++) {
            if (!R[j].plain || R[j].deferred) continue;
            if (to_host) {
                if (hd.stop.load()) break;
                PlainHostForward f;
                f.hd = &hd; f.ws = &ws; f.pass = &pass; f.ctx = ctx; f.njobs = njobs; f.job = j;
                f.capacity = jobs[j].capacity;
                f.skip = R[j].delivered;
                const gf_status rs = gfa::catalog_run_in_multi(ctx, &jobs[j], forward_plain_host, &f, &S[j]);
                if (f.err != GF_OK) return fail(f.err, f.msg);
                if (rs != GF_OK && !hd.stop.load()) return rs;
            } else {
                PlainForward f;
                f.cb = cb; f.user = user; f.njobs = njobs; f.job = j;
                f.skip = R[j].delivered;
                f.begin.assign(njobs, 0);
                f.count.assign(njobs, 0);
                GF_TRY(gfa::catalog_run_in_multi(ctx, &jobs[j], forward_plain_batch, &f, &S[j]));
            }
        }
    }
    if (to_host) {
        GF_CUDA(cudaStreamSynchronize(ws.copy_stream));
        if (hd.stop.load()) return fail(GF_E_STATE, "stopped by the host callback");
    }
    return GF_OK;
}

}  // namespace

namespace {
struct CountingMulti {
    gf_multi_callback cb;
    void *user;
    std::atomic<long long> calls{0};
};
int counting_multi(void *u, int32_t model, const gf_table *t, const int64_t *rb, const int64_t *rc)
{
    CountingMulti *c = (CountingMulti *)u;
    c->calls++;
    return c->cb ? c->cb(c->user, model, t, rb, rc) : 0;
}

/* An out-of-memory failure before any rows were delivered frees the context's
 * cached buffers and runs the call once more, as the reference collects garbage
 * and retries a failed allocation (cux.cpp:189-198).  Every request's streams
 * are seeded again, so the retry is the same run. */
gf_status run_multi_retry(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, gf_multi_host_callback hcb,
                          int64_t piece_rows, void *user, gf_catalog_stats *stats, gfa::Admission *adm = nullptr)
{
    CountingMulti c;
    c.cb = cb ? cb : hcb;
    c.user = user;
    gf_multi_callback d = cb ? counting_multi : nullptr;
    gf_multi_host_callback h = hcb ? counting_multi : nullptr;
    gf_status st = run_multi(ctx, jobs, njobs, d, h, piece_rows, &c, stats, adm);
    if (st == GF_E_OOM && c.calls.load() == 0) {
        gfa::release_caches(ctx);
        st = run_multi(ctx, jobs, njobs, d, h, piece_rows, &c, stats, adm);
    }
    return st;
}
}  // namespace

namespace gfa {
gf_status catalog_run_multi_admitted(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, void *user,
                                     gf_catalog_stats *stats, Admission *adm)
{
    return run_multi_retry(ctx, jobs, njobs, cb, nullptr, 0, user, stats, adm);
}
}  // namespace gfa

extern "C" gf_status gf_catalog_run_multi(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, void *user,
                                          gf_catalog_stats *stats)
{
    return run_multi_retry(ctx, jobs, njobs, cb, nullptr, 0, user, stats);
}

extern "C" gf_status gf_catalog_run_multi_host(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, int64_t piece_rows,
                                               gf_multi_host_callback cb, void *user, gf_catalog_stats *stats)
{
    if (!cb) return fail(GF_E_INVALID, "host delivery needs a callback");
    if (piece_rows < 0) return fail(GF_E_INVALID, "negative piece size");
    return run_multi_retry(ctx, jobs, njobs, nullptr, cb, piece_rows, user, stats);
}

extern "C" gf_status gf_multi_set_admission(gf_ctx *ctx, double sigmas)
{
    GF_TRY(gfa::check_ctx(ctx));
    if (!(sigmas >= -1000.0 && sigmas <= 1000.0)) return fail(GF_E_INVALID, "admission margin out of range");
    ctx->admit_sigma = sigmas;
    return GF_OK;
}

extern "C" gf_status gf_multi_set_host_columns(gf_ctx *ctx, uint32_t columns)
{
    GF_TRY(gfa::check_ctx(ctx));
    if (columns & ~(uint32_t)GF_COL_ALL) return fail(GF_E_INVALID, "unknown column bits");
    ctx->host_cols = columns;
    return GF_OK;
}

extern "C" gf_status gf_multi_set_memory_budget(gf_ctx *ctx, int64_t bytes)
{
    GF_TRY(gfa::check_ctx(ctx));
    if (bytes < 0) return fail(GF_E_INVALID, "negative memory budget");
    ctx->multi_budget = bytes;
    return GF_OK;
}

extern "C" gf_status gf_tuning_get(gf_ctx *ctx, int32_t model_kind, int32_t *warps_per_cta)
{
    GF_TRY(gfa::check_ctx(ctx));
    if (model_kind < 1 || model_kind > 2 || !warps_per_cta) return fail(GF_E_INVALID, "invalid arguments");
    *warps_per_cta = ctx->draw_wpc[model_kind];
    return GF_OK;
}

extern "C" gf_status gf_tuning_set(gf_ctx *ctx, int32_t model_kind, int32_t warps_per_cta)
{
    GF_TRY(gfa::check_ctx(ctx));
    if (model_kind < 1 || model_kind > 2) return fail(GF_E_INVALID, "invalid model kind");
    if (warps_per_cta != 0 && warps_per_cta != 1 && warps_per_cta != 2 && warps_per_cta != 4 && warps_per_cta != 8)
        return fail(GF_E_INVALID, "warps per CTA must be 1, 2, 4, 8 or 0 (tune again)");
    ctx->draw_wpc[model_kind] = warps_per_cta;
    return GF_OK;
}
