/*
 * gf_server.cpp -- the serving form: continuous batching of catalog requests.
 *
 * Requests are submitted at any time from any thread; submit copies the job and
 * everything it points to, so the caller's memory may be reused at once.  Each
 * worker thread owns a context (its own CUDA stream, streams, workspace) and
 * repeatedly takes the compatible requests waiting at the head of the queue and
 * generates them together (gf_catalog_run_multi).  Admission happens after the
 * call's integrate pass, when each request's device-memory need is known from
 * its expected star counts: the worker reserves, from the server's memory
 * budget, the needs of the leading requests that fit what is free and generates
 * those; the others go back to the head of the queue, where they join the
 * requests that arrived meanwhile in the next call of whichever worker is free.
 * A batch thus holds one memory-budget pass, a request waits at most for the
 * passes ahead of it, and batches of several workers run side by side on the
 * device when their reservations fit together.  Each request's rows are exactly
 * those gf_catalog_run gives it alone, whatever it was batched with.
 *
 * No counterpart in the reference, which generates one catalog per process.
 */
#include "gf_ctx.h"

#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

/* a job with its own copies of the arrays and configurations it points to */
struct OwnedJob {
    gf_job job;
    std::vector<gf_pencil_beam> pixels;
    std::vector<float> ammin;
    std::vector<gf_model_config> models;
    std::vector<std::vector<double>> lf_M, lf_phi;
    gf_footprint foot;
    gf_fixedfeh_config feh;
    gf_bond2010_config kin;
    gf_photometry_config phot;
    std::vector<float> colors;
    std::vector<uint8_t> eflags;
    gf_photoerr_config perr;
    std::vector<double> perr_mag, perr_sigma;
    gf_vel2pm_config v2pm;
    gf_feh_config feh_ivezic;
    gf_gaussfeh_config feh_gauss;
    gf_multiples_config multiples;
    gf_ext_map maps[2];
    std::vector<float> map_A[2];
    std::vector<std::vector<float>> cubes;
};

template <class T>
const T *copy_one(const T *src, T &dst)
{
    if (!src) return nullptr;
    dst = *src;
    return &dst;
}

/* nullptr when the job's arrays cannot be copied (negative or absurd sizes) */
std::shared_ptr<OwnedJob> own(const gf_job &j)
{
    auto o = std::make_shared<OwnedJob>();
    o->job = j;
    if (j.npixels < 0 || j.nmodels < 0 || j.nmodels > GF_MAX_MODELS) return nullptr;
    if (j.pixels) {
        o->pixels.assign(j.pixels, j.pixels + j.npixels);
        o->job.pixels = o->pixels.data();
    }
    size_t per_beam = 1;
    if (j.ext.kind == GF_EXT_MAPS) {
        /* the maps and the per-beam rows of nz minima */
        const gf_ext_map *mp[2] = {j.ext.north, j.ext.south};
        const gf_ext_map **dst[2] = {&o->job.ext.north, &o->job.ext.south};
        for (int h = 0; h < 2; h++) {
            if (!mp[h]) continue;
            if (!mp[h]->A || mp[h]->n[0] < 1 || mp[h]->n[1] < 1 || mp[h]->n[2] < 1) return nullptr;
            o->maps[h] = *mp[h];
            o->map_A[h].assign(mp[h]->A, mp[h]->A + (size_t)mp[h]->n[0] * mp[h]->n[1] * mp[h]->n[2]);
            o->maps[h].A = o->map_A[h].data();
            *dst[h] = &o->maps[h];
            per_beam = (size_t)mp[h]->n[2];
        }
    }
    if (j.beam_ammin) {
        o->ammin.assign(j.beam_ammin, j.beam_ammin + per_beam * (size_t)j.npixels);
        o->job.beam_ammin = o->ammin.data();
    }
    if (j.models) {
        o->models.assign(j.models, j.models + j.nmodels);
        o->lf_M.resize(j.nmodels);
        o->lf_phi.resize(j.nmodels);
        for (int i = 0; i < j.nmodels; i++) {
            gf_model_config &m = o->models[i];
            if (m.lf_n < 0) return nullptr;
            if (m.lf_M) { o->lf_M[i].assign(m.lf_M, m.lf_M + m.lf_n); m.lf_M = o->lf_M[i].data(); }
            if (m.lf_phi) { o->lf_phi[i].assign(m.lf_phi, m.lf_phi + m.lf_n); m.lf_phi = o->lf_phi[i].data(); }
            if (m.type == GF_MODEL_DENSITY_CUBE && m.cube) {
                if (m.cube_n[0] < 1 || m.cube_n[1] < 1 || m.cube_n[2] < 1) return nullptr;
                o->cubes.emplace_back(m.cube, m.cube + (size_t)m.cube_n[0] * m.cube_n[1] * m.cube_n[2]);
                m.cube = o->cubes.back().data();
            }
        }
        o->job.models = o->models.data();
    }
    o->job.foot = copy_one(j.foot, o->foot);
    o->job.feh = copy_one(j.feh, o->feh);
    o->job.kin = copy_one(j.kin, o->kin);
    o->job.v2pm = copy_one(j.v2pm, o->v2pm);
    o->job.feh_ivezic = copy_one(j.feh_ivezic, o->feh_ivezic);
    o->job.feh_gauss = copy_one(j.feh_gauss, o->feh_gauss);
    o->job.multiples = copy_one(j.multiples, o->multiples);
    if (j.phot) {
        o->phot = *j.phot;
        if (o->phot.nbands < 1 || o->phot.nMr < 0 || o->phot.nFeH < 0) return nullptr;
        const size_t n = (size_t)(o->phot.nbands - 1) * (size_t)o->phot.nMr * (size_t)o->phot.nFeH;
        if (o->phot.colors) { o->colors.assign(o->phot.colors, o->phot.colors + n); o->phot.colors = o->colors.data(); }
        if (o->phot.eflags) { o->eflags.assign(o->phot.eflags, o->phot.eflags + n); o->phot.eflags = o->eflags.data(); }
        o->job.phot = &o->phot;
    }
    if (j.perr) {
        o->perr = *j.perr;
        if (o->perr.nbands < 0 || o->perr.nknots < 0) return nullptr;
        const size_t n = (size_t)o->perr.nbands * (size_t)o->perr.nknots;
        if (o->perr.mag) { o->perr_mag.assign(o->perr.mag, o->perr.mag + n); o->perr.mag = o->perr_mag.data(); }
        if (o->perr.sigma) { o->perr_sigma.assign(o->perr.sigma, o->perr.sigma + n); o->perr.sigma = o->perr_sigma.data(); }
        o->job.perr = &o->perr;
    }
    return o;
}

struct Request {
    int64_t id;
    std::shared_ptr<OwnedJob> owned;
    gf_server_rows rows;
    gf_server_done done;
    void *user;
};

bool same_bytes(const void *a, const void *b, size_t n)
{
    if (!a || !b) return a == b;
    return memcmp(a, b, n) == 0;
}

/* the model kinds of a request in component order (os_skygen.cpp:392-399) */
std::vector<int32_t> model_kinds(const gf_job &j)
{
    std::vector<const gf_model_config *> m;
    for (int i = 0; i < j.nmodels; i++) m.push_back(&j.models[i]);
    std::stable_sort(m.begin(), m.end(), [](const gf_model_config *x, const gf_model_config *y) { return x->comp < y->comp; });
    std::vector<int32_t> k;
    for (auto *p : m) k.push_back(p->type == GF_MODEL_EXP_DISK ? GF_MODEL_EXP_DISK : GF_MODEL_POWER_LAW_ELLIPSOID);
    return k;
}

/* can two requests share one gf_catalog_run_multi call? */
bool compatible(const gf_job &a, const gf_job &b)
{
    if (a.sky.nthreads != b.sky.nthreads || a.nmodels != b.nmodels || a.gal2other != b.gal2other) return false;
    if (a.sky.nstars != 0.f || b.sky.nstars != 0.f || a.nstreams <= 0 || b.nstreams <= 0) return false;
    if (!!a.phot != !!b.phot || !!a.perr != !!b.perr) return false;
    if (!same_bytes(a.feh, b.feh, sizeof(gf_fixedfeh_config)) || !same_bytes(a.kin, b.kin, sizeof(gf_bond2010_config)) ||
        !same_bytes(a.v2pm, b.v2pm, sizeof(gf_vel2pm_config)) || !same_bytes(a.feh_ivezic, b.feh_ivezic, sizeof(gf_feh_config)) ||
        !same_bytes(a.feh_gauss, b.feh_gauss, sizeof(gf_gaussfeh_config)))
        return false;
    /* same model kinds in component order */
    return model_kinds(a) == model_kinds(b);
}

}  // namespace

struct gf_server {
    int device = 0;
    int64_t budget = 0;
    int32_t max_batch = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_idle, cv_budget;
    std::deque<Request> queue;
    int64_t next_id = 0;
    int64_t inflight = 0;                /* submitted and not yet done */
    int64_t reserved = 0;                /* device memory reserved by the running batches */
    int32_t running = 0;                 /* batches holding a reservation */
    int32_t active = 0;                  /* batches taken from the queue and not finished */
    bool paused = false;                 /* gf_server_pause: workers take no new batch */
    bool stop = false;
    gf_status first_error = GF_OK;
    gf_server_info info = {};
    std::vector<std::thread> workers;
};

namespace {

struct BatchForward {
    std::vector<Request> *reqs;
    gf_ctx *ctx;
};

int forward_rows(void *u, int32_t model, const gf_table *dev, const int64_t *row_begin, const int64_t *row_count)
{
    BatchForward *f = (BatchForward *)u;
    std::vector<Request> &r = *f->reqs;
    for (size_t j = 0; j < r.size(); j++) {
        if (row_count[j] <= 0 || !r[j].rows) continue;
        if (r[j].rows(r[j].user, r[j].id, model, f->ctx, dev, row_begin[j], row_count[j]) != 0) return 1;
    }
    return 0;
}

struct Reservation {
    gf_server *s;
    int64_t bytes = 0;
    bool held = false;
};

void release(Reservation &r)
{
    if (!r.held) return;
    {
        std::lock_guard<std::mutex> g(r.s->mu);
        r.s->reserved -= r.bytes;
        r.s->running--;
    }
    r.held = false;
    r.bytes = 0;
    r.s->cv_budget.notify_all();
}

/* the admission hook: wait until the first request's need fits what the running
 * batches leave free (or nothing else runs: a request larger than the whole budget
 * then runs alone), reserve the needs of the leading requests that fit */
int32_t admit(void *u, const double *need, int32_t n, int64_t *budget)
{
    Reservation &r = *(Reservation *)u;
    release(r);                       /* a retried call reserves afresh */
    gf_server *s = r.s;
    std::unique_lock<std::mutex> g(s->mu);
    s->cv_budget.wait(g, [&] { return (double)(s->budget - s->reserved) >= need[0] || s->running == 0; });
    const double avail = std::max((double)(s->budget - s->reserved), need[0]);
    double sum = 0;
    int32_t k = 0;
    while (k < n && sum + need[k] <= avail) sum += need[k++];
    if (k == 0) { k = 1; sum = need[0]; }
    r.bytes = (int64_t)std::ceil(sum);
    r.held = true;
    s->reserved += r.bytes;
    s->running++;
    s->info.peak_reserved = std::max(s->info.peak_reserved, s->reserved);
    s->info.peak_running = std::max(s->info.peak_running, s->running);
    *budget = std::max<int64_t>(r.bytes, 1);
    return k;
}

void worker_main(gf_server *s)
{
    gf_ctx *ctx = nullptr;
    gf_status st = gf_ctx_create(s->device, &ctx);
    if (st != GF_OK) {
        /* no context: this worker fails the requests it takes (gf_catalog_run_multi rejects a null context) */
        ctx = nullptr;
        std::lock_guard<std::mutex> g(s->mu);
        if (s->first_error == GF_OK) s->first_error = st;
    }
    for (;;) {
        std::vector<Request> batch;
        {
            std::unique_lock<std::mutex> g(s->mu);
            s->cv_work.wait(g, [&] { return s->stop || (!s->queue.empty() && !s->paused); });
            if (s->queue.empty() && s->stop) break;
            if (s->queue.empty() || (s->paused && !s->stop)) continue;
            /* the compatible requests at the head of the queue, in arrival order */
            batch.push_back(s->queue.front());
            s->queue.pop_front();
            while (!s->queue.empty() && (int32_t)batch.size() < s->max_batch &&
                   compatible(batch[0].owned->job, s->queue.front().owned->job)) {
                batch.push_back(s->queue.front());
                s->queue.pop_front();
            }
            s->active++;
        }
        std::vector<gf_job> jobs;
        for (auto &r : batch) jobs.push_back(r.owned->job);
        std::vector<gf_catalog_stats> stats(batch.size());
        BatchForward f;
        f.reqs = &batch;
        f.ctx = ctx;
        Reservation res;
        res.s = s;
        gfa::Admission adm;
        adm.admit = admit;
        adm.user = &res;
        st = ctx ? gfa::catalog_run_multi_admitted(ctx, jobs.data(), (int32_t)jobs.size(), forward_rows, &f, stats.data(), &adm)
                 : GF_E_STATE;
        release(res);
        /* deferred requests go back to the head of the queue in arrival order, unless the call failed */
        std::vector<size_t> finished;
        int64_t ndeferred = 0;
        {
            std::lock_guard<std::mutex> g(s->mu);
            for (size_t j = batch.size(); j-- > 0;) {
                if (st == GF_OK && j < adm.deferred.size() && adm.deferred[j]) {
                    s->queue.push_front(batch[j]);
                    ndeferred++;
                }
            }
            s->info.runs++;
            s->info.deferred += ndeferred;
            s->active--;
        }
        if (ndeferred) s->cv_work.notify_all();
        for (size_t j = 0; j < batch.size(); j++) {
            if (st == GF_OK && j < adm.deferred.size() && adm.deferred[j]) continue;
            if (batch[j].done) batch[j].done(batch[j].user, batch[j].id, st, &stats[j]);
            finished.push_back(j);
        }
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->inflight -= (int64_t)finished.size();
            s->info.completed += (int64_t)finished.size();
            if (st != GF_OK && s->first_error == GF_OK) s->first_error = st;
        }
        s->cv_idle.notify_all();
    }
    if (ctx) gf_ctx_destroy(ctx);
}

}  // namespace

extern "C" {

gf_status gf_server_create(int32_t device, int32_t nworkers, int64_t memory_budget, int32_t max_batch, gf_server **out)
{
    if (!out || nworkers <= 0 || nworkers > 16 || memory_budget <= 0 || max_batch <= 0) return GF_E_INVALID;
    gf_server *s = new gf_server();
    s->device = device;
    s->budget = memory_budget;
    s->max_batch = max_batch;
    for (int w = 0; w < nworkers; w++) s->workers.emplace_back(worker_main, s);
    *out = s;
    return GF_OK;
}

gf_status gf_server_submit(gf_server *s, const gf_job *job, gf_server_rows rows, gf_server_done done, void *user,
                           int64_t *request)
{
    if (!s || !job) return GF_E_INVALID;
    std::shared_ptr<OwnedJob> o = own(*job);
    if (!o) return GF_E_INVALID;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return GF_E_STATE;
        Request r;
        r.id = s->next_id++;
        r.owned = std::move(o);
        r.rows = rows;
        r.done = done;
        r.user = user;
        s->queue.push_back(r);
        s->inflight++;
        if (request) *request = r.id;
    }
    s->cv_work.notify_one();
    return GF_OK;
}

gf_status gf_server_drain(gf_server *s)
{
    if (!s) return GF_E_INVALID;
    std::unique_lock<std::mutex> g(s->mu);
    s->cv_idle.wait(g, [&] { return s->inflight == 0; });
    return s->first_error;
}

gf_status gf_server_get_info(gf_server *s, gf_server_info *out)
{
    if (!s || !out) return GF_E_INVALID;
    std::lock_guard<std::mutex> g(s->mu);
    *out = s->info;
    out->queued = (int32_t)s->queue.size();
    out->active = s->active;
    return GF_OK;
}

gf_status gf_server_pause(gf_server *s, int32_t paused)
{
    if (!s) return GF_E_INVALID;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->paused = paused != 0;
    }
    s->cv_work.notify_all();
    return GF_OK;
}

gf_status gf_server_destroy(gf_server *s)
{
    if (!s) return GF_OK;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    gf_status e = s->first_error;
    delete s;
    return e;
}

}  /* extern "C" */
