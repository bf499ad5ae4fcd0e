/*
 * gf_server.cpp -- the serving form: continuous batching of catalog requests.
 *
 * Requests are submitted at any time from any thread.  Each worker thread owns
 * a context (its own CUDA stream, streams, workspace) and repeatedly takes the
 * compatible requests waiting at the head of the queue, reserves its share of
 * the device-memory budget and generates them together with
 * gf_catalog_run_multi, whose chunking admits requests by their output-memory
 * estimate (expected stars from the integrate pass).  A request that arrives
 * while a batch is on the GPU is taken by the next worker that frees up, so
 * with two or more workers its work overlaps with the running batch on the
 * device.  Each request's rows are exactly those gf_catalog_run gives it alone,
 * whatever it was batched with.
 *
 * No counterpart in the reference, which generates one catalog per process.
 */
#include "../../include/galfast_b200.h"

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace {

struct Request {
    int64_t id;
    gf_job job;
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
    std::condition_variable cv_work, cv_idle;
    std::deque<Request> queue;
    int64_t next_id = 0;
    int64_t inflight = 0;                /* submitted and not yet done */
    int64_t free_budget = 0;             /* budget not reserved by a running batch */
    bool stop = false;
    gf_status first_error = GF_OK;
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

void worker_main(gf_server *s, int64_t share)
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
        int64_t reserved = 0;
        {
            std::unique_lock<std::mutex> g(s->mu);
            s->cv_work.wait(g, [&] { return s->stop || (!s->queue.empty() && s->free_budget > 0); });
            if (s->queue.empty() && s->stop) break;
            if (s->queue.empty()) continue;
            /* the compatible requests at the head of the queue, in arrival order */
            batch.push_back(s->queue.front());
            s->queue.pop_front();
            while (!s->queue.empty() && (int32_t)batch.size() < s->max_batch && compatible(batch[0].job, s->queue.front().job)) {
                batch.push_back(s->queue.front());
                s->queue.pop_front();
            }
            reserved = std::min(share, s->free_budget);
            s->free_budget -= reserved;
        }
        std::vector<gf_job> jobs;
        for (auto &r : batch) jobs.push_back(r.job);
        std::vector<gf_catalog_stats> stats(batch.size());
        BatchForward f;
        f.reqs = &batch;
        f.ctx = ctx;
        if (ctx) gf_multi_set_memory_budget(ctx, reserved);
        st = gf_catalog_run_multi(ctx, jobs.data(), (int32_t)jobs.size(), forward_rows, &f, stats.data());
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->free_budget += reserved;
        }
        s->cv_work.notify_all();
        for (size_t j = 0; j < batch.size(); j++)
            if (batch[j].done) batch[j].done(batch[j].user, batch[j].id, st, &stats[j]);
        {
            std::lock_guard<std::mutex> g(s->mu);
            s->inflight -= (int64_t)batch.size();
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
    s->free_budget = memory_budget;
    s->max_batch = max_batch;
    const int64_t share = memory_budget / nworkers;
    for (int w = 0; w < nworkers; w++) s->workers.emplace_back(worker_main, s, share);
    *out = s;
    return GF_OK;
}

gf_status gf_server_submit(gf_server *s, const gf_job *job, gf_server_rows rows, gf_server_done done, void *user,
                           int64_t *request)
{
    if (!s || !job) return GF_E_INVALID;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (s->stop) return GF_E_STATE;
        Request r;
        r.id = s->next_id++;
        r.job = *job;
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
