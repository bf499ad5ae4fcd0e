/*
 * gf_ctx.h -- the library context and the host-side error and allocation
 * helpers shared by the C ABI files (gf_api.cu, gf_multi.cu).
 */
#pragma once
#include <chrono>
#include <cuda_runtime.h>
#include <string>
#include <utility>
#include <vector>
#include "gf_launch.h"

struct MultiWS;

namespace gfa {

/* record the message returned by gf_last_error() and pass the status through */
gf_status fail(gf_status s, const std::string &msg);

template <typename T>
void dev_free(T *&p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

}  // namespace gfa

#define GF_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            return gfa::fail(e_ == cudaErrorMemoryAllocation ? GF_E_OOM : GF_E_CUDA,         \
                             std::string(#call) + ": " + cudaGetErrorString(e_));             \
        }                                                                                    \
    } while (0)

#define GF_TRY(call)                         \
    do {                                     \
        gf_status s_ = (call);               \
        if (s_ != GF_OK) return s_;          \
    } while (0)

namespace gfa {
/* Every device allocation of the library goes through here: cudaMalloc, or the
 * out-of-memory error that gf_debug_fail_allocations arranges, without calling it. */
cudaError_t device_malloc(void **p, size_t bytes);
/* gf_debug_fail_allocations */
void set_alloc_failures(long long after, long long count);

template <typename T>
gf_status dev_alloc(T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) return GF_OK;
    GF_CUDA(device_malloc((void **)p, n * sizeof(T)));
    return GF_OK;
}
}  // namespace gfa

struct gf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t *d_rng = nullptr;           /* persistent streams [3][rng_nstreams] */
    int32_t rng_nstreams = 0;
    uint32_t *d_mult = nullptr;
    JumpTables jt = {nullptr, nullptr};
    unsigned long long *d_counters = nullptr;   /* [0] record count, [1] visible count, [2] error flag */
    unsigned long long *h_counters = nullptr;   /* pinned */
    cudaEvent_t ev[16] = {};
    /* phase profiler */
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending;
    double prof_ms[GF_PROF_NPHASES] = {};
    int64_t prof_n[GF_PROF_NPHASES] = {};
    int64_t multi_budget = 0;            /* device bytes per multi-request chunk (0: 60% of free memory) */
    MultiWS *multi_ws = nullptr;         /* buffers of gf_catalog_run_multi kept between calls */
    gf_table plain_table = {};           /* output table of gf_catalog_run, kept for the next call of the same shape */
    void *rec_cache = nullptr;           /* star-record and placement buffers of a finished generator, for the next one */
    int32_t draw_wpc[3] = {0, 0, 0};      /* warps per CTA of the batched draw, by model kind (0: not tuned yet) */
    uint32_t host_cols = GF_COL_ALL;     /* columns gf_catalog_run_multi_host copies to host memory */
    double admit_sigma = 8.0;            /* batched if expected + admit_sigma sqrt(expected) + 1024 < capacity */
};

struct gf_photometry {
    gfk::PhotTables tab;
    float *d_colors = nullptr;
    uint8_t *d_eflags = nullptr;
};

struct gf_photoerr {
    gfk::PerrTables tab;
    double *d_mag = nullptr, *d_sigma = nullptr;
    int32_t *d_guide = nullptr;
};

namespace gfa {

/* Admission of a multi-request call (the serving workers' hook).  After the
 * integrate pass, admit() receives need[k], the device memory (bytes) of the
 * k-th batched request in submission order, returns how many of them, from the
 * first, to generate in this call (at least one) and sets *budget, the memory the
 * call's chunks may use.  The requests after them are not generated
 * (deferred[j] = 1) and receive no rows; requests that take the plain path are
 * always generated. */
struct Admission {
    int32_t (*admit)(void *user, const double *need, int32_t n, int64_t *budget) = nullptr;
    void *user = nullptr;
    std::vector<char> deferred;
};
gf_status catalog_run_multi_admitted(gf_ctx *ctx, const gf_job *jobs, int32_t njobs, gf_multi_callback cb, void *user,
                                     gf_catalog_stats *stats, Admission *adm);

gf_status check_ctx(gf_ctx *ctx);
/* zero the module columns (FeH, vcyl, mags, photoflags, obsmags, pm, radec) of rows
 * [0, n): rows a module skips (hidden stars) read zero whatever the table held before */
gf_status zero_module_rows(gf_ctx *ctx, const gf_table *t, int64_t n);
void free_multi_ws(gf_ctx *ctx);
/* free the buffers a context keeps between calls (output table, multi-request workspace) */
void release_caches(gf_ctx *ctx);
/* free the cached generator buffers (rec_cache) */
void free_rec_cache(gf_ctx *ctx);
/* gf_catalog_run for a request run inside a multi-request call: an out-of-memory
 * failure before its first batch frees only the plain path's output table before the
 * retry, so the multi-request workspace the caller is using stays in place */
gf_status catalog_run_in_multi(gf_ctx *ctx, const gf_job *job, gf_batch_callback cb, void *user, gf_catalog_stats *stats);
/* multipliers and jump tables of all 65536 streams on the context's device */
gf_status ensure_multipliers(gf_ctx *ctx);

inline cudaEvent_t prof_event(gf_ctx *c)
{
    if (!c->ev_pool.empty()) { cudaEvent_t e = c->ev_pool.back(); c->ev_pool.pop_back(); return e; }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

/* brackets the kernels of one phase with events when profiling is enabled */
struct ProfScope {
    gf_ctx *c; int kind; cudaEvent_t a = nullptr;
    ProfScope(gf_ctx *c_, int k) : c(c_), kind(k)
    {
        if (c->prof) { a = prof_event(c); cudaEventRecord(a, c->stream); }
    }
    ~ProfScope()
    {
        if (!a) return;
        cudaEvent_t b = prof_event(c);
        cudaEventRecord(b, c->stream);
        c->prof_pending.push_back({kind, {a, b}});
    }
};

/* host wall time of a phase, added to the context's profile when it is enabled */
struct HostScope {
    gf_ctx *c; int kind; bool on;
    std::chrono::steady_clock::time_point t0;
    HostScope(gf_ctx *c_, int k) : c(c_), kind(k), on(c_->prof), t0(std::chrono::steady_clock::now()) {}
    void stop()
    {
        if (!on) return;
        on = false;
        c->prof_ms[kind] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        c->prof_n[kind] += 1;
    }
    ~HostScope() { stop(); }
};

}  // namespace gfa
