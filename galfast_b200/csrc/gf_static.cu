/*
 * gf_static.cu -- expected star counts of one density model without any
 * device allocation.
 *
 * Who needs it: some hosts own all of the GPU's memory themselves -- a
 * pipeline framework that reserves one arena up front and hands out slices
 * of it, or a process that must not let a library call cudaMalloc/cudaFree
 * while it runs (those calls synchronise the device and can fail once the
 * memory is committed).  Such a caller passes its own device buffers for the
 * inputs and the result; the scratch the integrate pass needs (one pair of
 * partial sums per crawl stream, the luminosity function and the distance
 * table) lives in the fixed array below instead.
 *
 * The array is a file-scope __device__ object: every GPU that loads this
 * library holds its 1.3 MB until the process exits.  Its device address is
 * looked up once per device (devices 0-63), on the first call made with that
 * device current, with cudaGetSymbolAddress.  Every call copies the LF from
 * host memory and synchronises its stream before it returns, also when it
 * fails, so it must not be called while its stream is being captured.  All
 * calls share the array and it keeps the last call's contents (the partial
 * sums are cleared at the start of every call), so calls that overlap on the
 * GPU -- from two host threads, or on two streams -- race; calls made one
 * after another from one thread do not overlap.
 */
#include "gf_launch.h"
#include "gf_host.h"

#include <mutex>
#include <string>
#include <vector>

namespace {

/* limits of the fixed scratch */
constexpr int kMaxStreams = 65536;     /* crawl streams (the reference's maximum) */
constexpr int kMaxLF = 1024;           /* luminosity-function samples */
constexpr int kMaxBins = 65536;        /* nm * nM magnitude bins of one pixel */

struct StaticScratch {
    double counts[kMaxStreams];        /* per-stream expected counts */
    double covered[kMaxStreams];       /* ... weighted by the covered fraction */
    float lf[kMaxLF];
    float dtab[kMaxBins];              /* D[im][iM] */
};

static __device__ __align__(256) StaticScratch g_static_scratch;

std::mutex g_addr_mutex;
StaticScratch *g_addr[64] = {};        /* device address of the scratch, per device */

/* the partial sums in stream order, as skygenHost<T>::download adds them (skyconfig_impl.h:148-154) */
__global__ void static_reduce(const StaticScratch *s, int n, double *out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double e = 0, ec = 0;
    for (int i = 0; i < n; i++) { e += s->counts[i]; ec += s->covered[i]; }
    out[0] = e;
    out[1] = ec;
}

gf_status sfail(gf_status st, const std::string &m)
{
    gfk::set_last_error(m);
    return st;
}

}  // namespace

extern "C" gf_status gf_skygen_integrate_static(const gf_skygen_config *cfg, const gf_pencil_beam *d_pixels, int32_t npixels,
                                                const float *d_beam_ammin, const gf_extinction *ext,
                                                const gf_model_config *model, double *d_result, void *stream_ptr)
{
    if (!cfg || !d_pixels || npixels <= 0 || !model || !d_result) return sfail(GF_E_INVALID, "invalid arguments");
    if (cfg->nthreads <= 0 || cfg->nthreads > kMaxStreams)
        return sfail(GF_E_INVALID, "nthreads above the static scratch limit of 65536 streams");
    std::vector<gfh::HostModel> hms;
    std::string err;
    if (!gfh::setup_models(*cfg, npixels, model, 1, hms, err)) return sfail(GF_E_INVALID, err);
    const SkyModel &hm = hms[0].m;
    if (ext && ext->kind == GF_EXT_MAPS)
        return sfail(GF_E_UNSUPPORTED, "3-D extinction maps need device copies (use gf_skygen_integrate)");
    if (hm.type == GF_MODEL_DENSITY_CUBE)
        return sfail(GF_E_UNSUPPORTED, "the density cube needs a device copy of its grid (use gf_skygen_integrate)");
    if (hm.lf_n > kMaxLF) return sfail(GF_E_INVALID, "luminosity function above the static scratch limit of 1024 samples");
    if ((long long)hm.nm * hm.nM > kMaxBins)
        return sfail(GF_E_INVALID, "nm*nM above the static scratch limit of 65536 bins per pixel");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return sfail(GF_E_CUDA, "no current CUDA device");
    if (dev >= 64) return sfail(GF_E_UNSUPPORTED, "device index above the static entry point's limit of 64 devices");
    StaticScratch *S = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_addr_mutex);
        if (!g_addr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
            if (e != cudaSuccess || !p) return sfail(GF_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_addr[dev] = (StaticScratch *)p;
        }
        S = g_addr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream_ptr;
    cudaError_t e = cudaMemcpyAsync(S->lf, hms[0].lf.data(), sizeof(float) * (size_t)hm.lf_n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->counts, 0, sizeof(double) * (size_t)cfg->nthreads, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->covered, 0, sizeof(double) * (size_t)cfg->nthreads, st);
    if (e == cudaSuccess) e = gfk::launch_dtab(hm, S->dtab, st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);     /* nothing of this call stays in flight on the shared array */
        return sfail(GF_E_CUDA, std::string("setup: ") + cudaGetErrorString(e));
    }

    gfk::LaunchCrawl L;
    memset(&L, 0, sizeof(L));
    L.m = hm;
    L.m.lf = S->lf;
    L.g.pixels = d_pixels;
    L.g.npixels = npixels;
    L.g.ammin = d_beam_ammin;
    L.g.ext_kind = ext ? ext->kind : GF_EXT_NONE;
    L.g.A0 = ext ? ext->A0 : 0.f;
    L.g.proj[0] = cfg->proj[0];
    L.g.proj[1] = cfg->proj[1];
    L.stream_begin = 0;
    L.stream_end = cfg->nthreads;
    L.counts = S->counts;
    L.countsCovered = S->covered;
    L.Dtab = S->dtab;
    const long long kmax = (long long)hm.nm * hm.nM;
    if (kmax % GF_BLOCK == 0) {
        e = gfk::launch_crawl(L, 0, st);
    } else {
        /* pixel blocks of 2^21 / nthreads pixels (skyconfig_impl.h:344-387) */
        const int PIXBLOCK = 1024 * 1024 * 2 / cfg->nthreads;
        for (int p0 = 0; p0 < npixels && e == cudaSuccess; p0 += PIXBLOCK) {
            L.g.pixels = d_pixels + p0;
            L.g.npixels = std::min(PIXBLOCK, npixels - p0);
            L.pix_base = p0;
            e = gfk::launch_crawl(L, 0, st);
        }
    }
    if (e == cudaSuccess) {
        static_reduce<<<1, 32, 0, st>>>(S, cfg->nthreads, d_result);
        gfk::count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        return sfail(GF_E_CUDA, std::string("integrate: ") + cudaGetErrorString(e));
    }
    return GF_OK;
}
