/*
 * gf_host.h -- host-side setup of the skygen generator and modules.
 */
#pragma once
#include <stdint.h>
#include <string>
#include <vector>
#include "gf_internal.h"

namespace gfh {

/* glibc-compatible drand48 family (POSIX: X_{n+1} = (0x5DEECE66D X_n + 0xB) mod 2^48). */
struct Rand48 {
    uint64_t X = 0x1234ABCD330Eull;
    void srand(uint32_t seed) { X = ((uint64_t)seed << 16) | 0x330Eu; }
    uint64_t next() { X = (0x5DEECE66Dull * X + 0xBull) & ((1ull << 48) - 1); return X; }
    uint32_t lrand() { return (uint32_t)(next() >> 17); }
    double drand() { return (double)next() * 0x1p-48; }
};

/* MT19937 (Matsumoto & Nishimura 1998) with the 2002 initialisation, as GSL's default generator. */
struct MT19937 {
    uint32_t mt[624];
    int mti;
    void seed(uint32_t s);
    uint32_t next();
};

/* Stream states [3][nstreams] from an srand48 seed (cux.cpp:404-414, cuda_rng.h:466-497). */
void seed_streams(uint32_t seed48, int nstreams, const uint32_t *mult, uint32_t *state);

/* The stream multipliers (regenerated once per process, or read from the
 * table written next to the library at build time). */
const std::vector<uint32_t> &multipliers();

/* gsl_interp_linear evaluation with linear extrapolation beyond the end knots. */
double interp_linear(const std::vector<double> &xa, const std::vector<double> &ya, double x);

/* Model setup: the SkyModel of each model (without the device LF pointer)
 * and its resampled LF. */
struct HostModel {
    SkyModel m;
    std::vector<float> lf;
    const float *cube = nullptr;       /* the caller's density grid (GF_MODEL_DENSITY_CUBE), nx*ny*nz floats */
    size_t cube_size = 0;
};
bool setup_models(const gf_skygen_config &cfg, int npixels, const gf_model_config *mc, int nmodels,
                  std::vector<HostModel> &out, std::string &err);

}  // namespace gfh
