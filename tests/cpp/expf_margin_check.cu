// Device check of the exp bracket of gfr::Mwc::poisson_small and
// gfr::exceeds_exp_neg (galfast_b200/csrc/gf_rng.h): for EVERY float mu in
// [GF_FASTEXP_MIN_MU, GF_FASTEXP_MAX_MU], the correctly rounded exp(-mu)
// (gfm::expf_) lies strictly inside (__expf(-mu) (1 - margin), __expf(-mu) (1 + margin)),
// the bracket as the device computes it.  Prints the number of floats checked,
// the number outside the bracket and the largest relative difference seen.
#include <cstdio>
#include <cstdint>
#include <cstring>
#include "gf_rng.h"

__global__ void check(uint32_t b0, uint32_t n, unsigned long long *bad, unsigned int *maxrel_bits)
{
    float worst = 0.f;
    unsigned long long nbad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float mu = __uint_as_float(b0 + i);
        if (!(mu >= GF_FASTEXP_MIN_MU && mu <= GF_FASTEXP_MAX_MU)) continue;
        const float ea = __expf(-mu);
        const float lo = ea * (1.0f - GF_FASTEXP_MARGIN), hi = ea * (1.0f + GF_FASTEXP_MARGIN);
        const float ex = gfm::expf_(-mu);
        if (!(ex > lo && ex < hi)) nbad++;
        const float rel = fabsf(ea - ex) / ex;
        worst = rel > worst ? rel : worst;
    }
    if (nbad) atomicAdd(bad, nbad);
    atomicMax(maxrel_bits, __float_as_uint(worst));
}

int main()
{
    unsigned long long *bad = nullptr;
    unsigned int *mx = nullptr;
    if (cudaMalloc(&bad, 8) != cudaSuccess || cudaMalloc(&mx, 4) != cudaSuccess) return 2;
    cudaMemset(bad, 0, 8);
    cudaMemset(mx, 0, 4);
    /* the bit patterns of [0, 10.5] and of (-0.01, -0] (negative mu: an LF extrapolated below 0) */
    const uint32_t pos_end = 0x41280000u + 1;            /* 10.5f */
    const uint32_t neg_end = 0x3c23d70au + 1;            /* 0.01f magnitude */
    unsigned long long checked = (unsigned long long)pos_end + neg_end;
    check<<<148 * 16, 256>>>(0u, pos_end, bad, mx);
    check<<<148 * 16, 256>>>(0x80000000u, neg_end, bad, mx);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    unsigned long long hb = 0;
    unsigned int hm = 0;
    cudaMemcpy(&hb, bad, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&hm, mx, 4, cudaMemcpyDeviceToHost);
    float worst;
    memcpy(&worst, &hm, 4);
    std::printf("%llu %llu %.9g\n", checked, hb, worst);
    return hb != 0;
}
