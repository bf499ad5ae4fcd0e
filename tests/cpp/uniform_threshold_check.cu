// Host check of gfr::uniform_threshold (galfast_b200/csrc/gf_rng.h): for every
// threshold tested, x = threshold passes u <= thr and x + 1 does not, where
// u = 2^-32 * (float)x with round-to-nearest-even conversion (as on the device).
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <random>
#include "gf_rng.h"

static bool passes(uint64_t x, float thr)
{
    const float u = 2.32830643708e-10f * (float)(uint32_t)x;
    return u <= thr;
}

int main()
{
    std::mt19937_64 g(12345);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    long bad = 0, n = 0;
    auto check = [&](float thr) {
        const int64_t X = gfr::uniform_threshold(thr);
        n++;
        if (X < -1 || X > 0xffffffffll) { bad++; return; }
        if (X >= 0 && !passes((uint64_t)X, thr)) bad++;
        if (X < 0xffffffffll && passes((uint64_t)(X + 1), thr)) bad++;
        /* every x up to X passes: spot-check below X */
        if (X >= 0 && X >= 3 && !passes((uint64_t)(X - 3), thr)) bad++;
        /* the cheaper threshold: never above the exact one, its x passes, at most 3.6e-7 below */
        const int64_t Y = gfr::uniform_threshold_lower(thr);
        if (Y > X) bad++;
        if (Y >= 0 && !passes((uint64_t)Y, thr)) bad++;
        if (thr > 1e-6f && thr < 1.f && (double)(X - Y) > 3.6e-7 * (double)X + 2.0) bad++;
    };
    for (int i = 0; i < 2000000; i++) check((float)U(g));
    for (int i = 0; i < 200000; i++) check((float)std::exp(-40.0 * U(g)));
    for (int e = -40; e <= 0; e++) {
        float p = std::ldexp(1.0f, e);
        for (int k = -3; k <= 3; k++) check(std::nextafter(p, k < 0 ? 0.f : 2.f) + 0.f * k);
        check(p);
        check(std::nextafter(p, 0.f));
        check(std::nextafter(p, 2.f));
    }
    const float edge[] = {0.f, -0.f, -1e-30f, -1.f, 1.f, 1.5f, 2.f, 1e-45f, 0.99999994f, 3.9e-3f, 5.960464e-8f};
    for (float t : edge) check(t);
    std::printf("%ld %ld\n", n, bad);
    return bad != 0;
}
