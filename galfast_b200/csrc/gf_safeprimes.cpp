// Regeneration of the MWC stream multipliers by primality testing.
// See gf_safeprimes.h for the enumeration that reproduces the reference table
// (src/common/cuda_rng.h:466-497 reads it; data/safeprimes32.txt holds it).
#include "gf_safeprimes.h"
#include <vector>

namespace {

typedef unsigned __int128 u128;

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m) { return (uint64_t)((u128)a * b % m); }

uint64_t powmod(uint64_t b, uint64_t e, uint64_t m)
{
    uint64_t r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = mulmod(r, b, m);
        b = mulmod(b, b, m);
        e >>= 1;
    }
    return r;
}

// Miller-Rabin with the first 12 prime bases is deterministic for n < 3.3e24.
bool miller_rabin(uint64_t n)
{
    static const uint64_t bases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (uint64_t p : bases) {
        if (n % p == 0) return n == p;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (uint64_t a : bases) {
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = false; break; }
        }
        if (comp) return false;
    }
    return true;
}

// small primes for a quick sieve before Miller-Rabin
struct SmallPrimes {
    std::vector<uint32_t> p;
    SmallPrimes()
    {
        const int N = 2000;
        std::vector<bool> c(N, false);
        for (int i = 2; i < N; i++) {
            if (c[i]) continue;
            p.push_back(i);
            for (int j = i * i; j < N; j += i) c[j] = true;
        }
    }
};

bool is_multiplier(uint64_t a, const SmallPrimes &sp)
{
    uint64_t p = (a << 32) - 1;
    uint64_t q = (a << 31) - 1;
    for (uint32_t s : sp.p) {
        if (p % s == 0 && p != s) return false;
        if (q % s == 0 && q != s) return false;
    }
    return miller_rabin(q) && miller_rabin(p);
}

}  // namespace

extern "C" int gf_is_prime_u64(uint64_t n) { return miller_rabin(n) ? 1 : 0; }

extern "C" int gf_safeprimes_generate(uint32_t *out, int n)
{
    if (n < 0 || n > GF_MAX_STREAMS) return 1;
    SmallPrimes sp;
    int k = 0;
    // segment A: increasing from 1
    for (uint64_t a = 1; k < n && k < GF_SAFEPRIME_SEG_A; a++) {
        if (is_multiplier(a, sp)) out[k++] = (uint32_t)a;
    }
    // segment B: decreasing from 2^31 - 1
    int kb = 0;
    for (uint64_t a = 0x7fffffffull; k < n && kb < GF_SAFEPRIME_SEG_B; a--) {
        if (is_multiplier(a, sp)) { out[k++] = (uint32_t)a; kb++; }
    }
    // segment C: decreasing from 2^32 - 1
    for (uint64_t a = 0xffffffffull; k < n; a--) {
        if (is_multiplier(a, sp)) out[k++] = (uint32_t)a;
    }
    return 0;
}
