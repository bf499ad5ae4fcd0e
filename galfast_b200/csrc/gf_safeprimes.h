/*
 * gf_safeprimes.h -- multipliers of galfast's multiply-with-carry streams.
 *
 * Stream i of the MWC generator uses a multiplier a_i for which
 * p = a_i * 2^32 - 1 and (p - 1)/2 = a_i * 2^31 - 1 are both prime (a "safe
 * prime" p; the MWC with base 2^32 is then a full-period LCG modulo p).  The
 * reference reads its multipliers from a text table, one row per stream
 * (src/common/cuda_rng.h:466-497, rows "a p (p-1)/2").  That table is the
 * concatenation of three complete enumerations, which this file regenerates
 * by primality testing (deterministic Miller-Rabin for 64-bit integers):
 *
 *   rows [0, 17158)      every such a in [1, 2^23 + 447 ...] in increasing order
 *                        (the 17158 smallest multipliers),
 *   rows [17158, 54735)  every such a <= 2^31 - 1 in decreasing order, down to
 *                        the 37577th one,
 *   rows [54735, ...)    every such a <= 2^32 - 1 in decreasing order.
 *
 * Only the first 65536 rows are ever used (the reference's stream count is at
 * most 2^16).  gf_safeprimes_generate() is exact and is checked against the
 * reference's table in the test suite.
 */
#pragma once
#include <stdint.h>

#define GF_SAFEPRIME_SEG_A 17158
#define GF_SAFEPRIME_SEG_B 37577
#define GF_MAX_STREAMS 65536

#ifdef __cplusplus
extern "C" {
#endif
/* Fill out[0..n) (n <= GF_MAX_STREAMS) with the stream multipliers.  Returns 0 on success. */
int gf_safeprimes_generate(uint32_t *out, int n);
/* Deterministic primality test for 64-bit integers. */
int gf_is_prime_u64(uint64_t n);
#ifdef __cplusplus
}
#endif
