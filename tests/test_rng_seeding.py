"""Random-number streams (CPU only).

* the multiply-with-carry step (cuda_rng.h:439-463) against exact integer
  arithmetic, for the state of the reference's test_mwc_rng (tests.cpp:999-1009);
* the stream seeding of the product (its own drand48 restatement) against the
  oracle, which calls glibc's srand48/drand48/lrand48 as the reference does
  (cuda_rng.h:466-497), for all 65536 streams;
* the MWC as a Lehmer generator modulo the safe prime (the jump-ahead the GPU
  crawl relies on);
* MT19937 (the GSL default generator behind the reference's seed) against
  numpy's legacy seeding.
"""
import ctypes as C

import numpy as np
import pytest

import galfast_b200 as G
from oracle import oracle as O


def mwc_python(a, c, x, n):
    out = []
    for _ in range(n):
        t = a * x + c
        c, x = t >> 32, t & 0xFFFFFFFF
        out.append(np.float32(np.float32(2.32830643708e-10) * np.float32(x)))
    return out, c, x


def test_mwc_uniforms_reference_state():
    a, c, x = C.c_uint32(8834973), C.c_uint32(42), C.c_uint32(332)
    out = np.zeros(50, dtype=np.float32)
    O.load("p").or_mwc_uniforms(C.byref(a), C.byref(c), C.byref(x), 50, out.ctypes.data)
    ref, rc, rx = mwc_python(8834973, 42, 332, 50)
    assert np.array_equal(out, np.array(ref, dtype=np.float32))
    assert (c.value, x.value) == (rc, rx)


def test_mwc_scale_is_exactly_two_to_minus_32():
    assert float(np.float32(2.32830643708e-10)) == 2.0 ** -32


def test_seeding_matches_glibc(multipliers, lib):
    for seed in (42, 6283740, 0xFFFFFF):
        ora = O.seed_streams(seed, multipliers)
        mine = np.zeros(3 * 65536, dtype=np.uint32)
        lib.gf_rng_seed_host(seed, 65536, mine.ctypes.data_as(C.POINTER(C.c_uint32)))
        assert np.array_equal(ora, mine)
        # streams above 2^31 multipliers get the x86 out-of-range conversion (INT_MIN) for half their carries
        c = mine[65536:2 * 65536]
        assert (c[60000:] == 0x80000000).mean() > 0.3


def test_lehmer_jump_ahead(multipliers):
    rng = np.random.default_rng(7)
    for s in rng.integers(0, 65536, size=20):
        a = int(multipliers[s])
        p = a * 2 ** 32 - 1
        c0 = int(rng.integers(0, a))
        x0 = int(rng.integers(0, 2 ** 32))
        c, x = c0, x0
        for _ in range(37):
            t = a * x + c
            c, x = t >> 32, t & 0xFFFFFFFF
        v = (c0 << 32) | x0
        assert (pow(a, 37, p) * v) % p == (c << 32) | x


def test_mt19937_matches_numpy_legacy(lib):
    for seed in (5489, 42, 1):
        out = (C.c_uint32 * 10)()
        lib.gf_mt19937_outputs(seed, 10, out)
        ref = np.random.RandomState(seed).randint(0, 2 ** 32, size=10, dtype=np.uint64)
        assert list(out) == [int(v) for v in ref]
    out = (C.c_uint32 * 1)()
    lib.gf_mt19937_outputs(5489, 1, out)
    assert out[0] == 3499211612


def test_seed48_from_cli_seed(lib):
    # (uint32)((float)(mt19937(seed) / 2^32) * 2^24), cux.cpp:409 with gpu.h:362-382
    for seed in (1, 42, 12345):
        u = np.random.RandomState(seed).randint(0, 2 ** 32, dtype=np.uint64) / 4294967296.0
        assert lib.gf_rng_seed48_from_cli_seed(seed) == int(np.float32(np.float32(u) * np.float32(2 ** 24)))


def test_poisson_and_gaussian_statistics():
    """The restated GSL samplers (cuda_rng.h:165-182, 344-376) reproduce their distributions."""
    L = O.load("p")
    a, c, x = C.c_uint32(4294967118), C.c_uint32(123456), C.c_uint32(987654321)
    for mu in (0.01, 0.7, 4.0, 25.0, 300.0):
        n = 20000
        mus = np.full(n, mu, dtype=np.float32)
        out = np.zeros(n, dtype=np.uint32)
        L.or_mwc_poisson(C.byref(a), C.byref(c), C.byref(x), mus.ctypes.data, n, out.ctypes.data)
        assert abs(out.mean() - mu) < 5 * np.sqrt(mu / n) + 1e-3
        assert abs(out.var() - mu) < 0.1 * mu + 0.01
    g = np.zeros(50000, dtype=np.float32)
    L.or_mwc_gaussian(C.byref(a), C.byref(c), C.byref(x), C.c_float(2.0), len(g), g.ctypes.data)
    assert abs(g.mean()) < 0.05 and abs(g.std() - 2.0) < 0.03
