"""Properties of the CPU oracle itself (CPU only, small workloads).

* the portable-math flavour agrees with the libm flavour (the reference's own
  CPU build) on expected counts to 1e-6 and on the drawn stars up to rare
  ulp-level differences;
* batching is transparent when no module consumes the streams between batches:
  the stars of a many-batch run are exactly the stars of a single-batch run;
* with Bond2010 consuming the same streams between batches the catalog depends
  on the batch size, as in the reference (skyconfig_impl.h:445-534);
* the integrate pass is independent of the crawl's stream count.
"""
import ctypes as C
import math

import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W, _abi as A
from oracle import oracle as O


def patch(lib, half_deg=1.0, **kw):
    half = half_deg * math.pi / 180
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    return W.build_workload(lib, foot=foot, dx_deg=0.25, m0=15.0, m1=kw.pop("m1", 20.0), **kw)


def collect(w, mult, flavour="p"):
    rows = []
    O.run_catalog(w, mult, flavour=flavour, sink=lambda m, t, off: rows.append(t.as_dict(G.SKYGEN_COLUMNS)))
    return rows


def star_set(rows, exact_lb=True):
    """(comp, l, b, DM, M) of every star; without exact_lb, l and b are rounded to 1e-9 deg
    (the two math flavours differ in the last bits of asin/atan2)."""
    keys = []
    for r in rows:
        for k in range(len(r["DM"])):
            l, b = r["lb"][0][k], r["lb"][1][k]
            if not exact_lb:
                l, b = round(l, 9), round(b, 9)
            keys.append((r["comp"][k], l, b, r["DM"][k], r["absmag"][k]))
    return sorted(keys)


def test_flavours_agree(lib, multipliers):
    w = patch(lib, with_modules=False)
    p, l = O.OracleSkygen(w, "p"), O.OracleSkygen(w, "l")
    for m in range(3):
        ep, _, _ = p.integrate_counts(m)
        el, _, _ = l.integrate_counts(m)
        assert ep == pytest.approx(el, rel=1e-6)
    sp = star_set(collect(w, multipliers, "p"), exact_lb=False)
    sl = star_set(collect(w, multipliers, "l"), exact_lb=False)
    assert abs(len(sp) - len(sl)) <= max(3, 1e-3 * len(sp))
    common = len(set(sp) & set(sl))
    assert common >= 0.97 * len(sp)


def test_batching_is_transparent_without_stream_consumers(lib, multipliers):
    w1 = patch(lib, with_modules=False, capacity=1 << 16)
    w2 = patch(lib, with_modules=False, capacity=997)
    r1, r2 = collect(w1, multipliers), collect(w2, multipliers)
    assert len(r1) == 3 and len(r2) > len(r1)
    assert star_set(r1) == star_set(r2)


def test_batching_changes_the_catalog_when_bond2010_shares_the_streams(lib, multipliers):
    """With two streams each holding ~1000 stars, a 1024-row batch stops stream 0 part-way;
    Bond2010 then draws from streams 0-3 before the crawl resumes, so the rest differs."""
    w1 = patch(lib, half_deg=2.0, nthreads=2, capacity=1 << 16)
    w2 = patch(lib, half_deg=2.0, nthreads=2, capacity=1024)
    r1, r2 = collect(w1, multipliers), collect(w2, multipliers)
    s1, s2 = set(star_set(r1)), set(star_set(r2))
    assert len(r2) > len(r1)
    assert s1 != s2
    assert len(s1 & s2) > 500        # the stars before the first batch boundary agree


def test_expected_counts_do_not_depend_on_the_stream_count(lib):
    e = []
    for nthreads in (7680, 333, 64):
        w = patch(lib, nthreads=nthreads, with_modules=False)
        sk = O.OracleSkygen(w)
        e.append([sk.integrate_counts(m)[0] for m in range(3)])
    np.testing.assert_allclose(e[0], e[1], rtol=1e-12)
    np.testing.assert_allclose(e[0], e[2], rtol=1e-12)


def test_draw_count_is_consistent_with_expectation(lib, multipliers):
    w = patch(lib, half_deg=2.0, with_modules=False)
    sk = O.OracleSkygen(w)
    exp = sum(sk.integrate_counts(m)[0] for m in range(3))
    st, _ = O.run_catalog(w, multipliers)
    gen = sum(st["generated"].values())
    assert abs(gen - exp) < 5 * math.sqrt(exp)


@pytest.mark.parametrize("nthreads,capacity", [(7680, 1 << 18), (7680, 1500), (97, 700), (3, 400)])
def test_parallel_oracle_equals_sequential(lib, multipliers, nthreads, capacity):
    """The oracle on several host threads (streams crawled in parallel, then the
    stream that crosses a batch boundary and the later ones run again; parallel
    sort, permutation and modules) gives the catalog, batch boundaries and stream
    states of the reference's one-thread-after-another order, including batches
    that stop part-way through a stream while Bond2010 shares the streams."""
    w = patch(lib, half_deg=1.5, nthreads=nthreads, capacity=capacity)
    runs = []
    for threads in (1, 4):
        rows = []
        st, state = O.run_catalog(w, multipliers, threads=threads,
                                  sink=lambda m, t, off: rows.append((m, off, t.as_dict())))
        runs.append((rows, st, state))
    (r1, s1, st1), (r4, s4, st4) = runs
    assert len(r1) == len(r4) and (capacity > 1 << 17 or len(r1) > 3)
    for (m1, o1, a), (m4, o4, b) in zip(r1, r4):
        assert (m1, o1) == (m4, o4)
        for c in a:
            np.testing.assert_array_equal(a[c], b[c], err_msg=c)
    assert s1["generated"] == s4["generated"] and s1["stored"] == s4["stored"]
    assert np.array_equal(st1, st4)


def test_parallel_seeding_equals_glibc(multipliers):
    """Stream seeding on several host threads (the drand48 recurrence with
    jump-ahead) equals glibc's srand48/drand48/lrand48 sequence."""
    L = O.load("p")
    try:
        for seed in (0, 42, 0xFFFFFFFF):
            L.or_set_threads(1)
            a = O.seed_streams(seed, multipliers)
            L.or_set_threads(5)
            b = O.seed_streams(seed, multipliers)
            assert np.array_equal(a, b), seed
    finally:
        L.or_set_threads(1)


def test_bulge_and_broken_power_law_setup_agrees_with_oracle(lib):
    """The library's host model setup (the per-piece factors of a broken power law,
    the LC bulge's LF scaled by f) equals the oracle's, and the broken power law's
    expected counts change smoothly across its break radius."""
    from galfast_b200 import _abi as A
    w = patch(lib, with_modules=False)
    h = w.models[2]
    h.type = A.GF_MODEL_BROKEN_POWER_LAW
    h.nbreaks = 2
    h.n_brk[0], h.n_brk[1], h.n_brk[2] = -2.5, -3.0, -4.0
    h.rbreak[0], h.rbreak[1] = 15000.0, 40000.0
    b = w.models[1]
    b.type = A.GF_MODEL_LCBULGE
    b.f, b.l, b.n, b.ba, b.ca = 3.0, 700.0, 2.0, 0.6, 0.4
    info = (G.ModelInfo * 3)()
    lf = np.zeros((3, 1024), dtype=np.float32)
    marr = (G.ModelConfig * 3)(*w.models)
    assert lib.gf_skygen_setup_host(C.byref(w.sky), w.npixels, marr, 3, info, lf.ctypes.data_as(C.POINTER(C.c_float))) == 0
    osk = O.OracleSkygen(w)
    for m in range(3):
        oi = osk.info(m)
        assert info[m].f == oi.f and info[m].nm == oi.nm and info[m].M1 == oi.M1, m
        np.testing.assert_array_equal(lf[m, :oi.lf_n], osk.lf(m))
    plain = O.OracleSkygen(patch(lib, with_modules=False))
    np.testing.assert_allclose(osk.lf(1), 3.0 * plain.lf(1).astype(np.float32), rtol=1e-7)
