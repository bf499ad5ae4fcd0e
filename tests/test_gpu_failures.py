"""Failure handling on the device path (B200), with failures made on the host:
allocations that fail through the library's allocation hook (no real
out-of-memory condition, no GPU fault), and malformed requests.

* An allocation failure before any rows were delivered is answered by freeing the
  context's cached buffers and running once more, as the reference collects
  garbage and retries a failed allocation (src/common/cux.cpp:189-198).
* Failures that persist return GF_E_OOM; the context stays usable and the next
  call gives the catalog of a clean run.
* Malformed requests are rejected with GF_E_INVALID before any work starts.
"""
import ctypes as C

import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W

pytestmark = pytest.mark.gpu

GF_E_INVALID, GF_E_OOM = -1, -2


def small_requests(lib, n=3):
    reqs = W.config4_requests(n, seed=99)
    ws = []
    for k, r in enumerate(reqs):
        r = dict(r, r=0.5 + 0.2 * k, rmax=19.5 + 0.3 * k)
        ws.append(W.config4_workload(lib, r, capacity=1 << 20))
    return ws


def multi_rows(ctx, ws):
    got = {}
    st = G.run_catalog_multi(ctx, ws, sink=lambda j, m, rows: got.setdefault((j, m), []).append(rows["lb"].copy()))
    return {k: np.concatenate(v, axis=-1) for k, v in got.items()}, st


def plain_rows(ctx, w):
    got = {}
    st = G.run_catalog(ctx, w, sink=lambda m, t, off: got.setdefault(m, []).append(t.as_dict(["lb", "DM"])))
    return {m: np.concatenate([p["lb"] for p in v], axis=-1) for m, v in got.items()}, st


def same(a, b):
    return sorted(a) == sorted(b) and all(np.array_equal(a[k], b[k]) for k in a)


@pytest.fixture
def lib_hook(lib):
    yield lib
    lib.gf_debug_fail_allocations(-1, 0)


def test_one_failed_allocation_is_retried(lib_hook):
    L = lib_hook
    ws = small_requests(L)
    ctx = G.Context(0)
    ref, _ = multi_rows(ctx, ws)
    pref, _ = plain_rows(ctx, ws[0])
    for after in (0, 2, 7, 25):
        ctx.close()
        ctx = G.Context(0)                     # a fresh context allocates its workspace again
        assert L.gf_debug_fail_allocations(after, 1) == 0
        got, _ = multi_rows(ctx, ws)
        assert same(ref, got), after
        L.gf_debug_fail_allocations(-1, 0)
    for after in (0, 3, 12):
        ctx.close()
        ctx = G.Context(0)
        assert L.gf_debug_fail_allocations(after, 1) == 0
        got, _ = plain_rows(ctx, ws[0])
        assert same(pref, got), after
        L.gf_debug_fail_allocations(-1, 0)
    ctx.close()


def test_persistent_allocation_failure_returns_oom_and_context_recovers(lib_hook):
    L = lib_hook
    ws = small_requests(L)
    ctx = G.Context(0)
    ref, _ = multi_rows(ctx, ws)
    pref, _ = plain_rows(ctx, ws[1])
    ctx.close()
    for after in (0, 5, 40):
        ctx = G.Context(0)
        assert L.gf_debug_fail_allocations(after, 0) == 0
        n = len(ws)
        jobs = (G.Job * n)(*[w.job(G.Job) for w in ws])
        st = L.gf_catalog_run_multi(ctx.h, jobs, n, G.MultiCallback(), None, None)
        assert st == GF_E_OOM, (after, st, L.gf_last_error())
        st = L.gf_catalog_run(ctx.h, C.byref(jobs[1]), G.BatchCallback(), None, None)
        assert st == GF_E_OOM, (after, st)
        L.gf_debug_fail_allocations(-1, 0)
        got, _ = multi_rows(ctx, ws)
        assert same(ref, got), after
        got, _ = plain_rows(ctx, ws[1])
        assert same(pref, got), after
        ctx.close()


def test_malformed_requests_are_rejected(lib):
    L = lib
    w = small_requests(L, 1)[0]
    ctx = G.Context(0)

    def run(mutate, multi=False):
        j = w.job(G.Job)
        mutate(j)
        if multi:
            jobs = (G.Job * 2)(w.job(G.Job), j)
            return L.gf_catalog_run_multi(ctx.h, jobs, 2, G.MultiCallback(), None, None)
        return L.gf_catalog_run(ctx.h, C.byref(j), G.BatchCallback(), None, None)

    def setattr_(name, v):
        return lambda j: setattr(j, name, v)

    def sky(name, v):
        return lambda j: setattr(j.sky, name, v)

    bad = [setattr_("nmodels", 0), setattr_("nmodels", 33), setattr_("capacity", 0),
           setattr_("capacity", 256 * 65536 + 1), setattr_("npixels", 0), sky("nthreads", 0),
           sky("nthreads", 70000), sky("dm", 0.0), sky("dm", -0.05), sky("m1", 10.0)]
    for k, mut in enumerate(bad):
        for multi in (False, True):
            st = run(mut, multi)
            assert st == GF_E_INVALID, (k, multi, st, L.gf_last_error())
    # a pixel with an invalid projection index
    pix = (G.PencilBeam * w.npixels).from_buffer_copy(w.pixels)
    pix[0].projIdx = 5
    j = w.job(G.Job)
    j.pixels = C.cast(pix, C.POINTER(G.PencilBeam))
    assert L.gf_catalog_run(ctx.h, C.byref(j), G.BatchCallback(), None, None) == GF_E_INVALID
    # the context still works
    got, _ = plain_rows(ctx, w)
    assert sum(v.shape[-1] for v in got.values()) > 0
    ctx.close()
