"""gf_server (B200): requests submitted while others are on the GPU are batched
with whatever is waiting, on two workers whose batches overlap on the device, and
each request's catalog is still exactly the one gf_catalog_run gives it alone.
Requests mix caps and galactic lon/lat rectangles, ugriz and ugrizy photometry."""
import time

import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W

pytestmark = pytest.mark.gpu

SKY = ["lb", "projIdx", "projXY", "DM", "absmag", "XYZ", "comp", "Am", "AmInf", "hidden"]
MODULE = ["FeH", "vcyl", "mags", "photoflags", "obsmags", "pm", "radec"]


def alone(ctx, w):
    per_model = {}
    G.run_catalog(ctx, w, sink=lambda m, t, off: per_model.setdefault(m, []).append(t.as_dict()))
    return {m: {k: np.concatenate([p[k] for p in parts], axis=-1) for k in parts[0]} for m, parts in per_model.items()}


def test_served_requests_equal_standalone(lib):
    reqs = W.config5_requests(9, rate=20.0, seed=5, area=(1.0, 6.0), rmax=(20.0, 21.5))
    ws = W.config5_workloads(lib, reqs, capacity=1 << 20)
    assert {r["kind"] for r in reqs} == {"cap", "rect"} and {r["lsst"] for r in reqs} == {True, False}
    srv = G.Server(0, workers=2, memory_budget=8 << 30, max_batch=3, keep_rows=True)
    t0 = time.perf_counter()
    ids = []
    for r, w in zip(reqs, ws):
        while time.perf_counter() - t0 < r["t"]:
            time.sleep(0.002)
        ids.append(srv.submit(w))
    srv.drain()
    ctx = G.Context(0)
    for rid, w in zip(ids, ws):
        assert srv.status[rid] == 0, rid
        ref = alone(ctx, w)
        got = srv.rows.get(rid, {})
        assert sorted(ref) == sorted(got), rid
        for m in ref:
            b = {k: np.concatenate([p[k] for p in got[m]], axis=-1) for k in got[m][0]}
            a = ref[m]
            for c in SKY:
                np.testing.assert_array_equal(a[c], b[c], err_msg="%s request %d model %d" % (c, rid, m))
            vis = a["hidden"] == 0
            for c in MODULE:
                x, y = a[c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]
                np.testing.assert_array_equal(x[..., vis], y[..., vis], err_msg="%s request %d model %d" % (c, rid, m))
    srv.close()
    ctx.close()


def _served(srv, ctx, ws, ids):
    """every request done, its rows equal to its standalone catalog"""
    for rid, w in zip(ids, ws):
        assert srv.status[rid] == 0, rid
        ref = alone(ctx, w)
        got = srv.rows.get(rid, {})
        assert sorted(ref) == sorted(got), rid
        for m in ref:
            b = {k: np.concatenate([p[k] for p in got[m]], axis=-1) for k in got[m][0]}
            for c in SKY:
                np.testing.assert_array_equal(ref[m][c], b[c], err_msg="%s request %d model %d" % (c, rid, m))


def _need_alone(lib, w):
    """the memory reservation of a request served alone (its need at admission)"""
    srv = G.Server(0, workers=1, memory_budget=64 << 30, max_batch=4)
    rid = srv.submit(w)
    srv.drain()
    info = srv.info()
    st = srv.stats[rid]
    srv.close()
    return info, st


def test_reservation_follows_the_requests_estimate(lib):
    """A batch reserves its requests' need (expected stars of the largest model plus
    8 sigma, about 370 bytes per star, and the slot densities of its pixels), not a
    fixed share of the budget."""
    w = W.config4_workload(lib, dict(l=40.0, b=35.0, r=0.8, rmax=20.0, h=300.0, q=0.65, seed48=77), capacity=1 << 20)
    info, st = _need_alone(lib, w)
    assert info["runs"] == 1 and info["completed"] == 1 and info["deferred"] == 0 and info["peak_running"] == 1
    e = max(st.expected[i] for i in range(len(w.models)))
    lo = (e + 8.0 * e ** 0.5 + 1024.0) * 368.0
    assert lo <= info["peak_reserved"] <= lo + 4.0 * w.npixels * (400 * 400 + 2) + 1
    assert info["peak_reserved"] < (64 << 30) // 8


def test_admission_defers_what_does_not_fit_and_late_requests_join(lib):
    """One worker, a budget of 2.5 times one request's need.  Four equal requests
    are taken as one batch; admission generates two and returns the others to the
    queue.  A small request submitted while that batch runs joins them: the second
    batch generates all three.  The caller's job memory is overwritten right after
    each submit (the server copies it), and every catalog still equals its
    standalone run."""
    import time
    base = dict(l=120.0, b=-40.0, r=1.0, rmax=20.5, h=300.0, q=0.65)
    small = dict(l=200.0, b=60.0, r=0.3, rmax=19.0, h=280.0, q=0.6, seed48=991)
    params = [dict(base, seed48=1000 + k) for k in range(4)] + [small]
    ws_ref = [W.config4_workload(lib, r, capacity=1 << 20) for r in params]
    need_a = _need_alone(lib, ws_ref[0])[0]["peak_reserved"]
    need_b = _need_alone(lib, ws_ref[4])[0]["peak_reserved"]
    assert 0 < need_b < 0.5 * need_a
    ws_sub = [W.config4_workload(lib, r, capacity=1 << 20) for r in params]

    def clobber(w):
        # the job's memory is the caller's again: overwrite the beams and the LF values
        w.pixels[:] = b"\xff" * len(w.pixels)
        w.ammin[:] = np.nan
        for mdl in w.models:
            if mdl.lf_n and mdl.lf_phi:
                for q in range(mdl.lf_n):
                    mdl.lf_phi[q] = -1.0

    srv = G.Server(0, workers=1, memory_budget=int(2.5 * need_a), max_batch=16, keep_rows=True)
    srv.pause()
    ids = []
    for w in ws_sub[:4]:
        ids.append(srv.submit(w))
        clobber(w)
    srv.pause(False)
    t0 = time.perf_counter()
    while True:                      # the worker has taken the four requests
        i = srv.info()
        if i["queued"] == 0 and i["active"] == 1:
            break
        assert time.perf_counter() - t0 < 60
        time.sleep(0.0005)
    ids.append(srv.submit(ws_sub[4]))
    clobber(ws_sub[4])
    srv.drain()
    info = srv.info()
    assert info["completed"] == 5
    assert info["runs"] == 2, info
    assert info["deferred"] == 2, info
    assert info["peak_reserved"] <= int(2.5 * need_a) + 1
    ctx = G.Context(0)
    _served(srv, ctx, ws_ref, ids)
    srv.close()
    ctx.close()
