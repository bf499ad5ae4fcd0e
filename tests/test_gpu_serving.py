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
