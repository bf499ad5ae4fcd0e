"""gf_catalog_run_multi against gf_catalog_run (B200): every request's catalog
is the one it gets alone, bit for bit, whether it was generated together with
the others or (capacity too small for one batch) ran alone inside the multi
call.  Requests differ in footprint, depth, model parameters, seed, capacity
and photometric system."""
import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W

pytestmark = pytest.mark.gpu

SKY = ["lb", "projIdx", "projXY", "DM", "absmag", "XYZ", "comp", "Am", "AmInf", "hidden"]
MODULE = ["FeH", "vcyl", "mags", "photoflags", "obsmags", "pm", "radec"]


def requests(lib, n=7):
    reqs = W.config4_requests(n, seed=777)
    ws = []
    for k, r in enumerate(reqs):
        r = dict(r)
        r["r"] = 0.4 + 0.25 * k            # 0.4 .. 1.9 deg caps
        r["rmax"] = 19.0 + 0.4 * k
        kw = {}
        if k % 3 == 2:
            kw = dict(nbands=6, m5=W.LSST_M5)
        w = W.config4_workload(lib, r, capacity=1 << 20, **kw)
        ws.append(w)
    # one request whose stars need several batches: it runs alone inside the multi call
    ws[1].capacity = 400
    # distance limits: anchors outside [dmin, dmax) cut their bins
    if n > 3:
        ws[3].sky.dmin = 400.0
        ws[3].sky.dmax = 12000.0
    return ws


def catalog_alone(ctx, w):
    per_model = {}

    def sink(model, t, off):
        d = t.as_dict()
        per_model.setdefault(model, []).append(d)
    st = G.run_catalog(ctx, w, sink=sink)
    out = {}
    for m, parts in per_model.items():
        out[m] = {k: np.concatenate([p[k] for p in parts], axis=-1) for k in parts[0]}
    return out, st


def test_multi_request_rows_equal_standalone(lib):
    ws = requests(lib)
    ctx = G.Context(0)
    got = {}

    def sink(j, model, rows):
        got.setdefault(j, {}).setdefault(model, []).append(rows)
    stats = G.run_catalog_multi(ctx, ws, sink=sink)
    assert len(got) == len(ws)
    for j, w in enumerate(ws):
        ref, st = catalog_alone(ctx, w)
        assert sorted(ref) == sorted(got[j]), j
        for m in ref:
            parts = got[j][m]
            mine = {k: np.concatenate([p[k] for p in parts], axis=-1) for k in parts[0]}
            a, b = ref[m], mine
            assert a["DM"].shape == b["DM"].shape, (j, m)
            for c in SKY:
                np.testing.assert_array_equal(a[c], b[c], err_msg="%s request %d model %d" % (c, j, m))
            vis = a["hidden"] == 0
            for c in MODULE:
                if c not in a or a[c].size == 0:
                    continue
                x, y = a[c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]             # the shared table holds the most bands of any request
                np.testing.assert_array_equal(x[..., vis], y[..., vis], err_msg="%s request %d model %d" % (c, j, m))
        for i in range(3):
            # batched requests integrate pixel by pixel, the standalone run stream by
            # stream: the same bins and float values, FP64 sums in another order
            assert stats[j].expected[i] == pytest.approx(st.expected[i], rel=1e-12)
            assert stats[j].expected_covered[i] == pytest.approx(st.expected_covered[i], rel=1e-12)
            assert stats[j].generated[i] == st.generated[i]
        if j == 1:
            assert stats[j].batches > 3        # the small-capacity request kept the plain batch rules
    ctx.close()


def test_multi_request_is_repeatable_and_chunking_is_transparent(lib):
    """A second run gives the same rows; so does a run whose memory budget puts every
    request in a chunk of its own."""
    ws = requests(lib, n=4)
    ctx = G.Context(0)
    runs = []
    for budget in (0, 0, 1):
        ctx.set_multi_budget(budget)
        got = {}

        def sink(j, model, rows):
            got.setdefault((j, model), []).append(rows["lb"].copy())
        G.run_catalog_multi(ctx, ws, sink=sink)
        runs.append(got)
    for other in runs[1:]:
        assert runs[0].keys() == other.keys()
        for k in runs[0]:
            np.testing.assert_array_equal(np.concatenate(runs[0][k], axis=-1), np.concatenate(other[k], axis=-1))
    ctx.close()


def test_draw_block_size_choice_does_not_change_rows(lib):
    """The tuner picks 1, 2, 4 or 8 warps per CTA for the batched draw; every forced
    choice gives the same rows."""
    ws = requests(lib, n=4)
    ctx = G.Context(0)
    assert set(ctx.tuning().values()) == {0}
    runs = []
    for cw in (None, 1, 2, 4, 8):
        if cw is not None:
            for kind in ctx.tuning():
                ctx.set_tuning(kind, cw)
        got = {}

        def sink(j, model, rows):
            got.setdefault((j, model), []).append(np.concatenate([rows["lb"].ravel(), rows["DM"].ravel(), rows["absmag"].ravel()]))
        G.run_catalog_multi(ctx, ws, sink=sink)
        if cw is None:
            assert all(v in (1, 2, 4, 8) for v in ctx.tuning().values())
        runs.append(got)
    for other in runs[1:]:
        assert runs[0].keys() == other.keys()
        for k in runs[0]:
            np.testing.assert_array_equal(np.concatenate(runs[0][k]), np.concatenate(other[k]))
    with pytest.raises(G.GalfastError):
        ctx.set_tuning(1, 3)
    ctx.close()


def test_host_delivery_equals_device_rows(lib):
    """gf_catalog_run_multi_host: rows copied to page-locked host memory while the
    device works on, in pieces small enough to split requests, equal the rows of
    gf_catalog_run_multi (including a request that needs the plain batch rules)."""
    ws = requests(lib, n=5)
    ctx = G.Context(0)
    ref = {}

    def sink(j, model, rows):
        ref.setdefault((j, model), []).append(rows)
    st_ref = G.run_catalog_multi(ctx, ws, sink=sink)
    for piece in (0, 1000):
        got = {}

        def hsink(j, model, rows):
            got.setdefault((j, model), []).append(rows)
        st = G.run_catalog_multi_host(ctx, ws, hsink, piece_rows=piece)
        assert sorted(got) == sorted(ref)
        if piece:
            assert max(len(v) for v in got.values()) > 1          # requests split over pieces
        for k in ref:
            a = {c: np.concatenate([p[c] for p in ref[k]], axis=-1) for c in ref[k][0]}
            b = {c: np.concatenate([p[c] for p in got[k]], axis=-1) for c in got[k][0]}
            for c in a:
                x, y = a[c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]
                np.testing.assert_array_equal(x, y, err_msg="%s %s" % (c, k))
        for j in range(len(ws)):
            assert st[j].generated[:3] == st_ref[j].generated[:3]
    ctx.close()


def test_host_delivery_stops_when_the_callback_asks(lib):
    """A nonzero return of the host callback ends gf_catalog_run_multi_host with
    GF_E_STATE, whether it comes during the batched passes' rows or during the rows
    of the request that takes the plain path (whose batches follow the batched
    rows through the same copy stream); no piece reaches the callback after it,
    and the context runs the next call as before."""
    ws = requests(lib, n=5)
    ctx = G.Context(0)
    ref = {}

    def sink(j, model, rows):
        ref.setdefault((j, model), []).append(rows)
    G.run_catalog_multi_host(ctx, ws, sink, piece_rows=1000)
    for stop_job in (0, 1):                     # request 1 takes the plain path
        seen = []

        def stopper(j, model, rows):
            seen.append(j)
            return j == stop_job
        with pytest.raises(G.GalfastError, match="stopped"):
            G.run_catalog_multi_host(ctx, ws, stopper, piece_rows=1000)
        assert seen and seen[-1] == stop_job and seen.count(stop_job) == 1
    got = {}

    def again(j, model, rows):
        got.setdefault((j, model), []).append(rows)
    G.run_catalog_multi_host(ctx, ws, again, piece_rows=1000)
    assert sorted(got) == sorted(ref)
    for k in ref:
        for a, b in zip(ref[k], got[k]):
            for c in a:
                np.testing.assert_array_equal(a[c], b[c], err_msg="%s %s" % (c, k))
    ctx.close()


def test_request_that_fills_a_batch_runs_alone(lib):
    """Admission lets every request into the batched passes (margin -1000 sigma);
    the first request's halo stars (about 2850) then fill its 2000-row batch while
    its thin and thick disks (about 1000 and 1600 stars) fit.  The call does not
    fail: the request's halo rows are withheld and it runs alone afterwards,
    delivering only the halo, so every request still gets exactly the catalog
    gf_catalog_run gives it alone (two halo batches for the first)."""
    ws = [W.build_workload(lib, foot=W.cap_footprint(60.0, 70.0, 1.0), dx_deg=0.1, m0=14.0, m1=21.5,
                           capacity=2000, seed48=4242)]
    ws += requests(lib, n=3)[::2]
    ctx = G.Context(0)
    ctx.set_admission(-1000.0)
    got = {}

    def sink(j, model, rows):
        got.setdefault(j, {}).setdefault(model, []).append(rows)
    stats = G.run_catalog_multi(ctx, ws, sink=sink)
    for j, w in enumerate(ws):
        ref, st = catalog_alone(ctx, w)
        assert sorted(ref) == sorted(got[j]), j
        for m in ref:
            b = {k: np.concatenate([p[k] for p in got[j][m]], axis=-1) for k in got[j][m][0]}
            for c in ref[m]:
                x, y = ref[m][c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]
                np.testing.assert_array_equal(x, y, err_msg="%s request %d model %d" % (c, j, m))
        assert list(stats[j].generated[:3]) == list(st.generated[:3]), j
    assert stats[0].generated[0] < 2000 <= stats[0].generated[2]
    assert len(got[0][2]) >= 2 and len(got[0][0]) == 1
    ctx.close()


def test_metallicity_modules_in_the_batched_passes(lib):
    """os_FeH and os_GaussianFeH over the rows of many requests, each request's
    256-row chunks drawing from its own streams: rows equal the standalone run's."""
    ws = requests(lib, n=4)
    for w in ws:
        w.feh_ivezic = W.feh_config()
        w.feh_gauss = W.gaussfeh_config(comp_mask=0b100)
    ctx = G.Context(0)
    got = {}
    G.run_catalog_multi(ctx, ws, sink=lambda j, m, rows: got.setdefault(j, {}).setdefault(m, []).append(rows))
    for j, w in enumerate(ws):
        ref, st = catalog_alone(ctx, w)
        for m in ref:
            b = {k: np.concatenate([p[k] for p in got[j][m]], axis=-1) for k in got[j][m][0]}
            for c in ref[m]:
                x, y = ref[m][c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]
                np.testing.assert_array_equal(x, y, err_msg="%s request %d model %d" % (c, j, m))
    ctx.close()


def test_unresolved_multiples_in_the_batched_passes(lib):
    """os_unresolvedMultiples over the rows of many requests (256-row chunks on
    each request's streams), with photometry over the systems: rows equal the
    standalone run's."""
    ws = requests(lib, n=4)
    for w in ws:
        w.multiples = W.multiples_config(lib, comp_mask=0b011, fraction=W.MULT_FRACTION, lf=W.MULT_LF)
    ctx = G.Context(0)
    got = {}
    G.run_catalog_multi(ctx, ws, sink=lambda j, m, rows: got.setdefault(j, {}).setdefault(m, []).append(rows))
    for j, w in enumerate(ws):
        ref, st = catalog_alone(ctx, w)
        for m in ref:
            b = {k: np.concatenate([p[k] for p in got[j][m]], axis=-1) for k in got[j][m][0]}
            for c in ref[m]:
                x, y = ref[m][c], b[c]
                if c in ("mags", "obsmags"):
                    y = y[: x.shape[0]]
                np.testing.assert_array_equal(x, y, err_msg="%s request %d model %d" % (c, j, m))
        assert any((ref[m]["absmagSysNcomp"] == 2).any() for m in ref)
    ctx.close()
