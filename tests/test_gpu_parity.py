"""GPU parity: the sm_100a library against the CPU oracle (the reference CPU
path restated) on the same seeded inputs, through the C ABI.

Per-bin expected counts, Poisson draws and every skygen column must be
bit-exact; the module columns are required to agree within 1e-5 relative
(they are computed with the same portable math, so they are normally exact).
"""
import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SKY_COLS = ["lb", "projIdx", "projXY", "DM", "absmag", "XYZ", "comp", "Am", "AmInf", "hidden"]
MODULE_COLS = ["FeH", "vcyl", "mags", "photoflags", "obsmags", "pm", "radec"]
RTOL = 1e-5


def small_patch(lib, half_deg=2.5, **kw):
    import math
    from galfast_b200 import _abi as A
    half = half_deg * math.pi / 180
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    return W.build_workload(lib, foot=foot, dx_deg=0.25, m0=15.0, m1=kw.pop("m1", 21.0), **kw)


def assert_same(g, o, names, exact=True):
    for n in names:
        a, b = g[n], o[n]
        assert a.shape == b.shape, n
        if exact:
            if a.dtype.kind == "f":
                same = (a == b) | (np.isnan(a) & np.isnan(b))
                assert same.all(), "%s differs in %d of %d values" % (n, (~same).sum(), same.size)
            else:
                assert np.array_equal(a, b), n
        else:
            if a.dtype.kind == "f":
                np.testing.assert_allclose(a, b, rtol=RTOL, atol=1e-6, err_msg=n)
            else:
                assert np.array_equal(a, b), n


def test_seed_parity(ctx, multipliers):
    ctx.rng_init(42, 65536)
    assert np.array_equal(ctx.rng_state(), O.seed_streams(42, multipliers))


@pytest.mark.parametrize("nthreads", [7680, 640, 33])
def test_integrate_parity(ctx, lib, nthreads):
    w = small_patch(lib, nthreads=nthreads, with_modules=False)
    sky = G.Skygen(ctx, w)
    osk = O.OracleSkygen(w)
    for m in range(3):
        ge, gc, gp = sky.integrate_counts(m, per_pixel=True)
        oe, oc, op = osk.integrate_counts(m, per_pixel=True)
        assert ge == pytest.approx(oe, rel=1e-12)
        assert gc == pytest.approx(oc, rel=1e-12)
        np.testing.assert_allclose(gp, op, rtol=1e-6)


def test_integrate_straddling_blocks(ctx, lib):
    """nm * nM not a multiple of 10: blocks run past the end of a pixel and the
    reference's pixel blocking changes the anchors (skyconfig_impl.h:344-387)."""
    w = small_patch(lib, half_deg=1.0, nthreads=300, with_modules=False, m1=21.05, M1=14.9)
    sky = G.Skygen(ctx, w)
    osk = O.OracleSkygen(w)
    inf = sky.info(0)
    assert (inf.nm * inf.nM) % 10 != 0
    for m in range(3):
        ge, gc, _ = sky.integrate_counts(m)
        oe, oc, _ = osk.integrate_counts(m)
        assert ge == pytest.approx(oe, rel=1e-12)


def draw_all(ctx, w, multipliers, capacity, between=None):
    """Draw every model batch by batch on both sides and compare each batch."""
    ctx.rng_init(w.seed48, 65536)
    ostate = O.seed_streams(w.seed48, multipliers)
    sky = G.Skygen(ctx, w)
    osk = O.OracleSkygen(w)
    for m in range(3):
        sky.integrate_counts(m)
        osk.integrate_counts(m)
    dt = G.DeviceTable(ctx, capacity, 0)
    ht = G.HostTable(capacity, 0)
    nb = 0
    total = 0
    try:
        for m in range(3):
            while True:
                ng, dg = sky.draw_sources(m, dt)
                no, do = osk.draw_sources(m, ostate, ht)
                assert (ng, dg) == (no, do)
                g = dt.download()
                assert g.size == ht.size
                assert_same(g.as_dict(SKY_COLS), ht.as_dict(SKY_COLS), SKY_COLS)
                N = w.sky.nthreads
                gs = ctx.rng_state().reshape(3, -1)[:, :N]
                os_ = ostate.reshape(3, -1)[:, :N]
                assert np.array_equal(gs, os_), "stream states differ after a batch"
                nb += 1
                total += ht.size
                if dg:
                    break
    finally:
        dt.free()
    return nb, total


def test_draw_single_batch(ctx, lib, multipliers):
    w = small_patch(lib, with_modules=False)
    nb, total = draw_all(ctx, w, multipliers, capacity=1 << 18)
    assert nb == 3 and total > 1000


@pytest.mark.parametrize("nthreads,capacity", [(7680, 3000), (97, 1777)])
def test_draw_multi_batch(ctx, lib, multipliers, nthreads, capacity):
    w = small_patch(lib, half_deg=1.5, nthreads=nthreads, with_modules=False)
    nb, total = draw_all(ctx, w, multipliers, capacity=capacity)
    assert nb > 3


def test_draw_straddling_blocks(ctx, lib, multipliers):
    w = small_patch(lib, half_deg=1.0, nthreads=300, with_modules=False, m1=21.05, M1=14.9)
    nb, total = draw_all(ctx, w, multipliers, capacity=1 << 16)
    assert total > 100


def run_both(ctx, w, multipliers):
    gb, ob = [], []

    def gsink(model, t, off):
        gb.append((model, off, t.as_dict()))

    def osink(model, t, off):
        ob.append((model, off, t.as_dict()))

    gs = G.run_catalog(ctx, w, gsink)
    os_, _ = O.run_catalog(w, multipliers, sink=osink)
    return gs, os_, gb, ob


@pytest.mark.parametrize("capacity", [1 << 18, 4000])
def test_catalog_parity(ctx, lib, multipliers, capacity):
    """The whole path -- skygen, clipper, fixedFeH, Bond2010 (sharing the streams
    between batches), photometry, photometric errors, vel2pm, gal2other."""
    w = small_patch(lib, capacity=capacity)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    assert len(gb) == len(ob) > 0
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert (gm, go) == (om, oo)
        assert_same(g, o, SKY_COLS)
        assert_same(g, o, MODULE_COLS, exact=False)
    for m in range(3):
        assert gs.generated[m] == os_["generated"][m]


def test_catalog_parity_lsst_ugrizy(ctx, lib, multipliers):
    """The six-band LSST-like system (five colours: two colour textures in the
    reference, photometry_host.cpp:233-344) with depths one magnitude deeper."""
    w = small_patch(lib, capacity=1 << 18, nbands=6, m5=W.LSST_M5)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    assert len(gb) == len(ob) > 0
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert (gm, go) == (om, oo)
        assert g["mags"].shape[0] == 6 and g["obsmags"].shape[0] == 6
        assert_same(g, o, SKY_COLS)
        assert_same(g, o, MODULE_COLS, exact=False)


@pytest.mark.parametrize("nbands,m5", [(5, W.SDSS_M5), (6, W.LSST_M5)])
def test_photometric_error_statistics(ctx, lib, nbands, m5):
    """os_photometricErrors draws obs = true + sigma(true) * N(0, 1) with
    sigma(m) = 0.005 + 0.04 * 10^(0.4 (m - m5)) (photometricErrors_host.cpp:112-131,
    the configurations' error model).  Over more than 1e6 rows per band: the
    normalised deviations have mean 0 (within 5 / sqrt(n)) and standard deviation 1
    (within 1 %), and in every 0.5-mag bin of true magnitude the spread of
    obs - true equals the formula's sigma within 3 %."""
    w = W.build_workload(lib, foot=W.cap_footprint(60.0, 40.0, 10.0), dx_deg=0.1, m0=14.0, m1=22.0,
                         capacity=1 << 22, nbands=nbands, m5=m5)
    true, obs = [], []

    def sink(model, t, off):
        d = t.as_dict(["mags", "obsmags", "hidden"])
        vis = d["hidden"] == 0
        true.append(d["mags"][:, vis].astype(np.float64))
        obs.append(d["obsmags"][:, vis].astype(np.float64))
    G.run_catalog(ctx, w, sink)
    true = np.concatenate(true, axis=1)
    obs = np.concatenate(obs, axis=1)
    n = true.shape[1]
    assert n > 1e6
    for b in range(nbands):
        m = true[b]
        sig = 0.005 + 0.04 * 10.0 ** (0.4 * (m - m5[b]))
        z = (obs[b] - m) / sig
        assert abs(z.mean()) < 5.0 / np.sqrt(n), (b, z.mean())
        assert abs(z.std() - 1.0) < 0.01, (b, z.std())
        edges = np.arange(np.floor(m.min()), np.ceil(m.max()) + 0.5, 0.5)
        which = np.digitize(m, edges)
        for k in np.unique(which):
            sel = which == k
            if sel.sum() < 20000:
                continue
            ratio = (obs[b][sel] - m[sel]).std() / np.sqrt(np.mean(sig[sel] ** 2))
            assert abs(ratio - 1.0) < 0.03, (b, edges[k - 1], ratio)


def test_config1_catalog(ctx, lib, multipliers):
    """Configuration 1 in full (about 1e5 stars)."""
    w = W.config1(lib)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    n = sum(len(g["DM"]) for _, _, g in gb)
    assert 5e4 < n < 2e5
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert_same(g, o, SKY_COLS)
        assert_same(g, o, MODULE_COLS, exact=False)


def test_metallicity_modules_parity(ctx, lib, multipliers):
    """os_FeH (Ivezic et al. 2008) and os_GaussianFeH (halo only, two Gaussians)
    draw from the shared streams between the clipper and Bond2010; a 4000-row
    batch capacity makes the streams carry over between batches."""
    w = small_patch(lib, capacity=4000)
    w.feh = None
    w.feh_ivezic = W.feh_config()
    w.feh_gauss = W.gaussfeh_config(comp_mask=0b100)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    assert len(gb) == len(ob) > 3
    nonzero = 0
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert (gm, go) == (om, oo)
        assert_same(g, o, SKY_COLS)
        assert_same(g, o, MODULE_COLS + ["FeH_comp"], exact=False)
        nonzero += int((g["FeH_comp"] == 1).sum())
    assert nonzero > 0


@pytest.mark.parametrize("algo", [1, 2, 3])
def test_unresolved_multiples_parity(ctx, lib, multipliers, algo):
    """os_unresolvedMultiples between the metallicities and Bond2010 (the disks
    only), for each secondary-magnitude algorithm: the system magnitudes, the
    component magnitudes and counts, and the photometry summed over the
    components equal the oracle's; the streams carry the module's uniforms into
    Bond2010 and across 4000-row batches."""
    w = small_patch(lib, capacity=4000)
    w.multiples = W.multiples_config(lib, algo=algo, comp_mask=0b011, fraction=W.MULT_FRACTION, lf=W.MULT_LF)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    assert len(gb) == len(ob) > 3
    binaries = singles = 0
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert (gm, go) == (om, oo)
        assert_same(g, o, SKY_COLS + ["absmagSys", "absmagSysNcomp"])
        assert_same(g, o, MODULE_COLS, exact=False)
        vis = g["hidden"] == 0
        disk = vis & (g["comp"] != 2)
        binaries += int((g["absmagSysNcomp"][disk] == 2).sum())
        singles += int((g["absmagSysNcomp"][disk] == 1).sum())
        assert (g["absmagSysNcomp"][vis & (g["comp"] == 2)] == 1).all()
        two = g["absmagSysNcomp"] == 2
        if algo == 1:
            assert (g["absmagSys"][1][two] >= g["absmagSys"][0][two]).all()
        if algo == 3:
            assert (g["absmagSys"][1][two] == g["absmagSys"][0][two]).all()
    assert binaries > 100 and singles > 100


def test_footprint_regions_parity(ctx, lib, multipliers):
    """GF_FOOT_REGIONS on the device clipper: an equatorial beam with a hole around
    (ra, dec) = (210, 30) and a galactic rectangle minus |b| < 52 deg; the clipped
    catalog (hidden flags and all columns) equals the oracle's, the clipper hides
    stars of both regions' edge pixels, and visible stars satisfy the regions."""
    import math
    foot = W.regions_footprint([dict(type="beam", coordsys="equ", v=(210.0, 30.0, 3.0, 1.0)),
                                dict(type="rect", v=(40.0, 48.0, 48.0, 58.0), bmin=52.0)])
    w = W.build_workload(lib, foot=foot, dx_deg=0.25, m0=15.0, m1=20.0, capacity=1 << 18, seed48=11)
    gs, os_, gb, ob = run_both(ctx, w, multipliers)
    assert len(gb) == len(ob) > 2
    hidden = visible = 0
    for (gm, go, g), (om, oo, o) in zip(gb, ob):
        assert (gm, go) == (om, oo)
        assert_same(g, o, SKY_COLS)
        vis = g["hidden"] == 0
        # module columns of the rows the clipper hid are not written (the oracle's
        # reused table keeps an earlier batch's values there): compare the visible rows
        assert_same({k: g[k][..., vis] for k in MODULE_COLS}, {k: o[k][..., vis] for k in MODULE_COLS}, MODULE_COLS,
                    exact=False)
        visible += int(vis.sum())
        hidden += int((~vis).sum())
        b = g["lb"][1][vis]
        rect = (g["lb"][0][vis] >= 40.0) & (g["lb"][0][vis] < 48.0)
        assert (np.abs(b[rect]) >= 52.0).all()
    assert visible > 1000 and hidden > 100
