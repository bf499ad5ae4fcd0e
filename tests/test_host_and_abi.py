"""Host logic and the C ABI (CPU only): the library loads and exports every
function include/galfast_b200.h declares; the safe-prime multipliers are
regenerated exactly; the portable math library is accurate; the host model
setup equals the oracle's; the footprint pixelisation has the configurations'
sizes; and the crawl's bin enumeration is a bijection."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W, _abi as A
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "galfast_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", src))
    return sorted(n for n in names if not n.endswith("_callback"))


def test_library_exports_every_declared_function(lib):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", G.LIBPATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (gf_\w+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in A.EXPORTS:
        assert n in exported, n


def test_struct_layouts(tmp_path):
    """Every ctypes mirror has the size and field offsets of its struct in
    include/galfast_b200.h (a C program compiled against the header prints them)."""
    import shutil
    import subprocess
    assert C.sizeof(A.PencilBeam) == 48
    assert C.sizeof(A.Lambert) == 32
    assert C.sizeof(A.Bond2010Config) == 4 * (4 + 3 * 45 + 12)
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = str(tmp_path / "abi_layout")
    here = os.path.dirname(os.path.abspath(__file__))
    subprocess.run([cc, "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", exe,
                    os.path.join(here, "cpp", "abi_layout.c")], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    mirror = {"gf_pencil_beam": A.PencilBeam, "gf_lambert": A.Lambert, "gf_skygen_config": A.SkygenConfig,
              "gf_model_config": A.ModelConfig, "gf_extinction": A.Extinction, "gf_footprint": A.Footprint,
              "gf_table": A.Table, "gf_fixedfeh_config": A.FixedFeHConfig, "gf_vmoments": A.VMoments,
              "gf_bond2010_config": A.Bond2010Config, "gf_feh_config": A.FehConfig, "gf_gaussfeh_config": A.GaussFehConfig,
              "gf_photometry_config": A.PhotometryConfig, "gf_photoerr_config": A.PhotoerrConfig,
              "gf_vel2pm_config": A.Vel2pmConfig, "gf_skygen_model_info": A.ModelInfo, "gf_job": G.Job,
              "gf_catalog_stats": G.CatalogStats, "gf_precision_report": A.PrecisionReport,
              "gf_textout_config": G.TextoutConfig, "gf_textout_set": G.TextoutSet,
              "gf_server_info": G.ServerInfo, "gf_multiples_config": A.MultiplesConfig,
              "gf_ext_map": A.ExtMap, "gf_region": A.Region}
    checked = 0
    for line in out.split("\n"):
        if not line.strip():
            continue
        name, field, value = line.split()
        T = mirror[name]
        if field == "-":
            assert C.sizeof(T) == int(value), (name, C.sizeof(T), value)
        else:
            assert getattr(T, field).offset == int(value), (name, field, getattr(T, field).offset, value)
        checked += 1
    assert checked > 60


def test_safeprime_multipliers_are_safe(multipliers):
    def is_prime(n):
        if n < 2:
            return False
        for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
            if n % p == 0:
                return n == p
        d, s = n - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
            x = pow(a, d, n)
            if x in (1, n - 1):
                continue
            for _ in range(s - 1):
                x = x * x % n
                if x == n - 1:
                    break
            else:
                return False
        return True
    rng = np.random.default_rng(3)
    for i in list(rng.integers(0, 65536, size=200)) + [0, 17157, 17158, 54734, 54735, 65535]:
        a = int(multipliers[i])
        assert is_prime(a * 2 ** 32 - 1) and is_prime(a * 2 ** 31 - 1), i
    # the three enumerations: increasing from 1, decreasing below 2^31 and below 2^32
    assert np.all(np.diff(multipliers[:17158].astype(np.int64)) > 0)
    assert np.all(np.diff(multipliers[17158:54735].astype(np.int64)) < 0) and multipliers[17158] < 2 ** 31
    assert np.all(np.diff(multipliers[54735:].astype(np.int64)) < 0) and multipliers[54735] > 2 ** 31


REFERENCE = os.environ.get("GALFAST_REFERENCE", "")


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "data", "safeprimes32.txt")),
                    reason="set GALFAST_REFERENCE to a galfast source tree")
def test_safeprime_multipliers_equal_reference_table(multipliers):
    ref = np.loadtxt(os.path.join(REFERENCE, "data", "safeprimes32.txt"), dtype=np.uint64, max_rows=65536)
    assert np.array_equal(ref[:, 0].astype(np.uint32), multipliers)
    assert np.array_equal(ref[:, 1], ref[:, 0] * 2 ** 32 - 1)


def ulp_diff32(a, b):
    ai = np.asarray(a, dtype=np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, dtype=np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, np.int64(-2 ** 31) - ai, ai)
    bi = np.where(bi < 0, np.int64(-2 ** 31) - bi, bi)
    return np.abs(ai - bi)


def test_portable_math_single_precision():
    """gf_math.h float functions are correctly rounded (vs float64 numpy) in all but rare cases."""
    L = O.load("p")
    rng = np.random.default_rng(11)
    n = 200000
    cases = [
        (0, rng.uniform(-87, 88, n).astype(np.float32), None, lambda x, y: np.exp(x.astype(np.float64))),
        (1, np.exp(rng.uniform(-80, 80, n)).astype(np.float32), None, lambda x, y: np.log(x.astype(np.float64))),
        (2, np.exp(rng.uniform(-80, 80, n)).astype(np.float32), None, lambda x, y: np.log10(x.astype(np.float64))),
        (3, rng.uniform(-37, 37, n).astype(np.float32), None, lambda x, y: 10.0 ** x.astype(np.float64)),
        (4, rng.uniform(-7, 7, n).astype(np.float32), None, lambda x, y: np.sin(x.astype(np.float64))),
        (5, rng.uniform(-7, 7, n).astype(np.float32), None, lambda x, y: np.cos(x.astype(np.float64))),
        (6, rng.uniform(0, 3.1415, n).astype(np.float32), None, lambda x, y: np.tan(x.astype(np.float64))),
        (7, rng.uniform(0, 100, n).astype(np.float32), rng.uniform(-10, 10, n).astype(np.float32),
         lambda x, y: x.astype(np.float64) ** y.astype(np.float64)),
    ]
    for kind, x, y, ref in cases:
        yy = y if y is not None else np.zeros_like(x)
        out = np.zeros_like(x)
        L.or_math_f(kind, n, x.ctypes.data, yy.ctypes.data, out.ctypes.data)
        r = ref(x, yy).astype(np.float32)
        d = ulp_diff32(out, r)
        assert d.max() <= 1, kind
        assert (d != 0).mean() < 1e-4, kind


def test_portable_math_double_precision():
    L = O.load("p")
    rng = np.random.default_rng(12)
    n = 100000
    for kind, x, y, ref, tol in [
        (0, rng.uniform(-700, 700, n), None, np.exp, 2e-16),
        (1, np.exp(rng.uniform(-700, 700, n)), None, np.log, 1e-15),
        (2, rng.uniform(-10, 10, n), None, np.sin, 1e-15),
        (3, rng.uniform(-10, 10, n), None, np.cos, 1e-15),
        (4, rng.uniform(-1, 1, n), None, np.arcsin, 1e-15),
        (5, rng.uniform(-1, 1, n), rng.uniform(-1, 1, n), np.arctan2, 1e-15),
    ]:
        yy = y if y is not None else np.zeros_like(x)
        out = np.zeros_like(x)
        L.or_math_d(kind, n, x.ctypes.data, yy.ctypes.data, out.ctypes.data)
        r = ref(x, yy) if kind == 5 else ref(x)
        err = np.abs(out - r) / np.maximum(np.abs(r), 1e-300)
        assert np.nanmax(err) < 4 * tol + 1e-300, kind


def test_host_model_setup_equals_oracle(lib):
    w = W.config1(lib, with_modules=False)
    n = len(w.models)
    info = (G.ModelInfo * n)()
    lf = np.zeros((n, 1024), dtype=np.float32)
    marr = (G.ModelConfig * n)(*w.models)
    assert lib.gf_skygen_setup_host(C.byref(w.sky), w.npixels, marr, n, info,
                                    lf.ctypes.data_as(C.POINTER(C.c_float))) == 0
    osk = O.OracleSkygen(w)
    for i in range(n):
        oi = osk.info(i)
        for f in ("m0", "m1", "dm", "M0", "M1", "dM", "nm", "nM", "f", "lf_x0", "lf_inv_dx", "lf_n"):
            assert getattr(info[i], f) == getattr(oi, f), (i, f)
        assert np.array_equal(lf[i, :info[i].lf_n], osk.lf(i))
    # the LF hint restricts the absolute-magnitude grid to the tabulated range (model_lib.h:97-112)
    assert info[0].nM == 240 and info[0].nm == 120


def test_pixelisation_sizes(lib):
    w1 = W.config1(lib, with_modules=False)
    assert w1.npixels == 1600
    pix = np.frombuffer(w1.pixels, dtype=np.float32).reshape(-1, 12)
    assert np.all(pix[:, 4] == 1.0)                  # fully covered
    X, Y = pix[:, 8], pix[:, 9]
    half = 5 * math.pi / 180
    assert np.all(np.abs(X) < half) and np.all(np.abs(Y) < half)
    w2 = W.config2(lib, with_modules=False)
    assert abs(w2.npixels - 3.41e6) / 3.41e6 < 0.01
    # the screen extinction's beam minimum never exceeds the extinction anywhere in the cell
    cb = np.frombuffer(w2.pixels, dtype=np.float32).reshape(-1, 12)
    sb = np.abs(cb[:, 3])
    assert np.all(w2.ammin <= w2.ext.A0 / sb * (1 + 1e-6))


def test_crawl_bin_order_is_a_bijection():
    """diagIndexToIJ enumerates every (m, M) bin once along diagonals of constant DM,
    and advance() steps to the next index (skygen.cu.h:231-358)."""
    L = O.load("p")
    for x, y in [(7, 5), (5, 7), (6, 6), (1, 4), (4, 1), (12, 31)]:
        seen = set()
        for k in range(x * y):
            i, j = C.c_int(), C.c_int()
            L.or_diag(k, x, y, C.byref(i), C.byref(j))
            assert 0 <= i.value < x and 0 <= j.value < y
            seen.add((i.value, j.value))
            if k + 1 < x * y:
                i2, j2 = C.c_int(), C.c_int()
                L.or_diag(k + 1, x, y, C.byref(i2), C.byref(j2))
                ii, jj = C.c_int(i.value), C.c_int(j.value)
                L.or_advance(C.byref(ii), C.byref(jj), x, y)
                assert (ii.value, jj.value) == (i2.value, j2.value), (x, y, k)
                assert i2.value + j2.value >= i.value + j.value
        assert len(seen) == x * y


def test_table_rows_reads_a_row_range_of_a_host_table():
    """table_rows (the host-delivery callback's view of a piece) copies rows [a, b) of
    every column of a gf_table in host memory, vector columns as (components, rows)."""
    h = G.HostTable(16, 5)
    for name, dt, nc in G.COLUMNS:
        k = 5 if nc == "bands" else nc
        arr = h.arrays[name]
        arr[...] = (np.arange(k * 16, dtype=np.float64).reshape(arr.shape) + 0.5).astype(dt)
    rows = G.table_rows(h.t, 3, 9)
    assert set(rows) == {name for name, _, _ in G.COLUMNS}
    for name, dt, nc in G.COLUMNS:
        full = h.arrays[name].reshape(-1, 16)
        want = full[:, 3:9]
        got = rows[name] if rows[name].ndim == 2 else rows[name][None, :]
        np.testing.assert_array_equal(got, want, err_msg=name)
        assert rows[name].dtype == np.dtype(dt)
    # copies, not views: the ring slot behind a delivered piece is reused after the callback
    rows["DM"][0] = -1.0
    assert h.arrays["DM"].reshape(-1)[3] != -1.0


def test_uniform_threshold_integer_test_equals_float_test(tmp_path):
    """The batched draw compares the MWC state x with an integer threshold instead
    of converting x to the uniform 2^-32 * (float)x: for 2.2e6 thresholds (random,
    tiny, and around every power of two) the threshold passes u <= thr and the next
    integer does not (tests/cpp/uniform_threshold_check.cu, run on the host)."""
    import shutil
    import subprocess
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "utc")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                    "-ffp-contract=off", "-I", os.path.join(ROOT, "galfast_b200", "csrc"), "-o", exe,
                    os.path.join(here, "cpp", "uniform_threshold_check.cu")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    n, bad = (int(x) for x in r.stdout.split())
    assert r.returncode == 0 and bad == 0 and n > 2000000, r.stdout


def _interp(xa, ya, x):
    """GSL linear interpolation with linear extrapolation (the reference's spline)."""
    n = len(xa)
    lo, hi = 0, n - 1
    while hi > lo + 1:
        mid = (hi + lo) // 2
        if xa[mid] > x:
            hi = mid
        else:
            lo = mid
    dx = xa[lo + 1] - xa[lo]
    return ya[lo] + (x - xa[lo]) / dx * (ya[lo + 1] - ya[lo]) if dx > 0 else 0.0


def test_multiples_tables_follow_the_reference_construction(lib):
    """gf_multiples_build: the binary fraction resampled to 64 texels, the
    normalised trapezoid integral of the secondaries' LF at 256 points and its
    inverse resampled to 256 texels (unresolvedMultiples_host.cpp:120-189,
    cux.cpp:330-350), restated here in Python double precision."""
    from galfast_b200 import workloads as W
    fm, fp = W.MULT_FRACTION
    lm, lp = W.MULT_LF
    c = W.multiples_config(lib, algo=A.GF_MULT_LF, comp_mask=5, fraction=W.MULT_FRACTION, lf=W.MULT_LF)
    assert c.algo == A.GF_MULT_LF and c.comp_mask == 5 and c.nsec == 64 and c.ncum == c.ninv == 256

    def resample(X, Y, n):
        X0, X1 = X[0], X[-1]
        dX = (X1 - X0) / (n - 1)
        return [np.float32(_interp(X, Y, X0 + i * dX)) for i in range(n)], np.float32(X0), np.float32(1.0 / dX)
    tab, x0, inv = resample(fm, fp, 64)
    assert list(np.array(c.secprob[:64], dtype=np.float32)) == tab and c.sec_x0 == x0 and c.sec_inv_dx == inv
    dx = (lm[-1] - lm[0]) / 255
    xc, yc = [lm[0]], [0.0]
    yprev = _interp(lm, lp, lm[0])
    for i in range(1, 256):
        xx = lm[0] + i * dx
        yy = _interp(lm, lp, xx)
        xc.append(xx)
        yc.append(yc[-1] + (yprev + 0.5 * (yy - yprev)) * dx)
        yprev = yy
    yc = [v / yc[-1] for v in yc]
    tab, x0, inv = resample(xc, yc, 256)
    assert list(np.array(c.cumlf[:256], dtype=np.float32)) == tab and c.cum_x0 == x0 and c.cum_inv_dx == inv
    tab, x0, inv = resample(yc, xc, 256)
    assert list(np.array(c.invcumlf[:256], dtype=np.float32)) == tab and c.inv_x0 == x0 and c.inv_inv_dx == inv
    # no fraction file: 1 over [-100, 100] (two texels); no LF: flat
    d = W.multiples_config(lib, algo=A.GF_MULT_EQUAL_MASS)
    assert d.nsec == 2 and list(d.secprob[:2]) == [1.0, 1.0] and d.sec_x0 == -100.0
    assert abs(d.cumlf[128] - 128 / 255) < 1e-6
    with pytest.raises(RuntimeError):
        W.multiples_config(lib, algo=7)


def test_extinction_beam_minima_follow_the_reference(lib):
    """gf_extinction_beam_minima restates find_extinction_minima
    (os_skygen.cpp:285-342): for every beam and DM texel z, the smallest A(x, y, z-1)
    (0 at z = 0) over the texels of each map within the beam's reach, skipping empty
    texels outside the hemisphere's disk.  Checked against a Python restatement on
    the beams of a cap that straddles the plane (both maps contribute)."""
    import math
    from galfast_b200 import workloads as W
    w = W.build_workload(lib, foot=W.cap_footprint(40.0, 2.0, 2.0), dx_deg=0.5, m0=15.0, m1=17.0, with_modules=False)
    W.use_extinction_maps(lib, w, nxy=40, nz=8)
    nz = len(w.ammin) // w.npixels
    assert nz == 8
    maps = [w.ext.north.contents, w.ext.south.contents]
    pix = w.pixel_array()
    f32 = np.float32
    for i in range(0, w.npixels, max(1, w.npixels // 25)):
        p = pix[i]
        want = np.full(nz, np.inf, dtype=np.float32)
        for h in range(2):
            e = maps[h]
            nx, ny, d = e.n[0], e.n[1], e.n[2]
            A_ = np.ctypeslib.as_array(e.A, shape=(d * ny * nx,)).reshape(d, ny, nx)
            pr = w.sky.proj[h]
            # float products and sums (as the reference's float expressions), widened to double
            cll0 = float(f32(f32(p.cl * pr.cl) + f32(p.sl * pr.sl)))
            sll0 = float(f32(f32(pr.cl * p.sl) - f32(p.cl * pr.sl)))
            kp = 1.414213562373095 * math.sqrt(1.0 / (1.0 + float(f32(pr.sb * p.sb)) + float(f32(pr.cb * p.cb)) * cll0))
            x = float(f32(kp * p.cb * sll0))
            y = float(f32(kp * (pr.cb * p.sb - float(f32(pr.sb * p.cb)) * cll0)))
            tcx0, tcxy, tcy0, tcyy = (float(e.tc[0][0]), float(e.tc[0][1]), float(e.tc[1][0]), float(e.tc[1][1]))
            dr = 1.0001 / 2.0 * math.sqrt(2) * (float(p.dx) + max(1.0 / tcxy, 1.0 / tcyy))
            xi = max(0, min(int((x - dr - tcx0) * tcxy) - 1, nx))
            yi = max(0, min(int((y - dr - tcy0) * tcyy) - 1, ny))
            xie = max(0, min(int((x + dr - tcx0) * tcxy) + 2, nx))
            yie = max(0, min(int((y + dr - tcy0) * tcyy) + 2, ny))
            for X in range(xi, xie):
                for Y in range(yi, yie):
                    if Y >= nx:
                        continue
                    if A_[d - 1, Y, X] == 0:
                        xx, yy = X / tcxy + tcx0, Y / tcyy + tcy0
                        if xx * xx + yy * yy > 2:
                            continue
                    col = np.concatenate([[0.0], A_[:d - 1, Y, X]]).astype(np.float32)
                    want = np.minimum(want, col)
        got = w.ammin[p.extIdx * nz:(p.extIdx + 1) * nz]
        np.testing.assert_array_equal(got, want, err_msg="beam %d" % i)


def _pixel_lb(w):
    pix = w.pixel_array()
    l = np.array([math.degrees(math.atan2(p.sl, p.cl)) % 360.0 for p in pix])
    b = np.array([math.degrees(math.atan2(p.sb, p.cb)) for p in pix])
    area = np.array([p.dA * p.coveredFraction for p in pix])
    return l, b, area


def test_footprint_regions_pixelise_to_their_areas(lib):
    """GF_FOOT_REGIONS: a beam with a hole, a union of overlapping beams, a lon/lat
    rectangle minus the |b| < bmin band, and an equatorial beam around the north
    celestial pole, pixelised on 0.2 deg Lambert cells: the covered areas match the
    regions' areas to 1 %, and the equatorial beam lands on the galactic position of
    the pole (l, b) = (122.93, 27.13) deg."""
    import math
    from galfast_b200 import workloads as W
    d2r = math.pi / 180

    def area_of(foot):
        w = W.build_workload(lib, foot=foot, dx_deg=0.2, m0=15.0, m1=16.0, with_modules=False)
        l, b, a = _pixel_lb(w)
        return a.sum(), l, b, a

    cap = lambda r: 2 * math.pi * (1 - math.cos(r * d2r))
    got, _, _, _ = area_of(W.regions_footprint([dict(type="beam", v=(40, 30, 6, 2))]))
    assert got == pytest.approx(cap(6) - cap(2), rel=0.01)
    got, _, _, _ = area_of(W.regions_footprint([dict(type="beam", v=(40, 30, 5, 0)), dict(type="beam", v=(40, 30, 3, 0)),
                                                dict(type="beam", v=(200, -40, 4, 0))]))
    assert got == pytest.approx(cap(5) + cap(4), rel=0.01)
    got, _, _, _ = area_of(W.regions_footprint([dict(type="rect", v=(100, 130, -20, 25), bmin=10)]))
    strip = lambda b0, b1: (math.sin(b1 * d2r) - math.sin(b0 * d2r)) * 30 * d2r
    assert got == pytest.approx(strip(-20, -10) + strip(10, 25), rel=0.01)
    got, l, b, a = area_of(W.regions_footprint([dict(type="beam", coordsys="equ", v=(0, 90, 3, 0))]))
    assert got == pytest.approx(cap(3), rel=0.01)
    assert np.average(b, weights=a) == pytest.approx(27.13, abs=0.2)
    assert np.average(l, weights=a) == pytest.approx(122.93, abs=0.5)
