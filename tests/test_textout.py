"""The catalog text writer (gf_textout, the reference's os_textout,
src/pipeline.cpp:199-289) on host tables -- CPU only.

Every number is compared with printf-style formatting of the same value
(Python's %-formatting gives the correctly rounded decimal with ties to even,
as glibc's printf; NaN keeps its sign as glibc prints it), the header with the
reference's column definitions (otable.cpp:409-467, 542-558) and column order
(otable.cpp:517-540).
"""
import math
import os

import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W


def printf(fmt, v):
    if isinstance(v, float) and math.isnan(v):
        s = ("-" if math.copysign(1.0, v) < 0 else (" " if fmt.startswith("% ") else "")) + "nan"
        return s.rjust(int(fmt.strip("% ").split(".")[0]))
    return fmt % v


# (column, printf format) of the ranked output columns of the configurations'
# module chain, in the reference's order (gal2other and vel2pm equatorial); the
# photometry columns follow, sorted by name without regard to case
RANKED = [("lb", "% 13.8f"), ("radec", "% 13.8f"), ("XYZ", "% 10.2f"), ("DM", "% 7.3f"), ("absmag", "% 7.3f"),
          ("comp", "%3d"), ("FeH", "% 6.3f"), ("vcyl", "% 7.1f"), ("pm", "% 8.2f"), ("Am", "%6.3f"),
          ("AmInf", "%6.3f")]


def photometry_columns(nbands):
    """(header definition, column, format) of the photometry columns in output order."""
    pre, bs = ("SDSS", "SDSSugriz") if nbands == 5 else ("LSST", "LSSTugrizy")
    names = [pre + c for c in "ugrizy"[:nbands]]
    fn = ",".join("%d:%s" % (i, b) for i, b in enumerate(names))
    ofn = ",".join("%d:obs%s" % (i, b) for i, b in enumerate(names))
    cols = [("%s[%d]{class=magnitude;fieldNames=%s;}" % (bs, nbands, fn), "mags", "% 7.3f"),
            ("%sPhotoFlags{class=flags;}" % bs, "photoflags", "% 4d"),
            ("obs%s[%d]{class=magnitude;fieldNames=%s;}" % (bs, nbands, ofn), "obsmags", "% 7.3f")]
    return sorted(cols, key=lambda c: c[0].split("[")[0].split("{")[0].lower()), names


def header(nbands=5, version=None):
    phot, names = photometry_columns(nbands)
    h = ("# lb[2] radec[2] XYZ[3] DM abs%s{alias=M1;alias=absmag;band=%s;} comp FeH vcyl[3] pmradec[3] Am AmInf "
         % (names[2], names[2])) + "".join(d + " " for d, _, _ in phot)
    if version:
        h += "\n# generated with galfast version " + version
    return h + "\n"


def expected_rows(cols, n, nbands=5, comp_ids=None):
    """printf-formatted lines of the rows that are not hidden; cols: {name: (ncomp, rows) array}."""
    order = RANKED + [(c, f) for _, c, f in photometry_columns(nbands)[0]]
    lines = []
    for r in range(n):
        if cols["hidden"][0, r]:
            continue
        f = []
        for name, fmt in order:
            a = cols[name]
            for k in range(a.shape[0]):
                v = a[k, r]
                if name == "comp" and comp_ids is not None:
                    v = comp_ids[v]
                f.append(printf(fmt, int(v) if fmt.endswith("d") else float(v)))
        lines.append(" ".join(f) + "\n")
    return "".join(lines)


def assert_same_text(got, exp):
    """Equal texts; otherwise the first differing line (a diff of the whole file is too slow)."""
    if got == exp:
        return
    g, e = got.split("\n"), exp.split("\n")
    for i, (a, b) in enumerate(zip(g, e)):
        if a != b:
            raise AssertionError("line %d differs:\n got %r\nwant %r" % (i, a, b))
    raise AssertionError("%d lines, want %d" % (len(g), len(e)))


def random_table(n, nbands=5, seed=1):
    rng = np.random.default_rng(seed)
    t = G.HostTable(n + 16, nbands)
    t.t.size = n
    A = t.arrays
    A["lb"][0, :n] = rng.uniform(0, 360, n)
    A["lb"][1, :n] = rng.uniform(-90, 90, n)
    A["radec"][0, :n] = rng.uniform(0, 360, n)
    A["radec"][1, :n] = rng.uniform(-90, 90, n)
    A["XYZ"][:, :n] = rng.normal(0, 5000, (3, n)).astype(np.float32)
    A["DM"][0, :n] = rng.uniform(5, 20, n)
    A["absmag"][0, :n] = rng.uniform(-1, 16, n)
    A["comp"][0, :n] = rng.integers(0, 3, n)
    A["FeH"][0, :n] = rng.uniform(-3, 0.5, n)
    A["vcyl"][:, :n] = rng.normal(0, 150, (3, n))
    A["pm"][:, :n] = rng.normal(0, 30, (3, n))
    A["Am"][0, :n] = rng.uniform(0, 1, n)
    A["AmInf"][0, :n] = rng.uniform(0, 1, n)
    A["mags"][:, :n] = rng.uniform(10, 30, (nbands, n))
    A["obsmags"][:, :n] = rng.uniform(10, 30, (nbands, n))
    A["photoflags"][0, :n] = rng.integers(0, 64, n)
    A["hidden"][0, :n] = (rng.uniform(0, 1, n) < 0.1).astype(np.int32)
    # ties at the printed precision, signed zeros, values that round across a
    # power of ten, NaN and infinities, the largest floats
    edge32 = np.array([0.0, -0.0, 0.0005, -0.0005, 0.0015, 0.0025, 9.9995, -9.9995, 99.9995, 1e-30, -1e-30,
                       np.inf, -np.inf, np.nan, -np.nan, 3.4e38, -3.4e38, 1234567.8, 0.125, 2.5], dtype=np.float32)
    k = len(edge32)
    for name in ("DM", "absmag", "FeH", "Am", "AmInf"):
        A[name][0, :k] = edge32
    A["XYZ"][0, :k] = edge32
    A["vcyl"][1, :k] = edge32
    A["pm"][2, :k] = edge32
    A["mags"][3, :k] = edge32
    edge64 = np.array([0.0, -0.0, 0.000000005, 0.000000015, 359.999999995, -89.999999995, 1e300, -1e300, 1e-300,
                       np.nan, np.inf, 2.0 ** 93, 2.0 ** 94 + 0.5, 123.456789125, 0.5e-8, 1.5e-8], dtype=np.float64)
    A["lb"][0, :len(edge64)] = edge64
    A["radec"][1, :len(edge64)] = edge64
    A["hidden"][0, :40] = 0
    A["photoflags"][0, :3] = [-5, 12345, -123456]
    return t


def workload(lib, **kw):
    return W.build_workload(lib, foot=W.cap_footprint(0.0, 90.0, 0.5), dx_deg=0.25, m0=15.0, m1=16.0, **kw)


@pytest.mark.parametrize("threads", [1, 5])
def test_text_rows_equal_printf(tmp_path, lib, threads):
    n = 50000
    t = random_table(n)
    cfg = G.textout_config(workload(lib), threads=threads, version="0.0.0-test")
    path = tmp_path / "sky.obs.txt"
    wr = G.TextWriter(path, cfg)
    wr.write(t.t, 0, 20000)
    wr.write(t.t, 20000, 20000)
    wr.write(t.t, 20000, n)
    rows, nbytes = wr.close()
    text = path.read_text()
    assert_same_text(text, header(version="0.0.0-test") + expected_rows(t.arrays, n))
    assert rows == int((t.arrays["hidden"][0, :n] == 0).sum())
    assert nbytes == os.path.getsize(path)


def test_text_component_ids_and_lsst_bands(tmp_path, lib):
    n = 3000
    t = random_table(n, nbands=6, seed=2)
    cfg = G.textout_config(workload(lib, nbands=6, m5=W.LSST_M5))
    ids = (G.C.c_int32 * 3)(10, 20, 30)
    cfg.comp_ids = ids
    cfg.ncomp = 3
    path = tmp_path / "lsst.txt"
    wr = G.TextWriter(path, cfg)
    wr.write(t.t, 0, n)
    wr.close()
    assert_same_text(path.read_text(), header(nbands=6) + expected_rows(t.arrays, n, nbands=6, comp_ids=[10, 20, 30]))


def test_text_writer_rejects_tables_without_its_columns(tmp_path, lib):
    t = random_table(10)
    t.t.radec = None
    wr = G.TextWriter(tmp_path / "x.txt", G.textout_config(workload(lib)))
    with pytest.raises(G.GalfastError):
        wr.write(t.t, 0, 10)
    wr.close()


@pytest.mark.gpu
def test_config1_text_catalog_equals_oracle(tmp_path, lib, multipliers):
    """Configuration 1 generated on the device and written through gf_textout
    equals the oracle's catalog formatted with printf, byte for byte."""
    from oracle import oracle as O
    w = W.config1(lib)
    ctx = G.Context(0)
    path = tmp_path / "gpu.txt"
    wr = G.TextWriter(path, G.textout_config(w, version="b200"))
    G.run_catalog(ctx, w, lambda m, t, off: wr.write(t.t, 0, t.size))
    rows, _ = wr.close()
    ctx.close()
    parts = [header(version="b200")]
    O.run_catalog(w, multipliers, sink=lambda m, t, off: parts.append(expected_rows(t.arrays, t.size)), threads=8)
    assert_same_text(path.read_text(), "".join(parts))
    assert rows > 5e4


@pytest.mark.gpu
def test_multi_request_catalogs_through_the_text_sink(tmp_path, lib):
    """gf_textout_multi_sink on gf_catalog_run_multi_host: every request's file
    equals the one written from its standalone gf_catalog_run."""
    L = lib
    reqs = W.config4_requests(3, seed=31)
    ws = [W.config4_workload(L, dict(r, r=0.6 + 0.3 * k, rmax=20.0 + 0.4 * k), capacity=1 << 20)
          for k, r in enumerate(reqs)]
    n = len(ws)
    ctx = G.Context(0)
    writers = [G.TextWriter(tmp_path / ("multi%d.txt" % j), G.textout_config(w)) for j, w in enumerate(ws)]
    arr = (G.C.c_void_p * n)(*[wr.h.value for wr in writers])
    tset = G.TextoutSet(n, G.C.cast(arr, G.C.POINTER(G.C.c_void_p)))
    sink = G.MultiHostCallback(G.C.cast(L.gf_textout_multi_sink, G.C.c_void_p).value)
    jobs = (G.Job * n)(*[w.job(G.Job) for w in ws])
    stats = (G.CatalogStats * n)()
    G.check(L.gf_catalog_run_multi_host(ctx.h, jobs, n, 5000, sink, G.C.byref(tset), stats))
    for wr in writers:
        wr.close()
    for j, w in enumerate(ws):
        p = tmp_path / ("alone%d.txt" % j)
        wr = G.TextWriter(p, G.textout_config(w))
        G.run_catalog(ctx, w, lambda m, t, off: wr.write(t.t, 0, t.size))
        wr.close()
        assert_same_text((tmp_path / ("multi%d.txt" % j)).read_text(), p.read_text())
    ctx.close()


# ---------------- FITS catalogs (os_fitsout) ----------------

def read_fits(path):
    """A minimal reader of this writer's files (FITS standard 4.0): the HDUs as
    (header cards {keyword: value}, raw data bytes)."""
    raw = open(path, "rb").read()
    assert len(raw) % 2880 == 0
    hdus, pos = [], 0
    while pos < len(raw):
        cards, order = {}, []
        while True:
            blk = raw[pos:pos + 2880]
            pos += 2880
            done = False
            for k in range(36):
                c = blk[80 * k:80 * k + 80].decode("ascii")
                key = c[:8].strip()
                if key == "END":
                    done = True
                    break
                if c[8:10] == "= ":
                    v = c[10:].strip()
                    if v.startswith("'"):
                        v = v[1:v.rindex("'")].replace("''", "'").rstrip()
                    elif v in ("T", "F"):
                        v = v == "T"
                    else:
                        v = int(v)
                    cards[key] = v
                    order.append(key)
            if done:
                break
        nbytes = cards.get("NAXIS1", 0) * cards.get("NAXIS2", 0) if cards.get("NAXIS", 0) == 2 else 0
        data = raw[pos:pos + nbytes]
        pos += (nbytes + 2879) // 2880 * 2880
        hdus.append((cards, order, data))
    return hdus


def fits_columns(cards, data):
    """{TTYPE: array (nrows, width)} of a binary table with D/E/J columns."""
    codes = {"D": ">f8", "E": ">f4", "J": ">i4"}
    fields = []
    for i in range(cards["TFIELDS"]):
        form = cards["TFORM%d" % (i + 1)]
        fields.append((cards["TTYPE%d" % (i + 1)], codes[form[-1]], (int(form[:-1]),)))
    rec = np.frombuffer(data, dtype=np.dtype(fields), count=cards["NAXIS2"])
    return {name: rec[name] for name, _, _ in fields}


def test_fits_catalog_structure_and_rows(tmp_path, lib):
    """The FITS catalog: an empty primary HDU, CATALOG with one column per output
    column in the text file's order and every visible row, big-endian; METADATA
    with the text header's column definitions."""
    n = 40000
    t = random_table(n)
    cfg = G.textout_config(workload(lib), threads=4, version="0.0.0-test")
    ids = (G.C.c_int32 * 3)(7, 8, 9)
    cfg.comp_ids = ids
    cfg.ncomp = 3
    path = tmp_path / "sky.fits"
    wr = G.FitsWriter(path, cfg)
    wr.write(t.t, 0, 15000)
    wr.write(t.t, 15000, n)
    rows, nbytes = wr.close()
    assert nbytes == os.path.getsize(path)
    hdus = read_fits(path)
    assert len(hdus) == 3
    prim, cat, meta = hdus
    assert prim[0]["SIMPLE"] is True and prim[0]["NAXIS"] == 0 and prim[0]["BITPIX"] == 8
    assert cat[0]["XTENSION"] == "BINTABLE" and cat[0]["EXTNAME"] == "CATALOG"
    assert cat[1][:8] == ["XTENSION", "BITPIX", "NAXIS", "NAXIS1", "NAXIS2", "PCOUNT", "GCOUNT", "TFIELDS"]
    vis = t.arrays["hidden"][0, :n] == 0
    assert cat[0]["NAXIS2"] == rows == int(vis.sum())
    names = [cat[0]["TTYPE%d" % (i + 1)] for i in range(cat[0]["TFIELDS"])]
    order = RANKED + [(c, f) for _, c, f in photometry_columns(5)[0]]
    want_names = ["lb", "radec", "XYZ", "DM", "absSDSSr", "comp", "FeH", "vcyl", "pmradec", "Am", "AmInf"]
    want_names += [d.split("[")[0].split("{")[0] for d, _, _ in photometry_columns(5)[0]]
    assert names == want_names
    cols = fits_columns(cat[0], cat[2])
    for (name, fmt), fname in zip(order, want_names):
        a = t.arrays[name][:, :n][:, vis]
        got = cols[fname].T
        if name == "comp":
            a = np.array([7, 8, 9])[a]
        if fmt.endswith("d"):
            np.testing.assert_array_equal(got, a.astype(np.int32), err_msg=fname)
        else:
            g = got.astype(got.dtype.newbyteorder("="))
            u = np.uint32 if g.itemsize == 4 else np.uint64
            np.testing.assert_array_equal(g.view(u), a.astype(g.dtype).view(u), err_msg=fname)
    assert meta[0]["EXTNAME"] == "METADATA" and meta[0]["NAXIS2"] == 1 and meta[0]["TTYPE1"] == "HEADER"
    text_header = header(version="0.0.0-test")[2:-1]
    assert meta[2].rstrip(b"\0").decode() == text_header


def test_multiples_columns_in_the_text_header(tmp_path, lib):
    """With unresolved multiples the absolute magnitude loses its M1 alias and the
    system columns absSDSSrSys[2] and absSDSSrSysNcomp join the name-sorted
    columns (unresolvedMultiples_host.cpp:56-80, serialize_def order)."""
    n = 500
    t = random_table(n)
    A_ = t.arrays
    A_["absmagSys"][:, :n] = np.random.default_rng(3).uniform(-1, 16, (2, n))
    A_["absmagSys"][1, :n:3] = 99.999
    A_["absmagSysNcomp"][0, :n] = np.where(A_["absmagSys"][1, :n] < 99, 2, 1)
    w = workload(lib)
    w.multiples = W.multiples_config(lib)
    cfg = G.textout_config(w)
    path = tmp_path / "m.txt"
    wr = G.TextWriter(path, cfg)
    wr.write(t.t, 0, n)
    wr.close()
    lines = path.read_text().split("\n")
    defs = lines[0][2:].split()
    assert defs[4] == "absSDSSr{alias=absmag;band=SDSSr;}"
    assert defs[11:13] == ["absSDSSrSys[2]{class=magnitude;fieldNames=0:M1,1:M2;alias=absmagSys;band=SDSSr;}",
                           "absSDSSrSysNcomp{type=int;fmt=%1d;}"]
    vis = np.nonzero(A_["hidden"][0, :n] == 0)[0]
    first = lines[1].split(" ")
    r = vis[0]
    # lb 2, radec 2, XYZ 3, DM, absmag, comp, FeH, vcyl 3, pm 3, Am, AmInf = 19 fields, then the system columns
    sysf = [f for f in first if f != ""]
    assert printf("% 7.3f", float(A_["absmagSys"][0, r])).strip() == sysf[19]
    assert str(int(A_["absmagSysNcomp"][0, r])) == sysf[21]
