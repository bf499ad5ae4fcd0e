"""Synthetic catalog workloads with the shapes of galfast's configurations.

Everything here is host-side setup: footprints are pixelised by the native
library (gf_footprint_pixelize), the luminosity function, colour loci and
error curves are generated from closed-form expressions with fixed seeds.

    config 1  10x10 deg patch at the north galactic pole, 0.25 deg pixels, 15 < r < 21
    config 2  whole sky with |b| > 10 deg, 0.1 deg pixels, 14 < r < 22, 16M-star batches
    config 4  4096 pencil beams (batched form), per-request model variants and seeds
    config 5  served requests: Poisson arrivals, caps and lon/lat rectangles of 1-1000 deg^2,
              14 < r < U(20, 25), SDSS-like or LSST-like photometry
"""
import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi as A

D2R = math.pi / 180.0

# SDSS-like extinction-to-reddening ratios A_b / E(B-V) for u g r i z
SDSS_AE = np.array([5.155, 3.793, 2.751, 2.086, 1.479])
SDSS_M5 = np.array([22.5, 23.0, 23.0, 23.0, 22.2])
# LSST-like u g r i z y: the same ratios plus y, 5-sigma depths one magnitude deeper
LSST_AE = np.array([5.155, 3.793, 2.751, 2.086, 1.479, 1.263])
LSST_M5 = np.array([23.5, 24.0, 24.0, 24.0, 23.2, 22.9])


def lf_table():
    """Mr from 3 to 15 in 0.1 mag steps, log10 phi rising linearly from -3.5 to -2.0."""
    M = np.round(np.arange(121) * 0.1 + 3.0, 10)
    phi = 10.0 ** (-3.5 + 1.5 * (M - 3.0) / 12.0)
    return M.astype(np.float64), phi.astype(np.float64)


def color_coefficients(nbands=5, seed=20240611):
    """Cubic colour-magnitude relations c_i(Mr) = sum_k a_ik t^k, t = (Mr - 9)/6, for
    the colours band_i - band_(i+1); base colours of a main-sequence-like locus."""
    rng = np.random.default_rng(seed)
    a = rng.normal(0.0, 0.1, size=(nbands - 1, 4))
    base = np.array([1.2, 0.45, 0.18, 0.08, 0.05, 0.04][: nbands - 1])
    slope = np.array([0.6, 0.55, 0.35, 0.2, 0.15, 0.1][: nbands - 1])
    a[:, 0] += base
    a[:, 1] += slope
    return a


def photosys_rows(coef, Mr0=3.0, Mr1=15.0, dMr=0.01, FeHs=(-3.0, 1.0)):
    """A photosys-format table (Mr, FeH, c_1..c_n) sampled every dMr."""
    n = int(round((Mr1 - Mr0) / dMr)) + 1
    Mr = np.round(Mr0 + np.arange(n) * dMr, 10)
    t = (Mr - 9.0) / 6.0
    cols = np.stack([sum(c[k] * t ** k for k in range(4)) for c in coef], axis=1)
    rows = []
    for feh in FeHs:
        rows.append(np.column_stack([Mr, np.full(n, feh), cols]))
    return np.ascontiguousarray(np.concatenate(rows), dtype=np.float64)


def error_knots(m5):
    """sigma(m) = 0.005 + 0.04 * 10^(0.4 (m - m5)) tabulated from 0 to 40 in 0.01 steps,
    accumulating m exactly as os_modelPhotoErrors::construct (photometricErrors_host.cpp:236-240)."""
    mags = []
    m = 0.0
    while m < 40:
        mags.append(m)
        m += 0.01
    mags = np.array(mags)
    sig = np.stack([0.005 + 0.04 * 10.0 ** (0.4 * (mags - mm)) for mm in m5])
    return np.ascontiguousarray(np.tile(mags, (len(m5), 1))), np.ascontiguousarray(sig)


def galplane_frame(Rg=8000.0, z0=25.0):
    """The galplane rotation and translation as float32 (transform.cpp:122-135, 194-213)."""
    sina = -z0 / Rg
    cosa = math.sqrt(1 - sina * sina)
    M = np.array([-cosa, 0, sina, 0, -1, 0, sina, 0, cosa], dtype=np.float32)
    T = np.array([-Rg, 0.0, -0.0], dtype=np.float32)
    return M, T


def feh_config(Rg=8000.0, z0=25.0, thin=1, thick=2, halo=4):
    """os_FeH with the reference's default parameters (FeH_host.cpp:88-108): disk
    Gaussians A = (0.63, 0.37) (normalised), sigma 0.20, offsets 0 and 0.14, median
    -0.82 + 0.55 exp(-|Z| / 500 pc); halo N(-1.46, 0.30); galplane frame."""
    c = A.FehConfig()
    a0, a1 = 0.63, 0.37
    s_ = a0 + a1
    c.A[0], c.A[1] = a0 / s_, a1 / s_
    c.sigma[0], c.sigma[1], c.sigma[2] = 0.20, 0.20, 0.30
    c.offs[0], c.offs[1], c.offs[2] = 0.00, 0.14, -1.46
    c.Hmu, c.muInf, c.DeltaMu = 500.0, -0.82, 0.55
    c.comp_thin, c.comp_thick, c.comp_halo = thin, thick, halo
    M, T = galplane_frame(Rg, z0)
    for i in range(9):
        c.M[i] = float(M[i])
    for i in range(3):
        c.T[i] = float(T[i])
    return c


def gaussfeh_config(mean=(-0.6, -1.5), sigma=(0.2, 0.3), wt=(3.0, 1.0), comp_mask=0xFFFFFFFF):
    """os_GaussianFeH (GaussianFeH_host.cpp:78-104): a mixture of Gaussians with
    cumulative weights normalised to 1, in float as the reference stores them."""
    c = A.GaussFehConfig()
    c.ncomp = len(mean)
    acc = 0.0
    pc = []
    for w_ in wt:
        acc += w_
        pc.append(np.float32(acc))
    for i in range(c.ncomp):
        c.mean[i] = mean[i]
        c.sigma[i] = sigma[i]
        c.pcum[i] = float(np.float32(pc[i]) / np.float32(pc[-1]))
    c.comp_mask = comp_mask
    return c


def multiples_config(lib, algo=A.GF_MULT_LF_M2_GT_M1, comp_mask=0xFFFFFFFF, fraction=None, lf=None):
    """os_unresolvedMultiples through gf_multiples_build.  fraction: (M, p) knots of
    the binary fraction (None: 1 everywhere); lf: (M, phi) knots of the secondaries'
    luminosity function (None: flat).  The default synthetic choices: a binary
    fraction falling from 0.6 at M = 0 to 0.3 at M = 14, and a secondary LF rising
    towards faint magnitudes."""
    c = A.MultiplesConfig()
    dp = C.POINTER(C.c_double)

    def arr(v):
        a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
        return a, a.ctypes.data_as(dp)
    fm = fp = lm = lp = None
    nf = nl = 0
    keep = []
    if fraction is not None:
        (a, fm), (b, fp) = arr(fraction[0]), arr(fraction[1])
        keep += [a, b]
        nf = len(a)
    if lf is not None:
        (a, lm), (b, lp) = arr(lf[0]), arr(lf[1])
        keep += [a, b]
        nl = len(a)
    st = lib.gf_multiples_build(fm, fp, nf, lm, lp, nl, algo, comp_mask, C.byref(c))
    if st != 0:
        raise RuntimeError("gf_multiples_build failed (%d)" % st)
    return c


MULT_FRACTION = ([-2.0, 0.0, 6.0, 14.0, 20.0], [0.6, 0.6, 0.45, 0.3, 0.3])
MULT_LF = ([-2.0, 2.0, 6.0, 10.0, 14.0, 18.0], [0.2, 0.5, 1.0, 2.0, 3.0, 3.2])


def bond2010_config(disk_sigma=(35.0, 25.0, 20.0), halo_sigma=(140.0, 100.0, 95.0), Rg=8000.0, z0=25.0):
    """Bond et al. (2010) kinematics with constant dispersions (Bond2010_host.cpp:142-227 layout)."""
    cfg = A.Bond2010Config()
    cfg.comp_thin, cfg.comp_thick, cfg.comp_halo = 1, 2, 4
    fk = 3.0
    cfg.fk = fk / (1.0 + fk)

    def setv(arr, vals):
        for i in range(5):
            arr[i] = vals[i] if i < len(vals) else 0.0

    d1 = cfg.disk_1
    setv(d1.m[0], [0])                       # vR
    setv(d1.m[1], [-194, 19.2, 1.25])        # vPhi
    setv(d1.m[2], [0])                       # vZ
    setv(d1.ss[0], [disk_sigma[0]])          # sigmaR
    setv(d1.ss[1], [0])
    setv(d1.ss[2], [0])
    setv(d1.ss[3], [disk_sigma[1]])          # sigmaPhi1
    setv(d1.ss[4], [0])
    setv(d1.ss[5], [disk_sigma[2]])          # sigmaZ
    C.memmove(C.addressof(cfg.disk_2), C.addressof(cfg.disk_1), C.sizeof(A.VMoments))
    cfg.disk_2.m[1][0] += 34.0               # DeltavPhi
    setv(cfg.disk_2.ss[3], [disk_sigma[1]])  # sigmaPhi2
    h = cfg.halo
    for i in range(3):
        setv(h.m[i], [0])
    setv(h.ss[0], [halo_sigma[0]])           # HsigmaR
    setv(h.ss[1], [0])
    setv(h.ss[2], [0])
    setv(h.ss[3], [halo_sigma[2]])           # HsigmaTh
    setv(h.ss[4], [0])
    setv(h.ss[5], [halo_sigma[1]])           # HsigmaPhi
    M, T = galplane_frame(Rg, z0)
    for i in range(9):
        cfg.M[i] = float(M[i])
    for i in range(3):
        cfg.T[i] = float(T[i])
    return cfg


@dataclass
class Workload:
    """One catalog request: generator inputs plus the module chain."""
    sky: A.SkygenConfig
    pixels: np.ndarray                 # structured bytes of gf_pencil_beam
    npixels: int
    ammin: np.ndarray
    ext: A.Extinction
    models: List[A.ModelConfig]
    seed48: int
    nstreams: int
    capacity: int
    nbands: int
    foot: Optional[A.Footprint] = None
    feh: Optional[A.FixedFeHConfig] = None
    kin: Optional[A.Bond2010Config] = None
    phot: Optional[A.PhotometryConfig] = None
    perr: Optional[A.PhotoerrConfig] = None
    v2pm: Optional[A.Vel2pmConfig] = None
    gal2other: int = 0
    feh_ivezic: Optional[A.FehConfig] = None
    feh_gauss: Optional[A.GaussFehConfig] = None
    multiples: Optional[A.MultiplesConfig] = None
    keep: list = field(default_factory=list)   # keeps ctypes buffers alive

    def pixel_array(self):
        return (A.PencilBeam * self.npixels).from_buffer(self.pixels)

    def job(self, lib_types):
        """The gf_job structure (lib_types: galfast_b200.Job)."""
        j = lib_types()
        j.sky = self.sky
        j.pixels = C.cast(self.pixel_array(), C.POINTER(A.PencilBeam))
        j.npixels = self.npixels
        j.beam_ammin = self.ammin.ctypes.data_as(C.POINTER(C.c_float))
        j.ext = self.ext
        marr = (A.ModelConfig * len(self.models))(*self.models)
        self.keep.append(marr)
        j.models = C.cast(marr, C.POINTER(A.ModelConfig))
        j.nmodels = len(self.models)
        j.seed48 = self.seed48
        j.nstreams = self.nstreams
        j.capacity = self.capacity
        j.nbands = self.nbands
        for name in ("foot", "feh", "kin", "phot", "perr", "v2pm", "feh_ivezic", "feh_gauss", "multiples"):
            v = getattr(self, name)
            if v is not None:
                setattr(j, name, C.pointer(v))
        j.gal2other = self.gal2other
        return j


def _lambert_pair(lib):
    pr = (A.Lambert * 2)()
    lib.gf_lambert_init(C.c_double(90.0), C.c_double(90.0), C.byref(pr[0]))
    lib.gf_lambert_init(C.c_double(270.0), C.c_double(-90.0), C.byref(pr[1]))
    return pr


def pixelize(lib, foot, dx_deg, proj, ext):
    n = C.c_int64(0)
    st = lib.gf_footprint_pixelize(C.byref(foot), C.c_double(dx_deg), proj, C.byref(ext), None, None, C.c_int64(0), C.byref(n))
    if st != 0:
        raise RuntimeError("pixelisation failed")
    npix = n.value
    buf = bytearray(C.sizeof(A.PencilBeam) * max(npix, 1))
    pix = (A.PencilBeam * max(npix, 1)).from_buffer(buf)
    ammin = np.zeros(max(npix, 1), dtype=np.float32)
    st = lib.gf_footprint_pixelize(C.byref(foot), C.c_double(dx_deg), proj, C.byref(ext), pix,
                                   ammin.ctypes.data_as(C.POINTER(C.c_float)), C.c_int64(npix), C.byref(n))
    if st != 0:
        raise RuntimeError("pixelisation failed")
    return buf, npix, ammin


def _model(kind, comp, f, Rg, z0, lfM, lfphi, **kw):
    m = A.ModelConfig()
    m.type = kind
    m.comp = comp
    m.f = f
    m.frame = A.GF_FRAME_GALPLANE
    m.Rg, m.z0 = Rg, z0
    m.lf_M = lfM.ctypes.data_as(C.POINTER(C.c_double))
    m.lf_phi = lfphi.ctypes.data_as(C.POINTER(C.c_double))
    m.lf_n = len(lfM)
    m.ba = 1.0
    m.ca = 1.0
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def use_extinction_maps(lib, w, nxy=96, nz=24, dm_range=(4.0, 20.0), A0=0.06, D0=1500.0):
    """Switch a workload to 3-D extinction maps (GF_EXT_MAPS): for each hemisphere a
    grid over its Lambert plane (X, Y in [-2, 2], nxy texels a side, texel i at
    -2 + 4 i / (nxy - 1) as the reference's default map coordinates) and nz distance
    moduli over dm_range, holding A0 / sin|b| (capped at 20 A0) times
    (1 - exp(-D / D0)): extinction growing with distance, steeper towards the plane,
    zero outside the hemisphere's disk.  The per-beam rows come from
    gf_extinction_beam_minima."""
    xs = np.linspace(-2.0, 2.0, nxy)
    dms = np.linspace(dm_range[0], dm_range[1], nz)
    X, Y = np.meshgrid(xs, xs, indexing="xy")           # [y][x]
    r2 = X ** 2 + Y ** 2
    sinb = np.clip(1.0 - 0.5 * r2, 0.0, None)
    screen = np.where(r2 <= 2.0, A0 / np.maximum(sinb, 0.05), 0.0)
    D = 10.0 ** (0.2 * dms + 1.0)
    cube = (screen[None, :, :] * (1.0 - np.exp(-D / D0))[:, None, None]).astype(np.float32)   # [z][y][x]
    maps = []
    for h in range(2):
        a = np.ascontiguousarray(cube * (1.0 if h == 0 else 1.3), dtype=np.float32)
        e = A.ExtMap()
        e.A = a.ctypes.data_as(C.POINTER(C.c_float))
        e.n[0], e.n[1], e.n[2] = nxy, nxy, nz
        for ax, (lo, hi, n) in enumerate(((-2.0, 2.0, nxy), (-2.0, 2.0, nxy), (dm_range[0], dm_range[1], nz))):
            e.tc[ax][0] = lo
            e.tc[ax][1] = float(np.float32((n - 1) / (hi - lo)))
        maps.append((a, e))
    ext = A.Extinction()
    ext.kind = A.GF_EXT_MAPS
    ext.A0 = 0.0
    ext.north = C.pointer(maps[0][1])
    ext.south = C.pointer(maps[1][1])
    proj = (A.Lambert * 2)(w.sky.proj[0], w.sky.proj[1])
    nzc = C.c_int32(0)
    pix = w.pixel_array()
    st = lib.gf_extinction_beam_minima(C.byref(ext), proj, pix, w.npixels, None, C.byref(nzc))
    if st != 0:
        raise RuntimeError("gf_extinction_beam_minima failed")
    table = np.zeros(w.npixels * nzc.value, dtype=np.float32)
    st = lib.gf_extinction_beam_minima(C.byref(ext), proj, pix, w.npixels, table.ctypes.data_as(C.POINTER(C.c_float)),
                                       C.byref(nzc))
    if st != 0:
        raise RuntimeError("gf_extinction_beam_minima failed")
    w.ext = ext
    w.ammin = table
    w.keep += [maps, proj]
    return w


def density_cube_model(comp, f=1.0, Rg=8000.0, half=(20000.0, 20000.0, 5000.0), step=(500.0, 500.0, 250.0),
                       scale=(2600.0, 300.0), lf=None, keep=None):
    """A density-cube model (GF_MODEL_DENSITY_CUBE) whose grid samples a galactocentric
    exponential disk exp(-R/l - |z|/h) on a regular grid (x, y, z in [-half, half] with the
    given step, one empty texel of padding on each side as the reference's text loader
    adds, model_densityCube.cpp:108-150); texture coordinates map the first and last grid
    points to texels 1 and n - 2.  keep receives the arrays that must outlive the model."""
    l_, h_ = scale
    axes = [np.arange(-half[a], half[a] + 0.5 * step[a], step[a]) for a in range(3)]
    n = [len(ax) + 2 for ax in axes]
    cube = np.zeros((n[2], n[1], n[0]), dtype=np.float32)
    X, Y, Z = np.meshgrid(axes[0], axes[1], axes[2], indexing="ij")
    rho = np.exp(-np.sqrt(X ** 2 + Y ** 2) / l_ - np.abs(Z) / h_).astype(np.float32)
    cube[1:-1, 1:-1, 1:-1] = np.transpose(rho, (2, 1, 0))
    m = A.ModelConfig()
    m.type = A.GF_MODEL_DENSITY_CUBE
    m.comp = comp
    m.f = f
    m.Rg = Rg
    m.frame = A.GF_FRAME_GALPLANE
    m.cube = cube.ctypes.data_as(C.POINTER(C.c_float))
    for a in range(3):
        m.cube_n[a] = n[a]
        # texcoord_from_range(1, n - 2, first, last): (x0, 1/dx) with texel 1 at the first point
        x0, x1 = float(axes[a][0]), float(axes[a][-1])
        inv = np.float32((n[a] - 3) / (x1 - x0))
        m.cube_tc[a][0] = float(np.float32((-(n[a] - 2) * x0 + 1 * x1) / (1 - (n[a] - 2))))
        m.cube_tc[a][1] = float(inv)
    keep_ = [cube]
    if lf is not None:
        M_, phi = (np.ascontiguousarray(np.asarray(v, dtype=np.float64)) for v in lf)
        m.lf_M = M_.ctypes.data_as(C.POINTER(C.c_double))
        m.lf_phi = phi.ctypes.data_as(C.POINTER(C.c_double))
        m.lf_n = len(M_)
        keep_ += [M_, phi]
    if keep is not None:
        keep.extend(keep_)
    return m


_TABLES = {}


def _module_tables(lib, nbands, m5):
    """Photometry and photometric-error tables of one photometric system, built once
    per process and shared by every request that uses the system."""
    key = (nbands, m5)
    if key in _TABLES:
        return _TABLES[key]
    coef = color_coefficients(nbands)
    rows = photosys_rows(coef)
    nFeH = C.c_int32(0)
    nMr = C.c_int32(0)
    tcF = (C.c_float * 2)()
    tcM = (C.c_float * 2)()
    st = lib.gf_photometry_build(rows.ctypes.data_as(C.POINTER(C.c_double)), rows.shape[0], nbands - 1,
                                 C.c_double(0.01), C.c_double(0.01), None, None, C.byref(nFeH), C.byref(nMr), tcF, tcM)
    if st != 0:
        raise RuntimeError("photometry build failed")
    ncol = nbands - 1
    colors = np.zeros(ncol * nMr.value * nFeH.value, dtype=np.float32)
    eflags = np.zeros(ncol * nMr.value * nFeH.value, dtype=np.uint8)
    lib.gf_photometry_build(rows.ctypes.data_as(C.POINTER(C.c_double)), rows.shape[0], ncol,
                            C.c_double(0.01), C.c_double(0.01), colors.ctypes.data_as(C.POINTER(C.c_float)),
                            eflags.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(nFeH), C.byref(nMr), tcF, tcM)
    red = np.ones(A.GF_MAX_BANDS, dtype=np.float32)
    AE = SDSS_AE if nbands <= 5 else LSST_AE
    red[:nbands] = (AE[:nbands] / AE[2]).astype(np.float32)
    mk, sg = error_knots(list(m5))
    t = dict(rows=rows, colors=colors, eflags=eflags, nFeH=nFeH.value, nMr=nMr.value, tcF=(tcF[0], tcF[1]),
             tcM=(tcM[0], tcM[1]), red=red, mk=mk, sg=sg)
    _TABLES[key] = t
    return t


def build_workload(lib, *, foot, dx_deg, m0, m1, nthreads=7680, seed48=42, capacity=1 << 20,
                   thin_h=300.0, halo_q=0.64, with_modules=True, nbands=5, m5=SDSS_M5,
                   perr_seed=0x5eed, M0=3.0, M1=15.0, ext_E=0.02):
    proj = _lambert_pair(lib)
    ext = A.Extinction()
    ext.kind = A.GF_EXT_SCREEN_CSCB if ext_E > 0 else A.GF_EXT_NONE
    ext.A0 = float(SDSS_AE[2] * ext_E)
    pixbuf, npix, ammin = pixelize(lib, foot, dx_deg, proj, ext)
    sky = A.SkygenConfig()
    sky.m0, sky.m1, sky.dm = m0, m1, 0.05
    sky.M0, sky.M1 = M0, M1
    sky.dmin = sky.dmax = 0.0
    sky.nthreads = nthreads
    sky.nstars = 0.0
    sky.proj[0], sky.proj[1] = proj[0], proj[1]
    lfM, lfphi = lf_table()
    Rg, z0 = 8000.0, 25.0
    models = [
        _model(A.GF_MODEL_EXP_DISK, 0, 1.0, Rg, z0, lfM, lfphi, l=2600.0, h=thin_h),
        _model(A.GF_MODEL_EXP_DISK, 1, 0.12, Rg, z0, lfM, lfphi, l=3600.0, h=900.0),
        _model(A.GF_MODEL_POWER_LAW_ELLIPSOID, 2, 0.005, Rg, z0, lfM, lfphi, n=-2.77, ca=halo_q, ba=1.0),
    ]
    w = Workload(sky=sky, pixels=pixbuf, npixels=npix, ammin=ammin, ext=ext, models=models, seed48=seed48,
                 nstreams=65536, capacity=capacity, nbands=nbands if with_modules else 0, foot=foot)
    w.keep += [lfM, lfphi, proj]
    if not with_modules:
        return w
    feh = A.FixedFeHConfig()
    feh.FeH = 0.0
    feh.comp_mask = 0xFFFFFFFF
    w.feh = feh
    w.kin = bond2010_config(Rg=Rg, z0=z0)
    tabs = _module_tables(lib, nbands, tuple(float(x) for x in list(m5)[:nbands]))
    ph = A.PhotometryConfig()
    ph.nbands = nbands
    ph.bidx = 2
    for i in range(A.GF_MAX_BANDS):
        ph.reddening[i] = float(tabs["red"][i])
    ph.nFeH, ph.nMr = tabs["nFeH"], tabs["nMr"]
    ph.tcFeH[0], ph.tcFeH[1] = tabs["tcF"][0], tabs["tcF"][1]
    ph.tcMr[0], ph.tcMr[1] = tabs["tcM"][0], tabs["tcM"][1]
    ph.colors = tabs["colors"].ctypes.data_as(C.POINTER(C.c_float))
    ph.eflags = tabs["eflags"].ctypes.data_as(C.POINTER(C.c_uint8))
    ph.comp_mask = 0xFFFFFFFF
    w.phot = ph
    mk, sg = tabs["mk"], tabs["sg"]
    pe = A.PhotoerrConfig()
    pe.nbands = nbands
    pe.nknots = mk.shape[1]
    pe.mag = mk.ctypes.data_as(C.POINTER(C.c_double))
    pe.sigma = sg.ctypes.data_as(C.POINTER(C.c_double))
    pe.seed = perr_seed
    w.perr = pe
    v = A.Vel2pmConfig()
    v.coordsys = 1
    v.vLSR, v.u0, v.v0, v.w0, v.Rg = -220.0, -10.0, -5.3, 7.2, Rg
    w.v2pm = v
    w.gal2other = 1
    w.keep += [tabs]
    return w


def restrict_pixels(w, idx):
    """The workload `w` restricted to the pixels `idx` (per-beam extinction rows
    renumbered); the grid, models, seeds and module chain are unchanged."""
    import copy
    sub = copy.copy(w)
    pix = np.frombuffer(w.pixels, dtype=np.uint8).reshape(w.npixels, -1)[idx].copy()
    pb = (A.PencilBeam * len(idx)).from_buffer(pix)
    for k in range(len(idx)):
        pb[k].extIdx = k
    sub.pixels = bytearray(pix.tobytes())
    sub.npixels = len(idx)
    sub.ammin = np.ascontiguousarray(w.ammin[idx])
    sub.keep = list(w.keep)
    return sub


def config1(lib, **kw):
    """10x10 deg patch centred on the north galactic pole, 0.25 deg pixels, 15 < r < 21."""
    half = 5.0 * D2R
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    return build_workload(lib, foot=foot, dx_deg=0.25, m0=15.0, m1=21.0, **kw)


def config2(lib, **kw):
    """The whole sky with |b| > 10 deg, 0.1 deg pixels, 14 < r < 22."""
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LATCUT
    foot.a = 10.0
    kw.setdefault("capacity", 1 << 24)
    return build_workload(lib, foot=foot, dx_deg=0.1, m0=14.0, m1=22.0, **kw)


def cap_footprint(l_deg, b_deg, r_deg):
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_CAP
    foot.a, foot.b, foot.c = l_deg, b_deg, r_deg
    return foot


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def config4_requests(n=4096, seed=1234567):
    """Parameters of the batched form: pencil beams with |b| > 5 deg, radius log-uniform in
    [0.5, 5] deg, r_max uniform in [19, 24], thin-disk h in [250, 350] pc, halo q in [0.55, 0.75]."""
    out = []
    for r in range(n):
        s = splitmix64(seed + r)
        g = np.random.default_rng(s)
        while True:
            z = g.uniform(-1, 1)
            b = math.degrees(math.asin(z))
            if abs(b) > 5.0:
                break
        l = g.uniform(0, 360)
        rad = math.exp(g.uniform(math.log(0.5), math.log(5.0)))
        rmax = g.uniform(19, 24)
        h = g.uniform(250, 350)
        q = g.uniform(0.55, 0.75)
        out.append(dict(l=l, b=b, r=rad, rmax=rmax, h=h, q=q, seed48=s & 0xFFFFFFFF, perr_seed=splitmix64(s)))
    return out


def config4_workload(lib, req, **kw):
    foot = cap_footprint(req["l"], req["b"], req["r"])
    kw.setdefault("perr_seed", req.get("perr_seed", 0x5eed))
    return build_workload(lib, foot=foot, dx_deg=0.1, m0=14.0, m1=req["rmax"], thin_h=req["h"],
                          halo_q=req["q"], seed48=req["seed48"], **kw)


def config4_workloads(lib, reqs, threads=None, **kw):
    """config4_workload for many requests on a thread pool (the pixelisation is
    native code and runs without the interpreter lock)."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    _module_tables(lib, kw.get("nbands", 5), tuple(float(x) for x in list(kw.get("m5", SDSS_M5))[:kw.get("nbands", 5)]))
    n = threads or min(32, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=n) as ex:
        return list(ex.map(lambda r: config4_workload(lib, r, **kw), reqs))


def regions_footprint(regions):
    """GF_FOOT_REGIONS: the union of up to 8 regions, each a dict
    type ("beam" or "rect"), coordsys ("gal" or "equ"), the four values
    (beam: lon, lat, r, rhole; rect: lon0, lon1, lat0, lat1; degrees) and bmin."""
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_REGIONS
    foot.nregions = len(regions)
    for i, r in enumerate(regions):
        g = foot.regions[i]
        g.type = A.GF_REGION_BEAM if r["type"] == "beam" else A.GF_REGION_RECT
        g.coordsys = A.GF_COORD_EQU if r.get("coordsys", "gal") == "equ" else A.GF_COORD_GAL
        g.a, g.b, g.c, g.d = (float(v) for v in r["v"])
        g.bmin = float(r.get("bmin", 0.0))
    return foot


def lb_rect_footprint(l0, l1, b0, b1):
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LB_RECT
    foot.a, foot.b, foot.c, foot.d = l0 % 360.0, l1 % 360.0, b0, b1
    return foot


def config5_requests(n, rate, seed=99, area=(1.0, 1000.0), rmax=(20.0, 25.0)):
    """The served request stream: arrival times of a Poisson process of the given rate
    (requests/s), footprint areas log-uniform in `area` deg^2, caps or galactic
    lon/lat rectangles (half each) at random centres with |b| > 10 deg, depth r_max
    uniform in `rmax`, half SDSS-like ugriz and half LSST-like ugrizy, own seeds."""
    g = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += g.exponential(1.0 / rate)
        while True:
            z = g.uniform(-1, 1)
            b = math.degrees(math.asin(z))
            if abs(b) > 10.0:
                break
        l = g.uniform(0, 360)
        A_deg2 = math.exp(g.uniform(math.log(area[0]), math.log(area[1])))
        a_sr = A_deg2 * D2R * D2R
        if g.uniform() < 0.5:
            shape = dict(kind="cap", r=math.degrees(math.acos(1.0 - a_sr / (2 * math.pi))))
        else:
            db = math.sqrt(A_deg2)
            b0 = max(-90.0, b - 0.5 * db)
            b1 = min(90.0, b + 0.5 * db)
            dl = math.degrees(a_sr / (math.sin(math.radians(b1)) - math.sin(math.radians(b0))))
            shape = dict(kind="rect", l0=l - 0.5 * min(dl, 359.0), l1=l + 0.5 * min(dl, 359.0), b0=b0, b1=b1)
        s = splitmix64(seed * 1000003 + k)
        out.append(dict(t=t, l=l, b=b, area=A_deg2, rmax=g.uniform(*rmax), lsst=bool(g.uniform() < 0.5),
                        seed48=s & 0xFFFFFFFF, perr_seed=splitmix64(s), **shape))
    return out


def config5_workload(lib, req, capacity=1 << 24, **kw):
    if req["kind"] == "cap":
        foot = cap_footprint(req["l"], req["b"], req["r"])
    else:
        foot = lb_rect_footprint(req["l0"], req["l1"], req["b0"], req["b1"])
    if req["lsst"]:
        kw.setdefault("nbands", 6)
        kw.setdefault("m5", LSST_M5)
    return build_workload(lib, foot=foot, dx_deg=0.1, m0=14.0, m1=req["rmax"], seed48=req["seed48"],
                          perr_seed=req["perr_seed"], capacity=capacity, **kw)


def config5_workloads(lib, reqs, threads=None, **kw):
    import os
    from concurrent.futures import ThreadPoolExecutor
    for nb, m5 in ((5, SDSS_M5), (6, LSST_M5)):
        _module_tables(lib, nb, tuple(float(x) for x in m5))
    n = threads or min(32, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=n) as ex:
        return list(ex.map(lambda r: config5_workload(lib, r, **kw), reqs))
