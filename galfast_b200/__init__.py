"""galfast_b200 -- B200-native galfast catalog hot path (skygen + photometry +
kinematics + proper motions) behind a C ABI (include/galfast_b200.h).

The Python layer mirrors the reference's module interface for tests and
benchmarks: a Skygen object plays the part of the skygen source module
(integrateCounts / drawSources, src/skygen/skygen.h:47-60) and the module
functions the osink::process of each postprocessing module.  All compute runs
in the sm_100a library; there is no CPU fallback: importing this package on a
machine without the built library raises.
"""
import ctypes as C
import os

import numpy as np

from . import _abi as A
from ._abi import (PencilBeam, Lambert, SkygenConfig, ModelConfig, Extinction, Footprint, Table,
                   FixedFeHConfig, Bond2010Config, PhotometryConfig, PhotoerrConfig, Vel2pmConfig, ModelInfo)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_lib", "libgalfast_b200.so")


class GalfastError(RuntimeError):
    pass


class Job(C.Structure):
    _fields_ = [("sky", SkygenConfig), ("pixels", C.POINTER(PencilBeam)), ("npixels", C.c_int32),
                ("beam_ammin", C.POINTER(C.c_float)), ("ext", Extinction),
                ("models", C.POINTER(ModelConfig)), ("nmodels", C.c_int32),
                ("seed48", C.c_uint32), ("nstreams", C.c_int32), ("capacity", C.c_int64), ("nbands", C.c_int32),
                ("foot", C.POINTER(Footprint)), ("feh", C.POINTER(FixedFeHConfig)),
                ("kin", C.POINTER(Bond2010Config)), ("phot", C.POINTER(PhotometryConfig)),
                ("perr", C.POINTER(PhotoerrConfig)), ("v2pm", C.POINTER(Vel2pmConfig)), ("gal2other", C.c_int32),
                ("feh_ivezic", C.POINTER(A.FehConfig)), ("feh_gauss", C.POINTER(A.GaussFehConfig)),
                ("multiples", C.POINTER(A.MultiplesConfig))]


class CatalogStats(C.Structure):
    _fields_ = [("expected", C.c_double * 32), ("expected_covered", C.c_double * 32),
                ("generated", C.c_int64 * 32), ("stored", C.c_int64 * 32), ("batches", C.c_int32),
                ("norm", C.c_float)]


class ServerInfo(C.Structure):
    _fields_ = [("runs", C.c_int64), ("completed", C.c_int64), ("deferred", C.c_int64), ("peak_reserved", C.c_int64),
                ("peak_running", C.c_int32), ("queued", C.c_int32), ("active", C.c_int32), ("pad", C.c_int32)]


BatchCallback = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.POINTER(Table), C.c_int64)
ServerRows = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.POINTER(Table), C.c_int64, C.c_int64)
ServerDone = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_int32, C.POINTER(CatalogStats))
MultiCallback = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.POINTER(Table), C.POINTER(C.c_int64), C.POINTER(C.c_int64))
MultiHostCallback = MultiCallback      # the same signature; the table is in host memory

_lib = None


def lib():
    """The native library; raises GalfastError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise GalfastError("libgalfast_b200.so is not built: run `python -m galfast_b200.build`")
        L = C.CDLL(LIBPATH)
        vp = C.c_void_p
        L.gf_last_error.restype = C.c_char_p
        L.gf_ctx_create.argtypes = [C.c_int, C.POINTER(vp)]
        L.gf_ctx_destroy.argtypes = [vp]
        L.gf_ctx_sync.argtypes = [vp]
        L.gf_ctx_mark.argtypes = [vp, C.c_int32]
        L.gf_ctx_elapsed.argtypes = [vp, C.c_int32, C.c_int32, C.POINTER(C.c_float)]
        L.gf_launch_count.restype = C.c_int64
        L.gf_profile_enable.argtypes = [vp, C.c_int32]
        L.gf_profile_read.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.gf_rng_init.argtypes = [vp, C.c_uint32, C.c_int32]
        L.gf_rng_seed48_from_cli_seed.argtypes = [C.c_uint64]
        L.gf_rng_seed48_from_cli_seed.restype = C.c_uint32
        L.gf_rng_get_state.argtypes = [vp, vp, C.c_int32]
        L.gf_rng_set_state.argtypes = [vp, vp, C.c_int32]
        L.gf_rng_poisson.argtypes = [vp, vp, vp, C.c_int32, vp]
        L.gf_skygen_create.argtypes = [vp, C.POINTER(SkygenConfig), C.POINTER(PencilBeam), C.c_int32,
                                       C.POINTER(C.c_float), C.POINTER(Extinction), C.POINTER(ModelConfig),
                                       C.c_int32, C.POINTER(vp)]
        L.gf_skygen_destroy.argtypes = [vp]
        L.gf_skygen_model_info_get.argtypes = [vp, C.c_int32, C.POINTER(ModelInfo)]
        L.gf_skygen_model_lf_get.argtypes = [vp, C.c_int32, C.POINTER(C.c_float)]
        L.gf_skygen_integrate.argtypes = [vp, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        L.gf_skygen_set_norm.argtypes = [vp, C.c_int32, C.c_float]
        L.gf_skygen_draw.argtypes = [vp, C.c_int32, C.POINTER(Table), C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
        L.gf_table_alloc.argtypes = [vp, C.c_int64, C.c_int32, C.POINTER(Table)]
        L.gf_table_free.argtypes = [vp, C.POINTER(Table)]
        L.gf_table_download.argtypes = [vp, C.POINTER(Table), C.POINTER(Table)]
        L.gf_module_clipper.argtypes = [vp, C.POINTER(Footprint), C.POINTER(Lambert), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_fixedfeh.argtypes = [vp, C.POINTER(FixedFeHConfig), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_bond2010.argtypes = [vp, C.POINTER(Bond2010Config), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_feh.argtypes = [vp, C.POINTER(A.FehConfig), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_gaussfeh.argtypes = [vp, C.POINTER(A.GaussFehConfig), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_multiples.argtypes = [vp, C.POINTER(A.MultiplesConfig), C.POINTER(Table), C.c_int64, C.c_int64]
        dp = C.POINTER(C.c_double)
        L.gf_multiples_build.argtypes = [dp, dp, C.c_int32, dp, dp, C.c_int32, C.c_int32, C.c_uint32,
                                         C.POINTER(A.MultiplesConfig)]
        L.gf_photometry_create.argtypes = [vp, C.POINTER(PhotometryConfig), C.POINTER(vp)]
        L.gf_photometry_destroy.argtypes = [vp]
        L.gf_module_photometry.argtypes = [vp, vp, C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_photoerr_create.argtypes = [vp, C.POINTER(PhotoerrConfig), C.POINTER(vp)]
        L.gf_photoerr_destroy.argtypes = [vp]
        L.gf_module_photoerrors.argtypes = [vp, vp, C.c_int64, C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_vel2pm.argtypes = [vp, C.POINTER(Vel2pmConfig), C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_module_gal2other.argtypes = [vp, C.c_int32, C.POINTER(Table), C.c_int64, C.c_int64]
        L.gf_catalog_run.argtypes = [vp, C.POINTER(Job), BatchCallback, vp, C.POINTER(CatalogStats)]
        L.gf_catalog_run_multi.argtypes = [vp, C.POINTER(Job), C.c_int32, MultiCallback, vp, C.POINTER(CatalogStats)]
        L.gf_catalog_run_multi_host.argtypes = [vp, C.POINTER(Job), C.c_int32, C.c_int64, MultiHostCallback, vp,
                                                C.POINTER(CatalogStats)]
        L.gf_multi_set_memory_budget.argtypes = [vp, C.c_int64]
        L.gf_multi_set_host_columns.argtypes = [vp, C.c_uint32]
        L.gf_multi_set_admission.argtypes = [vp, C.c_double]
        L.gf_debug_fail_allocations.argtypes = [C.c_int64, C.c_int64]
        L.gf_textout_open.argtypes = [C.c_char_p, vp, C.POINTER(vp)]
        L.gf_fitsout_open.argtypes = [C.c_char_p, vp, C.POINTER(vp)]
        L.gf_textout_write.argtypes = [vp, vp, C.c_int64, C.c_int64]
        L.gf_textout_close.argtypes = [vp, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.gf_textout_multi_sink.argtypes = [vp, C.c_int32, vp, vp, vp]
        L.gf_tuning_get.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32)]
        L.gf_tuning_set.argtypes = [vp, C.c_int32, C.c_int32]
        L.gf_table_download_rows.argtypes = [vp, C.POINTER(Table), C.c_int64, C.c_int64, C.POINTER(Table)]
        L.gf_server_create.argtypes = [C.c_int32, C.c_int32, C.c_int64, C.c_int32, C.POINTER(vp)]
        L.gf_server_submit.argtypes = [vp, C.POINTER(Job), ServerRows, ServerDone, vp, C.POINTER(C.c_int64)]
        L.gf_server_drain.argtypes = [vp]
        L.gf_server_get_info.argtypes = [vp, C.POINTER(ServerInfo)]
        L.gf_server_pause.argtypes = [vp, C.c_int32]
        L.gf_server_destroy.argtypes = [vp]
        L.gf_skygen_precision.argtypes = [vp, C.c_int32, C.POINTER(A.PrecisionReport), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.gf_lambert_init.argtypes = [C.c_double, C.c_double, C.POINTER(Lambert)]
        L.gf_footprint_pixelize.argtypes = [C.POINTER(Footprint), C.c_double, C.POINTER(Lambert),
                                            C.POINTER(Extinction), C.POINTER(PencilBeam), C.POINTER(C.c_float),
                                            C.c_int64, C.POINTER(C.c_int64)]
        L.gf_extinction_beam_minima.argtypes = [C.POINTER(Extinction), C.POINTER(Lambert), C.POINTER(PencilBeam), C.c_int32,
                                                C.POINTER(C.c_float), C.POINTER(C.c_int32)]
        L.gf_photometry_build.argtypes = [C.POINTER(C.c_double), C.c_int32, C.c_int32, C.c_double, C.c_double,
                                          C.POINTER(C.c_float), C.POINTER(C.c_uint8), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.gf_multipliers.argtypes = [C.POINTER(C.c_uint32), C.c_int32]
        L.gf_rng_seed_host.argtypes = [C.c_uint32, C.c_int32, C.POINTER(C.c_uint32)]
        L.gf_mt19937_outputs.argtypes = [C.c_uint32, C.c_int, C.POINTER(C.c_uint32)]
        L.gf_skygen_setup_host.argtypes = [C.POINTER(SkygenConfig), C.c_int32, C.POINTER(ModelConfig), C.c_int32,
                                           C.POINTER(ModelInfo), C.POINTER(C.c_float)]
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise GalfastError("galfast_b200 error %d: %s" % (status, lib().gf_last_error().decode()))


# ---------------------------------------------------------------------------
# host tables (numpy views with the library's column layout)
# ---------------------------------------------------------------------------
COLUMNS = [  # name, dtype, components (or "bands")
    ("lb", np.float64, 2), ("projIdx", np.int32, 1), ("projXY", np.float32, 2), ("DM", np.float32, 1),
    ("absmag", np.float32, 1), ("XYZ", np.float32, 3), ("comp", np.int32, 1), ("Am", np.float32, 1),
    ("AmInf", np.float32, 1), ("hidden", np.int32, 1), ("FeH", np.float32, 1), ("vcyl", np.float32, 3),
    ("mags", np.float32, "bands"), ("photoflags", np.int32, 1), ("obsmags", np.float32, "bands"),
    ("pm", np.float32, 3), ("radec", np.float64, 2), ("FeH_comp", np.int32, 1),
    ("absmagSys", np.float32, 2), ("absmagSysNcomp", np.int32, 1),
]
PROFILE_PHASES = ["integrate", "draw_window", "draw_rerun", "place", "sort", "clipper", "fixedfeh", "bond2010",
                  "photometry", "photoerrors", "vel2pm", "gal2other", "slot_density", "expand", "batch_draw",
                  "setup", "plain_requests"]
SKYGEN_COLUMNS = ["lb", "projIdx", "projXY", "DM", "absmag", "XYZ", "comp", "Am", "AmInf", "hidden"]
# column bits of gf_multi_set_host_columns (GF_COL_*): bit i is COLUMNS[i]
COL = {name: 1 << i for i, (name, _, _) in enumerate(COLUMNS)}
COL_ALL = (1 << len(COLUMNS)) - 1
COL_CATALOG = sum(COL[n] for n in ("radec", "DM", "absmag", "mags", "obsmags", "vcyl", "pm"))


class HostTable:
    """A gf_table in host memory backed by numpy arrays; vector columns are (ncomp, capacity)."""

    def __init__(self, capacity, nbands):
        self.capacity = int(capacity)
        self.nbands = int(nbands)
        self.arrays = {}
        self.t = Table()
        self.t.capacity = self.capacity
        self.t.size = 0
        self.t.nbands = self.nbands
        for name, dt, ncomp in COLUMNS:
            k = self.nbands if ncomp == "bands" else ncomp
            if k == 0:
                setattr(self.t, name, None)
                continue
            a = np.zeros((k, self.capacity), dtype=dt)
            self.arrays[name] = a
            setattr(self.t, name, a.ctypes.data)

    @property
    def size(self):
        return int(self.t.size)

    def col(self, name):
        a = self.arrays[name]
        return a[0, : self.size] if a.shape[0] == 1 else a[:, : self.size]

    def as_dict(self, names=None):
        return {n: np.array(self.col(n)) for n in (names or self.arrays.keys())}

    def rows(self, a, b, names=None):
        """Copies of rows [a, b) of every column (vector columns as (ncomp, b - a))."""
        out = {}
        for n in (names or self.arrays.keys()):
            x = self.arrays[n]
            out[n] = np.array(x[0, a:b] if x.shape[0] == 1 else x[:, a:b])
        return out


# ---------------------------------------------------------------------------
# context, generator, modules
# ---------------------------------------------------------------------------
class Context:
    """A CUDA context: one device, one stream, the persistent RNG streams."""

    def __init__(self, device=0):
        self.h = C.c_void_p()
        check(lib().gf_ctx_create(device, C.byref(self.h)))
        self.nstreams = 0

    def close(self):
        if self.h:
            lib().gf_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(lib().gf_ctx_sync(self.h))

    def mark(self, slot):
        """Record device event `slot` on the library's stream."""
        check(lib().gf_ctx_mark(self.h, slot))

    def profile(self, on=True):
        check(lib().gf_profile_enable(self.h, 1 if on else 0))

    def profile_read(self):
        """{phase: (milliseconds, launches)} accumulated since the last read."""
        ms = (C.c_double * len(PROFILE_PHASES))()
        n = (C.c_int64 * len(PROFILE_PHASES))()
        check(lib().gf_profile_read(self.h, ms, n))
        return {PROFILE_PHASES[i]: (ms[i], n[i]) for i in range(len(PROFILE_PHASES)) if n[i]}

    def elapsed_ms(self, a, b):
        ms = C.c_float()
        check(lib().gf_ctx_elapsed(self.h, a, b, C.byref(ms)))
        return ms.value

    def tuning(self):
        """{model kind: warps per CTA of the batched draw} (0 = not tuned yet)."""
        out = {}
        for k in (A.GF_MODEL_EXP_DISK, A.GF_MODEL_POWER_LAW_ELLIPSOID):
            w = C.c_int32()
            check(lib().gf_tuning_get(self.h, k, C.byref(w)))
            out[k] = w.value
        return out

    def set_tuning(self, model_kind, warps):
        check(lib().gf_tuning_set(self.h, model_kind, warps))

    def set_host_columns(self, mask):
        """Columns gf_catalog_run_multi_host copies to host memory (COL bits)."""
        check(lib().gf_multi_set_host_columns(self.h, int(mask)))

    def set_admission(self, sigmas):
        """gf_multi_set_admission: batched if expected + sigmas sqrt(expected) + 1024 < capacity."""
        check(lib().gf_multi_set_admission(self.h, float(sigmas)))

    def set_multi_budget(self, nbytes):
        """Device bytes per chunk of gf_catalog_run_multi (0 = 60% of free memory)."""
        check(lib().gf_multi_set_memory_budget(self.h, int(nbytes)))

    def rng_init(self, seed48, nstreams=65536):
        check(lib().gf_rng_init(self.h, seed48, nstreams))
        self.nstreams = nstreams + (-nstreams) % 64

    def rng_state(self, nstreams=None):
        """The [3][nstreams] stream states (nstreams: as seeded by rng_init, or given
        for streams a catalog run seeded)."""
        n = self.nstreams if nstreams is None else int(nstreams)
        s = np.zeros(3 * n, dtype=np.uint32)
        check(lib().gf_rng_get_state(self.h, s.ctypes.data, n))
        return s

    def set_rng_state(self, s):
        s = np.ascontiguousarray(s, dtype=np.uint32)
        check(lib().gf_rng_set_state(self.h, s.ctypes.data, self.nstreams))


class DeviceTable:
    def __init__(self, ctx, capacity, nbands):
        self.ctx = ctx
        self.t = Table()
        check(lib().gf_table_alloc(ctx.h, capacity, nbands, C.byref(self.t)))

    @property
    def size(self):
        return int(self.t.size)

    def download(self, host=None):
        host = host or HostTable(self.t.capacity, self.t.nbands)
        check(lib().gf_table_download(self.ctx.h, C.byref(self.t), C.byref(host.t)))
        return host

    def free(self):
        lib().gf_table_free(self.ctx.h, C.byref(self.t))


class Skygen:
    """The skygen source module for one workload (os_skygen + one skygenHost per model)."""

    def __init__(self, ctx, w):
        self.ctx = ctx
        self.w = w
        self.h = C.c_void_p()
        marr = (ModelConfig * len(w.models))(*w.models)
        self._marr = marr
        check(lib().gf_skygen_create(ctx.h, C.byref(w.sky), C.cast(w.pixel_array(), C.POINTER(PencilBeam)),
                                     w.npixels, w.ammin.ctypes.data_as(C.POINTER(C.c_float)), C.byref(w.ext),
                                     C.cast(marr, C.POINTER(ModelConfig)), len(w.models), C.byref(self.h)))

    def close(self):
        if self.h:
            lib().gf_skygen_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self, model):
        i = ModelInfo()
        check(lib().gf_skygen_model_info_get(self.h, model, C.byref(i)))
        return i

    def lf(self, model):
        n = self.info(model).lf_n
        a = np.zeros(n, dtype=np.float32)
        check(lib().gf_skygen_model_lf_get(self.h, model, a.ctypes.data_as(C.POINTER(C.c_float))))
        return a

    def integrate_counts(self, model, per_pixel=False):
        e = C.c_double()
        ec = C.c_double()
        pp = np.zeros(self.w.npixels) if per_pixel else None
        check(lib().gf_skygen_integrate(self.h, model, C.byref(e), C.byref(ec),
                                        pp.ctypes.data_as(C.POINTER(C.c_double)) if pp is not None else None))
        return e.value, ec.value, pp

    def precision(self, model):
        """gf_skygen_precision: (report, per-pixel FP32 sums, per-pixel FP64 sums, FP64 counts per DM row)."""
        i = self.info(model)
        rep = A.PrecisionReport()
        p32 = np.zeros(self.w.npixels)
        p64 = np.zeros(self.w.npixels)
        hist = np.zeros(i.nm + i.nM - 1)
        dp = C.POINTER(C.c_double)
        check(lib().gf_skygen_precision(self.h, model, C.byref(rep), p32.ctypes.data_as(dp), p64.ctypes.data_as(dp),
                                        hist.ctypes.data_as(dp)))
        return rep, p32, p64, hist

    def set_density_norm(self, model, norm):
        check(lib().gf_skygen_set_norm(self.h, model, norm))

    def draw_sources(self, model, table):
        n = C.c_int64()
        d = C.c_int32()
        check(lib().gf_skygen_draw(self.h, model, C.byref(table.t), C.byref(n), C.byref(d)))
        return n.value, bool(d.value)


def run_catalog(ctx, w, sink=None):
    """gf_catalog_run: os_skygen::run followed by the module chain for each batch.
    sink(model, HostTable, row_offset) receives every batch in host memory."""
    job = w.job(Job)
    stats = CatalogStats()
    host_cache = {}

    def cb(user, model, tptr, row_offset):
        if sink is None:
            return 0
        t = tptr.contents
        key = (t.capacity, t.nbands)
        if key not in host_cache:
            host_cache[key] = HostTable(t.capacity, t.nbands)
        h = host_cache[key]
        st = lib().gf_table_download(ctx.h, tptr, C.byref(h.t))
        if st != 0:
            return 1
        return 1 if sink(model, h, row_offset) else 0

    ccb = BatchCallback(cb)
    check(lib().gf_catalog_run(ctx.h, C.byref(job), ccb, None, C.byref(stats)))
    return stats


def run_catalog_multi(ctx, workloads, sink=None, device_sink=None):
    """gf_catalog_run_multi: the catalogs of many requests generated together.

    sink(job, model, rows) receives each request's rows of each model in host
    memory as a dict of column arrays (one download per model pass, then a split
    by request);
    device_sink(model, table_ptr, row_begin, row_count) sees the device table
    instead.  Returns the per-request CatalogStats."""
    n = len(workloads)
    jobs = (Job * n)(*[w.job(Job) for w in workloads])
    stats = (CatalogStats * n)()
    cache = {}

    def cb(user, model, tptr, rb, rc):
        if device_sink is not None:
            if device_sink(model, tptr, rb, rc):
                return 1
        if sink is None:
            return 0
        t = tptr.contents
        key = (t.capacity, t.nbands)
        if key not in cache:
            cache[key] = HostTable(t.capacity, t.nbands)
        h = cache[key]
        if lib().gf_table_download(ctx.h, tptr, C.byref(h.t)) != 0:
            return 1
        for j in range(n):
            if rc[j] > 0:
                if sink(j, model, h.rows(rb[j], rb[j] + rc[j])):
                    return 1
        return 0

    ccb = MultiCallback(cb)
    check(lib().gf_catalog_run_multi(ctx.h, jobs, n, ccb, None, stats))
    return list(stats)


def table_rows(t, a, b, names=None):
    """Copies of rows [a, b) of a gf_table in host memory (vector columns (ncomp, rows))."""
    out = {}
    cap = int(t.capacity)
    for name, dt, ncomp in COLUMNS:
        if names is not None and name not in names:
            continue
        k = int(t.nbands) if ncomp == "bands" else ncomp
        ptr = getattr(t, name)
        if not ptr or k == 0:
            continue
        arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), shape=(k * cap,))
        arr = arr.reshape(k, cap)[:, a:b].copy()
        out[name] = arr[0] if ncomp == 1 else arr
    return out


def run_catalog_multi_host(ctx, workloads, sink, piece_rows=0):
    """gf_catalog_run_multi_host: the catalogs of many requests generated together,
    their rows copied to page-locked host memory while the device works on.

    sink(job, model, rows) receives copies of a request's rows in one delivered
    piece (a dict of column arrays); a request's rows of a model may come in
    several pieces, in order.  Called from a CUDA driver thread.  Returns the
    per-request CatalogStats."""
    n = len(workloads)
    jobs = (Job * n)(*[w.job(Job) for w in workloads])
    stats = (CatalogStats * n)()

    def cb(user, model, tptr, rb, rc):
        try:
            t = tptr.contents
            for j in range(n):
                if rc[j] > 0 and sink(j, model, table_rows(t, rb[j], rb[j] + rc[j])):
                    return 1
            return 0
        except Exception:
            return 1

    ccb = MultiHostCallback(cb)
    check(lib().gf_catalog_run_multi_host(ctx.h, jobs, n, int(piece_rows), ccb, None, stats))
    return list(stats)


class Server:
    """gf_server: continuous batching of catalog requests on one device.

    submit(w) queues a workload (the server copies the job, so nothing of it has
    to be kept here); keep_rows=True keeps each request's rows in host
    memory (a dict per model of column arrays), a callable keep_rows(request id)
    those of the requests it accepts.  Completion wall-clock times are
    recorded for latency.  Callbacks run on the server's worker threads."""

    def __init__(self, device=0, workers=2, memory_budget=150 * 2 ** 30, max_batch=512, keep_rows=False):
        import threading
        import time as _time
        self._time = _time
        self.h = C.c_void_p()
        check(lib().gf_server_create(device, workers, int(memory_budget), max_batch, C.byref(self.h)))
        self.keep_rows = keep_rows
        self.lock = threading.Lock()
        self.submitted, self.finished, self.status, self.stats, self.rows = {}, {}, {}, {}, {}
        self._stage = {}

        def on_rows(user, rid, model, wctx, tptr, begin, count):
            if not (self.keep_rows(rid) if callable(self.keep_rows) else self.keep_rows):
                return 0
            t = tptr.contents
            h = HostTable(max(int(count), 1), t.nbands)
            if lib().gf_table_download_rows(wctx, tptr, begin, begin + count, C.byref(h.t)) != 0:
                return 1
            with self.lock:
                self.rows.setdefault(rid, {}).setdefault(model, []).append(h.rows(0, int(count)))
            return 0

        def on_done(user, rid, status, stats):
            t = self._time.perf_counter()
            st = CatalogStats()
            C.memmove(C.byref(st), stats, C.sizeof(CatalogStats))
            with self.lock:
                self.finished[rid] = t
                self.status[rid] = status
                self.stats[rid] = st

        self._rows_cb = ServerRows(on_rows)
        self._done_cb = ServerDone(on_done)

    def submit(self, w):
        job = w.job(Job)
        rid = C.c_int64()
        t = self._time.perf_counter()
        check(lib().gf_server_submit(self.h, C.byref(job), self._rows_cb, self._done_cb, None, C.byref(rid)))
        with self.lock:
            self.submitted[rid.value] = t
        return rid.value

    def drain(self):
        check(lib().gf_server_drain(self.h))

    def pause(self, paused=True):
        """gf_server_pause: hold (or release) the queue; running batches finish."""
        check(lib().gf_server_pause(self.h, 1 if paused else 0))

    def info(self):
        """gf_server_get_info: batches run, requests completed and deferred at
        admission, the largest memory reservation and most batches at once."""
        i = ServerInfo()
        check(lib().gf_server_get_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in ServerInfo._fields_ if k != "pad"}

    def close(self):
        if self.h:
            lib().gf_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# catalog text output (gf_textout, the reference's os_textout)
# ---------------------------------------------------------------------------
class TextoutConfig(C.Structure):
    _fields_ = [("bandset", C.c_char_p), ("bands", C.POINTER(C.c_char_p)), ("nbands", C.c_int32),
                ("band", C.c_char_p), ("absband", C.c_char_p), ("radec", C.c_int32), ("feh", C.c_int32),
                ("feh_comp", C.c_int32), ("vcyl", C.c_int32), ("pm_coordsys", C.c_int32), ("photoerrors", C.c_int32),
                ("comp_ids", C.POINTER(C.c_int32)), ("ncomp", C.c_int32), ("version", C.c_char_p),
                ("threads", C.c_int32), ("multiples", C.c_int32)]


class TextoutSet(C.Structure):
    _fields_ = [("njobs", C.c_int32), ("writers", C.POINTER(C.c_void_p))]


def textout_config(w, version=None, threads=0):
    """The text-output columns of a workload's module chain: SDSS-like ugriz
    (bandset SDSSugriz) or LSST-like ugrizy (LSSTugrizy) by the band count,
    bootstrap band r."""
    cfg = TextoutConfig()
    nb = int(w.nbands)
    keep = []
    if nb:
        pre, bs = ("SDSS", "SDSSugriz") if nb == 5 else ("LSST", "LSSTugrizy")
        bands = [pre + ch for ch in "ugrizy"[:nb]]
        arr = (C.c_char_p * nb)(*[b.encode() for b in bands])
        keep.append(arr)
        cfg.bandset = bs.encode()
        cfg.bands = arr
        cfg.nbands = nb
        cfg.band = bands[2].encode()
    else:
        cfg.band = b"SDSSr"
    cfg.radec = 1 if w.gal2other else 0
    cfg.feh = 1 if (w.feh is not None or w.feh_ivezic is not None or w.feh_gauss is not None) else 0
    cfg.feh_comp = 1 if w.feh_gauss is not None else 0
    cfg.vcyl = 1 if w.kin is not None else 0
    cfg.pm_coordsys = int(w.v2pm.coordsys) if w.v2pm is not None else -1
    cfg.photoerrors = 1 if w.perr is not None else 0
    cfg.version = version.encode() if version else None
    cfg.threads = int(threads)
    cfg.multiples = 1 if getattr(w, "multiples", None) is not None else 0
    cfg._keep = keep
    return cfg


class TextWriter:
    """gf_textout: a catalog text file in the reference's format."""

    _open = "gf_textout_open"

    def __init__(self, path, cfg):
        self.h = C.c_void_p()
        self.cfg = cfg
        check(getattr(lib(), self._open)(str(path).encode(), C.byref(cfg), C.byref(self.h)))

    def write(self, table, begin, end):
        check(lib().gf_textout_write(self.h, C.byref(table), int(begin), int(end)))

    def close(self):
        rows, nbytes = C.c_int64(), C.c_int64()
        if self.h:
            check(lib().gf_textout_close(self.h, C.byref(rows), C.byref(nbytes)))
            self.h = C.c_void_p()
        return rows.value, nbytes.value


class FitsWriter(TextWriter):
    """gf_fitsout_open: the same catalog as a FITS file (the reference's os_fitsout)."""

    _open = "gf_fitsout_open"
