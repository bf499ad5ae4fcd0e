"""Python binding of the CPU oracle (test infrastructure).

Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
It drives oracle/_build/liboracle_{p,l}.so -- the sequential restatement of the
reference CPU path -- on the same inputs the product library receives.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
_libs = {}


def build():
    subprocess.run(["sh", os.path.join(HERE, "build.sh")], check=True)


def load(flavour="p"):
    """flavour 'p': portable math (bit-comparable with the GPU); 'l': host libm."""
    if flavour not in _libs:
        path = os.path.join(BUILD, "liboracle_%s.so" % flavour)
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        L.or_last_error.restype = C.c_char_p
        L.or_set_threads.argtypes = [C.c_int]
        L.or_rng_seed.argtypes = [C.c_uint32, C.c_int32, vp, vp]
        L.or_mwc_uniforms.argtypes = [vp, vp, vp, C.c_int, vp]
        L.or_mwc_poisson.argtypes = [vp, vp, vp, vp, C.c_int, vp]
        L.or_mwc_gaussian.argtypes = [vp, vp, vp, C.c_float, C.c_int, vp]
        L.or_skygen_create.restype = vp
        L.or_skygen_create.argtypes = [vp, vp, C.c_int32, vp, vp, vp, C.c_int32]
        L.or_skygen_destroy.argtypes = [vp]
        L.or_skygen_model_info.argtypes = [vp, C.c_int32, vp]
        L.or_skygen_model_lf.argtypes = [vp, C.c_int32, vp]
        L.or_skygen_integrate.argtypes = [vp, C.c_int32, vp, vp, vp]
        L.or_expected_fp64.argtypes = [vp, C.c_int32, C.c_int32, vp, vp]
        L.or_count_bins_above.argtypes = [vp, C.c_int32, C.c_float, vp]
        L.or_skygen_set_norm.argtypes = [vp, C.c_int32, C.c_float]
        L.or_skygen_draw.argtypes = [vp, C.c_int32, vp, C.c_int32, vp, vp, vp]
        L.or_module_clipper.argtypes = [vp, vp, vp, C.c_int64, C.c_int64]
        L.or_module_fixedfeh.argtypes = [vp, vp, C.c_int64, C.c_int64]
        L.or_module_bond2010.argtypes = [vp, vp, C.c_int32, vp, C.c_int64, C.c_int64]
        L.or_module_feh.argtypes = [vp, vp, C.c_int32, vp, C.c_int64, C.c_int64]
        L.or_module_gaussfeh.argtypes = [vp, vp, C.c_int32, vp, C.c_int64, C.c_int64]
        L.or_module_multiples.argtypes = [vp, vp, C.c_int32, vp, C.c_int64, C.c_int64]
        L.or_module_photometry.argtypes = [vp, vp, C.c_int64, C.c_int64]
        L.or_module_photoerrors.argtypes = [vp, C.c_int64, vp, C.c_int64, C.c_int64]
        L.or_module_vel2pm.argtypes = [vp, vp, C.c_int64, C.c_int64]
        L.or_module_gal2other.argtypes = [C.c_int32, vp, C.c_int64, C.c_int64]
        L.or_vcyl2pm.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.or_error_normal.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32]
        L.or_error_normal.restype = C.c_double
        L.or_math_f.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        L.or_math_d.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        L.or_diag.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp]
        L.or_advance.argtypes = [vp, vp, C.c_int, C.c_int]
        _libs[flavour] = L
    return _libs[flavour]


def ref(x):
    return C.byref(x)


def seed_streams(seed48, multipliers, nstreams=65536, flavour="p"):
    L = load(flavour)
    st = np.zeros(3 * nstreams, dtype=np.uint32)
    mult = np.ascontiguousarray(multipliers, dtype=np.uint32)
    L.or_rng_seed(seed48, nstreams, mult.ctypes.data, st.ctypes.data)
    return st


class OracleSkygen:
    """skygen on the CPU for a galfast_b200.workloads.Workload."""

    def __init__(self, w, flavour="p"):
        import galfast_b200 as G
        self.G = G
        self.L = load(flavour)
        self.w = w
        marr = (G.ModelConfig * len(w.models))(*w.models)
        self._marr = marr
        self.h = self.L.or_skygen_create(C.addressof(w.sky), C.addressof(w.pixel_array()), w.npixels,
                                         w.ammin.ctypes.data, C.addressof(w.ext), C.addressof(marr), len(w.models))
        if not self.h:
            raise RuntimeError(self.L.or_last_error().decode())

    def close(self):
        if self.h:
            self.L.or_skygen_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self, model):
        i = self.G.ModelInfo()
        self.L.or_skygen_model_info(self.h, model, C.addressof(i))
        return i

    def lf(self, model):
        a = np.zeros(self.info(model).lf_n, dtype=np.float32)
        self.L.or_skygen_model_lf(self.h, model, a.ctypes.data)
        return a

    def integrate_counts(self, model, per_pixel=False):
        e = C.c_double()
        ec = C.c_double()
        pp = np.zeros(self.w.npixels) if per_pixel else None
        self.L.or_skygen_integrate(self.h, model, C.addressof(e), C.addressof(ec), pp.ctypes.data if pp is not None else None)
        return e.value, ec.value, pp

    def expected_fp64(self, model, pixel):
        """(reference float sum, FP64 sum) of the expected counts of one pixel."""
        a = C.c_double()
        b = C.c_double()
        if self.L.or_expected_fp64(self.h, model, pixel, C.addressof(a), C.addressof(b)) != 0:
            raise ValueError("pixel out of range or nm*nM not a multiple of 10")
        return a.value, b.value

    def count_bins_above(self, model, above):
        """Bins of `model` whose expected count exceeds `above` (diagnostics)."""
        n = C.c_int64()
        self.L.or_count_bins_above(self.h, model, above, C.addressof(n))
        return n.value

    def set_density_norm(self, model, norm):
        self.L.or_skygen_set_norm(self.h, model, norm)

    def draw_sources(self, model, rng_state, table):
        n = C.c_int64()
        d = C.c_int32()
        self.L.or_skygen_draw(self.h, model, rng_state.ctypes.data, len(rng_state) // 3, C.addressof(table.t),
                              C.addressof(n), C.addressof(d))
        return n.value, bool(d.value)


def run_catalog(w, multipliers, flavour="p", sink=None, threads=1, table=None):
    """The reference catalog path on the CPU: integrate all models, then draw
    every model's batches and run the module chain (os_skygen.cpp:866-932).
    table: a HostTable of w.capacity rows and w.nbands bands to reuse (the
    otable of the reference is reused from batch to batch the same way)."""
    import galfast_b200 as G
    L = load(flavour)
    L.or_set_threads(threads)
    state = seed_streams(w.seed48, multipliers, w.nstreams, flavour)
    sky = OracleSkygen(w, flavour)
    order = sorted(range(len(w.models)), key=lambda i: w.models[i].comp)
    expected = {}
    total = 0.0
    for i in range(len(w.models)):
        e, ec, _ = sky.integrate_counts(i)
        expected[i] = (e, ec)
        total += ec
    if w.sky.nstars:
        norm = float(np.float32(w.sky.nstars / total))
        for i in range(len(w.models)):
            sky.set_density_norm(i, norm)
    t = table if table is not None else G.HostTable(w.capacity, w.nbands)
    row_offset = 0
    stats = {"expected": expected, "generated": {}, "stored": {}, "batches": 0}
    NS = len(state) // 3
    for i in order:
        gen = stored = 0
        while True:
            n, done = sky.draw_sources(i, state, t)
            gen += n
            size = t.size
            if size:
                stats["batches"] += 1
                if w.foot is not None:
                    L.or_module_clipper(C.addressof(w.foot), None, C.addressof(t.t), 0, size)
                if w.feh is not None:
                    L.or_module_fixedfeh(C.addressof(w.feh), C.addressof(t.t), 0, size)
                t.t.systems = 0
                for fm, fn in ((getattr(w, "feh_ivezic", None), L.or_module_feh),
                               (getattr(w, "feh_gauss", None), L.or_module_gaussfeh),
                               (getattr(w, "multiples", None), L.or_module_multiples)):
                    if fm is not None and fn(C.addressof(fm), state.ctypes.data, NS, C.addressof(t.t), 0, size) != 0:
                        raise RuntimeError(L.or_last_error().decode())
                if w.kin is not None:
                    if L.or_module_bond2010(C.addressof(w.kin), state.ctypes.data, NS, C.addressof(t.t), 0, size) != 0:
                        raise RuntimeError(L.or_last_error().decode())
                if w.phot is not None:
                    L.or_module_photometry(C.addressof(w.phot), C.addressof(t.t), 0, size)
                if w.perr is not None:
                    L.or_module_photoerrors(C.addressof(w.perr), row_offset, C.addressof(t.t), 0, size)
                if w.v2pm is not None:
                    L.or_module_vel2pm(C.addressof(w.v2pm), C.addressof(t.t), 0, size)
                if w.gal2other:
                    L.or_module_gal2other(w.gal2other, C.addressof(t.t), 0, size)
                stored += size
                if sink is not None:
                    sink(w.models[i].comp, t, row_offset)
                row_offset += size
            if done:
                break
        stats["generated"][i] = gen
        stats["stored"][i] = stored
    sky.close()
    return stats, state
