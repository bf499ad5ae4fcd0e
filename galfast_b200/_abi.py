"""ctypes mirror of include/galfast_b200.h (structures only)."""
import ctypes as C

GF_OK = 0
GF_MODEL_EXP_DISK = 1
GF_MODEL_POWER_LAW_ELLIPSOID = 2
GF_MODEL_BROKEN_POWER_LAW = 3
GF_MODEL_LCBULGE = 4
GF_MODEL_DENSITY_CUBE = 5
GF_FRAME_GALPLANE = 0
GF_FRAME_EXPLICIT = 1
GF_EXT_NONE = 0
GF_EXT_SCREEN_CSCB = 1
GF_EXT_MAPS = 2
GF_FOOT_ALL = 0
GF_FOOT_LAMBERT_RECT = 1
GF_FOOT_CAP = 2
GF_FOOT_LB_RECT = 4
GF_FOOT_REGIONS = 5
GF_FOOT_LATCUT = 3
GF_MAX_BANDS = 17


class PencilBeam(C.Structure):
    _fields_ = [("cl", C.c_float), ("cb", C.c_float), ("sl", C.c_float), ("sb", C.c_float),
                ("coveredFraction", C.c_float), ("dx", C.c_float), ("dA", C.c_float),
                ("projIdx", C.c_int32), ("X", C.c_float), ("Y", C.c_float), ("extIdx", C.c_int32),
                ("pad_", C.c_int32)]


class Lambert(C.Structure):
    _fields_ = [("l0", C.c_double), ("b0", C.c_double),
                ("cl", C.c_float), ("cb", C.c_float), ("sl", C.c_float), ("sb", C.c_float)]


class SkygenConfig(C.Structure):
    _fields_ = [("m0", C.c_float), ("m1", C.c_float), ("dm", C.c_float),
                ("M0", C.c_float), ("M1", C.c_float),
                ("dmin", C.c_float), ("dmax", C.c_float),
                ("nthreads", C.c_int32), ("nstars", C.c_float),
                ("proj", Lambert * 2)]


class ModelConfig(C.Structure):
    _fields_ = [("type", C.c_int32), ("comp", C.c_int32), ("f", C.c_double),
                ("l", C.c_double), ("h", C.c_double), ("rcut", C.c_double),
                ("n", C.c_double), ("ba", C.c_double), ("ca", C.c_double),
                ("rmin", C.c_double), ("rmax", C.c_double),
                ("frame", C.c_int32), ("Rg", C.c_double), ("z0", C.c_double),
                ("T", C.c_double * 3), ("M", C.c_double * 9),
                ("lf_l", C.c_double), ("lf_b", C.c_double), ("lf_D", C.c_double),
                ("lf_M", C.POINTER(C.c_double)), ("lf_phi", C.POINTER(C.c_double)), ("lf_n", C.c_int32),
                ("nbreaks", C.c_int32), ("n_brk", C.c_double * 10), ("rbreak", C.c_double * 9),
                ("cube", C.POINTER(C.c_float)), ("cube_n", C.c_int32 * 3), ("cube_tc", (C.c_float * 2) * 3)]


class ExtMap(C.Structure):                # gf_ext_map: one hemisphere's 3-D extinction map
    _fields_ = [("A", C.POINTER(C.c_float)), ("n", C.c_int32 * 3), ("tc", (C.c_float * 2) * 3)]


class Extinction(C.Structure):
    _fields_ = [("kind", C.c_int32), ("A0", C.c_float), ("north", C.POINTER(ExtMap)), ("south", C.POINTER(ExtMap))]


GF_REGION_BEAM, GF_REGION_RECT = 1, 2
GF_COORD_GAL, GF_COORD_EQU = 0, 1
GF_MAX_REGIONS = 8


class Region(C.Structure):                # gf_region: one footprint specification
    _fields_ = [("type", C.c_int32), ("coordsys", C.c_int32), ("a", C.c_double), ("b", C.c_double),
                ("c", C.c_double), ("d", C.c_double), ("bmin", C.c_double)]


class Footprint(C.Structure):
    _fields_ = [("kind", C.c_int32), ("proj", C.c_int32),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double), ("d", C.c_double),
                ("nregions", C.c_int32), ("pad_", C.c_int32), ("regions", Region * GF_MAX_REGIONS)]


class Table(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("size", C.c_int64), ("nbands", C.c_int32),
                ("lb", C.c_void_p), ("projIdx", C.c_void_p), ("projXY", C.c_void_p),
                ("DM", C.c_void_p), ("absmag", C.c_void_p), ("XYZ", C.c_void_p),
                ("comp", C.c_void_p), ("Am", C.c_void_p), ("AmInf", C.c_void_p),
                ("hidden", C.c_void_p), ("FeH", C.c_void_p), ("vcyl", C.c_void_p),
                ("mags", C.c_void_p), ("photoflags", C.c_void_p), ("obsmags", C.c_void_p),
                ("pm", C.c_void_p), ("radec", C.c_void_p), ("FeH_comp", C.c_void_p),
                ("absmagSys", C.c_void_p), ("absmagSysNcomp", C.c_void_p), ("systems", C.c_int32)]


GF_MULT_LF_M2_GT_M1, GF_MULT_LF, GF_MULT_EQUAL_MASS = 1, 2, 3


class MultiplesConfig(C.Structure):     # gf_multiples_config (os_unresolvedMultiples)
    _fields_ = [("algo", C.c_int32), ("comp_mask", C.c_uint32),
                ("sec_x0", C.c_float), ("sec_inv_dx", C.c_float), ("nsec", C.c_int32), ("secprob", C.c_float * 64),
                ("cum_x0", C.c_float), ("cum_inv_dx", C.c_float), ("ncum", C.c_int32), ("cumlf", C.c_float * 256),
                ("inv_x0", C.c_float), ("inv_inv_dx", C.c_float), ("ninv", C.c_int32), ("invcumlf", C.c_float * 256)]


class FixedFeHConfig(C.Structure):
    _fields_ = [("FeH", C.c_float), ("comp_mask", C.c_uint32)]


class FehConfig(C.Structure):            # gf_feh_config (os_FeH, Ivezic et al. 2008)
    _fields_ = [("A", C.c_float * 2), ("sigma", C.c_float * 3), ("offs", C.c_float * 3), ("Hmu", C.c_float),
                ("muInf", C.c_float), ("DeltaMu", C.c_float), ("comp_thin", C.c_uint32), ("comp_thick", C.c_uint32),
                ("comp_halo", C.c_uint32), ("M", C.c_float * 9), ("T", C.c_float * 3)]


GF_GAUSSFEH_MAXCOMP = 10


class GaussFehConfig(C.Structure):       # gf_gaussfeh_config (os_GaussianFeH)
    _fields_ = [("ncomp", C.c_int32), ("mean", C.c_float * GF_GAUSSFEH_MAXCOMP),
                ("sigma", C.c_float * GF_GAUSSFEH_MAXCOMP), ("pcum", C.c_float * GF_GAUSSFEH_MAXCOMP),
                ("comp_mask", C.c_uint32)]


class VMoments(C.Structure):
    _fields_ = [("m", (C.c_float * 5) * 3), ("ss", (C.c_float * 5) * 6)]


class Bond2010Config(C.Structure):
    _fields_ = [("comp_thin", C.c_uint32), ("comp_thick", C.c_uint32), ("comp_halo", C.c_uint32),
                ("fk", C.c_float), ("disk_1", VMoments), ("disk_2", VMoments), ("halo", VMoments),
                ("M", C.c_float * 9), ("T", C.c_float * 3)]


class PhotometryConfig(C.Structure):
    _fields_ = [("nbands", C.c_int32), ("bidx", C.c_int32), ("reddening", C.c_float * GF_MAX_BANDS),
                ("nFeH", C.c_int32), ("nMr", C.c_int32), ("tcFeH", C.c_float * 2), ("tcMr", C.c_float * 2),
                ("colors", C.POINTER(C.c_float)), ("eflags", C.POINTER(C.c_uint8)), ("comp_mask", C.c_uint32)]


class PhotoerrConfig(C.Structure):
    _fields_ = [("nbands", C.c_int32), ("nknots", C.c_int32),
                ("mag", C.POINTER(C.c_double)), ("sigma", C.POINTER(C.c_double)), ("seed", C.c_uint64)]


class Vel2pmConfig(C.Structure):
    _fields_ = [("coordsys", C.c_int32), ("vLSR", C.c_float), ("u0", C.c_float), ("v0", C.c_float),
                ("w0", C.c_float), ("Rg", C.c_float)]


class ModelInfo(C.Structure):
    _fields_ = [("m0", C.c_float), ("m1", C.c_float), ("dm", C.c_float), ("M0", C.c_float),
                ("M1", C.c_float), ("dM", C.c_float), ("nm", C.c_int32), ("nM", C.c_int32),
                ("npixels", C.c_int32), ("nthreads", C.c_int32), ("f", C.c_float),
                ("lf_x0", C.c_float), ("lf_inv_dx", C.c_float), ("lf_n", C.c_int32), ("norm", C.c_float)]


# exported symbols of libgalfast_b200.so declared in include/galfast_b200.h
EXPORTS = [
    "gf_last_error", "gf_ctx_create", "gf_ctx_destroy", "gf_ctx_sync", "gf_ctx_mark", "gf_ctx_elapsed",
    "gf_launch_count", "gf_catalog_run", "gf_catalog_run_multi", "gf_multi_set_memory_budget", "gf_table_download_rows", "gf_server_create", "gf_server_submit", "gf_server_drain", "gf_server_get_info", "gf_server_pause", "gf_server_destroy", "gf_skygen_precision", "gf_tuning_get", "gf_tuning_set", "gf_catalog_run_multi_host", "gf_profile_enable", "gf_profile_read",
    "gf_rng_init", "gf_rng_seed48_from_cli_seed", "gf_rng_get_state", "gf_rng_set_state",
    "gf_skygen_create", "gf_skygen_destroy", "gf_skygen_model_info_get", "gf_skygen_model_lf_get",
    "gf_skygen_integrate", "gf_skygen_set_norm", "gf_skygen_draw",
    "gf_table_alloc", "gf_table_free", "gf_table_download",
    "gf_module_clipper", "gf_module_fixedfeh", "gf_module_bond2010", "gf_module_multiples", "gf_multiples_build",
    "gf_photometry_create", "gf_photometry_destroy", "gf_module_photometry",
    "gf_photoerr_create", "gf_photoerr_destroy", "gf_module_photoerrors",
    "gf_module_vel2pm", "gf_module_gal2other",
    "gf_lambert_init", "gf_footprint_pixelize", "gf_photometry_build", "gf_extinction_beam_minima",
    "gf_multipliers", "gf_rng_seed_host", "gf_mt19937_outputs", "gf_skygen_setup_host",
    "gf_skygen_integrate_static",
]


class PrecisionReport(C.Structure):
    _fields_ = [("expected32", C.c_double), ("expected64", C.c_double), ("total_rel_err", C.c_double),
                ("bin_max_rel_err", C.c_double), ("bin_mean_rel_err", C.c_double),
                ("pixel_max_rel_err", C.c_double), ("pixel_mean_rel_err", C.c_double), ("bins", C.c_int64)]
