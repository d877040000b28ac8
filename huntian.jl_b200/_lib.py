"""ctypes bindings of libhuntian_b200.so (include/huntian_b200.h).

The library is the product: every compute entry point of this package goes through it.
If it is missing or fails to load, import of the bindings raises -- there is no CPU or
PyTorch fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# HT_CHECKED=1 selects the bounds-checked build (build.py --checked), same C ABI
LIB_PATH = os.path.join(_HERE, "libhuntian_b200_checked.so" if os.environ.get("HT_CHECKED") == "1"
                        else "libhuntian_b200.so")

HT_OK = 0
HT_ERR_INVALID = 1
HT_ERR_CUDA = 2
HT_ERR_NOMEM = 3
HT_ERR_STATE = 4
HT_ERR_CAPACITY = 5
HT_ERR_FAULT = 6

HT_CONV_GPU = 0
HT_CONV_CPU = 1
HT_MODE_PLAIN = 0
HT_MODE_BATCHED = 1
HT_MODE_LEARNED = 2
HT_BRACKET_NPARAMS = 9928
HT_TUNE_BLOCK_BITS = 1
HT_TUNE_PF_KZ = 2
HT_TUNE_WALK_BPSM = 3
HT_TUNE_FFT_PATH = 4
HT_TUNE_WAIT_NS = 5
HT_TUNE_INJECT_TX = 6
# reject reasons (HT_REJECT_*), in counter order
REJECT_REASONS = ("premask", "no_fcrit", "m0_one", "no_collapse", "rthl_neg", "outside")

# every symbol include/huntian_b200.h declares
SYMBOLS = ("ht_ctx_create", "ht_ctx_destroy", "ht_last_error", "ht_ctx_shell_info",
           "ht_ctx_shell_r2", "ht_fsc_of_z", "ht_smooth_window", "ht_smooth_tile",
           "ht_smooth_tile_planes", "ht_smooth_pencil_supported", "ht_spectrum_pencil",
           "ht_smooth_pencil",
           "ht_smooth_filter",
           "ht_peakfind_filter",
           "ht_fields_pack",
           "ht_shell_analyse", "ht_shell_analyse_static", "ht_last_launch_stats",
           "ht_reject_counts", "ht_reset_reject_counts",
           "ht_record_gather_probe",
           "ht_device_status", "ht_bracket_features", "ht_bracket_predict", "ht_bracket_grad",
           "ht_bracket_adam", "ht_ctx_tune", "ht_ctx_set_cosmo", "ht_peak_lightcone",
           "ht_pack_halos", "ht_merge_halos", "ht_finalize_eulerian", "ht_evolve_ellipses",
           "ht_collapse_table")


class HTError(RuntimeError):
    """A huntian_b200 entry point returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"huntian_b200 error {code}: {msg}")
        self.code = code


_P = C.c_void_p


class HtPeaks(C.Structure):
    _fields_ = [("i", _P), ("j", _P), ("k", _P), ("delta", _P), ("lapd", _P),
                ("filter_idx", _P), ("count", _P), ("found", _P)]


class HtFields(C.Structure):
    _fields_ = [("delta", _P), ("etax", _P), ("etay", _P), ("etaz", _P), ("eta2x", _P),
                ("eta2y", _P), ("eta2z", _P), ("lapd", _P), ("n1", C.c_int32),
                ("n2", C.c_int32), ("n3", C.c_int32)]


class HtPeakBatch(C.Structure):
    _fields_ = [("pi", _P), ("pj", _P), ("pk", _P), ("Rf", _P), ("ir2min", _P), ("ZZon", _P),
                ("fcrit", _P), ("npeaks", C.c_int64), ("order", _P), ("cost", _P)]


RESULT_NAMES = ("RTHL", "Fbarx", "e_v", "p_v", "strain", "eigs", "Srb", "Sbar", "Sbar2",
                "gradpk", "gradpkf", "gradpkrf", "d2F", "zvir_half")
RESULT_WIDTH = {"strain": 9, "eigs": 3, "Sbar": 3, "Sbar2": 3, "gradpk": 3, "gradpkf": 3,
                "gradpkrf": 3}


# nullable Int32 diagnostics after the 14 result arrays
DIAG_NAMES = ("walk_shells", "collapse_shell")


class HtResults(C.Structure):
    _fields_ = [(n, _P) for n in RESULT_NAMES] + [(n, _P) for n in DIAG_NAMES]


class HtCosmo(C.Structure):
    _fields_ = [("chi", _P), ("zchi", _P), ("n_chi", C.c_int32), ("z_max", C.c_double),
                ("atab", _P), ("D_atab", _P), ("dlnD_dlna", _P), ("ntab", C.c_int32)] + \
        [(n, C.c_double) for n in ("amintab", "amaxtab", "D_ainfty", "D_a0", "HD_Hainfty",
                                   "HD_Ha0", "Om", "OL")]


class HtEllipsoid(C.Structure):
    _fields_ = [("Om", C.c_double), ("OL", C.c_double), ("iforce_strat", C.c_int32),
                ("ivir_strat", C.c_int32), ("fcoll", C.c_double * 3), ("tfac", C.c_double),
                ("nstepmax", C.c_int32), ("zinit_fac", C.c_double), ("solver", C.c_int32)]


HT_SOLVER_RK4 = 0
HT_SOLVER_TSIT5 = 1


class HtGrowth(C.Structure):
    _fields_ = [("atab", _P), ("D_atab", _P), ("dlnD_dlnatab", _P), ("ntab", C.c_int32)] + \
        [(n, C.c_double) for n in ("amintab", "amaxtab", "D_ainfty", "D_a0", "HD_Hainfty",
                                   "HD_Ha0")]


class HtTileGeom(C.Structure):
    _fields_ = [("n", C.c_int32), ("xbx", C.c_double), ("ybx", C.c_double),
                ("zbx", C.c_double), ("alatt", C.c_double)]


class HtCatalogPeaks(C.Structure):
    _fields_ = [(n, _P) for n in ("i", "j", "k", "Rf", "FcRf", "d2Rf", "z")] + \
        [("npeaks", C.c_int64)]


class HtBracketModel(C.Structure):
    _fields_ = [(n, _P) for n in ("W1", "W2", "W3", "W4", "b1", "b2", "b3", "b4", "mean",
                                  "istd")]


_lib = None


def load() -> C.CDLL:
    """Load libhuntian_b200.so (built by build.py); raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python huntian.jl_b200/build.py` (no fallback path exists)")
    L = C.CDLL(LIB_PATH)
    i32, i64, dbl = C.c_int32, C.c_int64, C.c_double
    L.ht_last_error.restype = C.c_char_p
    L.ht_last_error.argtypes = []
    L.ht_ctx_create.restype = C.c_int
    L.ht_ctx_create.argtypes = [C.c_int, C.c_int, _P, C.c_int, C.c_int, C.c_int, dbl, dbl,
                                dbl, dbl, dbl, dbl, dbl, C.POINTER(_P)]
    L.ht_ctx_destroy.restype = C.c_int
    L.ht_ctx_destroy.argtypes = [_P]
    L.ht_ctx_shell_info.restype = C.c_int
    L.ht_ctx_shell_info.argtypes = [_P, C.POINTER(i32), C.POINTER(i64)]
    L.ht_ctx_shell_r2.restype = C.c_int
    L.ht_ctx_shell_r2.argtypes = [_P, _P, i32]
    L.ht_fsc_of_z.restype = C.c_int
    L.ht_fsc_of_z.argtypes = [_P, dbl, C.POINTER(dbl)]
    L.ht_smooth_window.restype = C.c_int
    L.ht_smooth_window.argtypes = [_P, _P, _P, C.c_int, dbl, dbl, C.c_int, _P]
    L.ht_smooth_tile.restype = C.c_int
    L.ht_smooth_tile.argtypes = [_P, _P, _P, C.c_int, dbl, dbl, C.c_int, _P]
    L.ht_smooth_tile_planes.restype = C.c_int
    L.ht_smooth_tile_planes.argtypes = [_P, _P, _P, C.c_int, dbl, dbl, C.c_int, C.c_int,
                                        C.c_int, _P]
    L.ht_smooth_pencil_supported.restype = C.c_int
    L.ht_smooth_pencil_supported.argtypes = [C.c_int]
    L.ht_spectrum_pencil.restype = C.c_int
    L.ht_spectrum_pencil.argtypes = [_P, _P, _P, C.c_int, _P]
    L.ht_smooth_pencil.restype = C.c_int
    L.ht_smooth_pencil.argtypes = [_P, _P, _P, C.c_int, dbl, dbl, C.c_int, C.c_int, C.c_int, _P]
    L.ht_smooth_filter.restype = C.c_int
    L.ht_smooth_filter.argtypes = [_P, _P, _P, C.c_int, C.c_int, dbl, dbl, C.c_int, _P]
    L.ht_peakfind_filter.restype = C.c_int
    L.ht_peakfind_filter.argtypes = [_P, _P, _P, _P, C.c_int, C.c_int, C.c_float, i32, i64,
                                     C.POINTER(HtPeaks), _P]
    L.ht_fields_pack.restype = C.c_int
    L.ht_fields_pack.argtypes = [_P, C.POINTER(HtFields), _P]
    L.ht_shell_analyse.restype = C.c_int
    L.ht_shell_analyse.argtypes = [_P, C.POINTER(HtPeakBatch), dbl, dbl, i32, _P, i32, i32,
                                   C.POINTER(HtResults), _P]
    L.ht_shell_analyse_static.restype = C.c_int
    L.ht_shell_analyse_static.argtypes = [_P, C.POINTER(HtFields), C.POINTER(HtPeakBatch), dbl,
                                          dbl, i32, _P, i32, C.POINTER(HtResults), _P]
    L.ht_last_launch_stats.restype = C.c_int
    L.ht_last_launch_stats.argtypes = [_P, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64)]
    L.ht_reject_counts.restype = C.c_int
    L.ht_reject_counts.argtypes = [_P, C.POINTER(i64)]
    L.ht_reset_reject_counts.restype = C.c_int
    L.ht_reset_reject_counts.argtypes = [_P, _P]
    L.ht_record_gather_probe.restype = C.c_int
    L.ht_record_gather_probe.argtypes = [_P, _P, i64, _P, _P]
    L.ht_device_status.restype = C.c_int
    L.ht_device_status.argtypes = [_P, C.POINTER(i32)]
    L.ht_ctx_tune.restype = C.c_int
    L.ht_ctx_tune.argtypes = [_P, i32, i64]
    L.ht_bracket_features.restype = C.c_int
    L.ht_bracket_features.argtypes = [_P, C.POINTER(HtPeakBatch), _P, dbl, _P, _P]
    L.ht_bracket_predict.restype = C.c_int
    L.ht_bracket_predict.argtypes = [_P, C.POINTER(HtBracketModel), _P, i64, _P, _P]
    L.ht_bracket_grad.restype = C.c_int
    L.ht_bracket_grad.argtypes = [_P, C.POINTER(HtBracketModel), _P, _P, i64, _P, _P, _P]
    L.ht_bracket_adam.restype = C.c_int
    L.ht_bracket_adam.argtypes = [_P, _P, _P, _P, _P, i32, C.c_float,
                                  C.POINTER(HtBracketModel), _P]
    L.ht_ctx_set_cosmo.restype = C.c_int
    L.ht_ctx_set_cosmo.argtypes = [_P, C.POINTER(HtCosmo)]
    L.ht_peak_lightcone.restype = C.c_int
    L.ht_peak_lightcone.argtypes = [_P, _P, _P, _P, i64, C.POINTER(HtTileGeom), _P, dbl, _P,
                                    _P, _P, _P, _P, _P]
    L.ht_pack_halos.restype = C.c_int
    L.ht_pack_halos.argtypes = [_P, C.POINTER(HtCatalogPeaks), C.POINTER(HtResults),
                                C.POINTER(HtTileGeom), dbl, dbl, i32, i32, _P, i64, _P, _P]
    L.ht_merge_halos.restype = C.c_int
    L.ht_merge_halos.argtypes = [_P, _P, i64, i32, i32, i32, _P, _P, _P]
    L.ht_finalize_eulerian.restype = C.c_int
    L.ht_finalize_eulerian.argtypes = [_P, _P, i64, i32, _P, i32, dbl, _P]
    L.ht_evolve_ellipses.restype = C.c_int
    L.ht_evolve_ellipses.argtypes = [C.c_int, C.POINTER(HtEllipsoid), C.POINTER(HtGrowth), i64,
                                     _P, _P, _P, i32, _P, _P, _P, _P, _P]
    L.ht_collapse_table.restype = C.c_int
    L.ht_collapse_table.argtypes = [C.c_int, C.POINTER(HtEllipsoid), C.POINTER(HtGrowth), i32,
                                    i32, i32] + [dbl] * 6 + [_P]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != HT_OK:
        raise HTError(rc, load().ht_last_error().decode(errors="replace"))
