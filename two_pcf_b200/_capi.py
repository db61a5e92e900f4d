"""ctypes declarations of the C ABI in include/two_pcf_b200.h.

The shared library is built in-tree (two_pcf_b200/build.py ->
two_pcf_b200/lib/libtpcf_b200.so).  There is no fallback: if the library is
missing or cannot be loaded, import fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libtpcf_b200.so")
# the checked build (device bounds checks) of the same library
CHECKED_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "checked", "libtpcf_b200.so")
if os.environ.get("TPCF_CHECKED") == "1":
    LIB_PATH = CHECKED_LIB_PATH

TPCF_OK = 0
TPCF_E_INVALID_ARG = 1
TPCF_E_OOM = 2
TPCF_E_CUDA = 3
TPCF_E_DEVICE_TIMEOUT = 4
TPCF_E_OVERFLOW = 5
TPCF_E_UNSUPPORTED = 6
TPCF_E_DEVICE_CHECK = 7

MONOPOLE, SIGMA_PI, S_MU, ANGULAR = 0, 1, 2, 3
FP32_GUARD, FP64 = 0, 1


class AxisSpec(C.Structure):
    _fields_ = [("min", C.c_double), ("max", C.c_double), ("log_base", C.c_double), ("n_bins", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("candidates", C.c_uint64), ("in_range", C.c_uint64), ("guard_evals", C.c_uint64),
                ("overflow_updates", C.c_uint64), ("work_items", C.c_uint64), ("ms_kernel", C.c_double),
                ("ms_total", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


WEIGHTS_PLAIN, WEIGHTS_INVP_DD, WEIGHTS_INVP_DR, WEIGHTS_INVP_DD_DITHER = 0, 1, 2, 3
LOS_ANGULAR, LOS_MIDPOINT = 0, 1
BATCH_DD, BATCH_DR, BATCH_AUTOTUNE = 1, 2, -1


class WeightSpec(C.Structure):
    _fields_ = [("weighting", C.c_int32), ("n_bitwise_runs", C.c_int32), ("theta_axis", AxisSpec),
                ("up_numerator", C.c_void_p), ("up_denominator", C.c_void_p)]


class CountJob(C.Structure):
    _fields_ = [("a", C.c_void_p), ("b", C.c_void_p), ("bin", C.c_void_p), ("spec", C.c_void_p),
                ("precision", C.c_int32), ("reference_form", C.c_int32), ("full_out", C.c_void_p),
                ("region_out", C.c_void_p), ("stats", C.c_void_p)]


# Every symbol the header declares, with (restype, argtypes).
_vp = C.c_void_p
_PROTOTYPES = {
    "tpcf_abi_version": (C.c_int, []),
    "tpcf_status_string": (C.c_char_p, [C.c_int]),
    "tpcf_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "tpcf_destroy": (C.c_int, [_vp]),
    "tpcf_last_error": (C.c_char_p, [_vp]),
    "tpcf_set_stream": (C.c_int, [_vp, _vp]),
    "tpcf_set_refinement": (C.c_int, [_vp, C.c_int]),
    "tpcf_synchronize": (C.c_int, [_vp]),
    "tpcf_catalog_create": (C.c_int, [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int32, _vp, C.c_int32,
                                      C.POINTER(_vp)]),
    "tpcf_catalog_destroy": (C.c_int, [_vp]),
    "tpcf_catalog_n_used": (C.c_int64, [_vp]),
    "tpcf_catalog_release_cache": (C.c_int, [_vp]),
    "tpcf_binning_create": (C.c_int, [_vp, C.c_int, C.POINTER(AxisSpec), C.POINTER(AxisSpec), C.c_int32,
                                      C.POINTER(_vp)]),
    "tpcf_binning_destroy": (C.c_int, [_vp]),
    "tpcf_binning_total_bins": (C.c_int, [_vp]),
    "tpcf_binning_thresholds": (C.c_int, [_vp, C.c_int, _vp, C.c_int]),
    "tpcf_count": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_count_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_count_many": (C.c_int, [_vp, _vp, C.c_int32]),
    "tpcf_count_shard": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_int, C.c_int32, C.c_int32, _vp,
                                   C.POINTER(C.c_int32), C.POINTER(Stats)]),
    "tpcf_shard_combine": (C.c_int, [_vp, _vp, C.c_int32, _vp, _vp]),
    "tpcf_count_weighted": (C.c_int, [_vp, _vp, _vp, _vp, C.POINTER(WeightSpec), C.c_int, _vp, _vp,
                                      C.POINTER(Stats)]),
    "tpcf_pair_count_weighted": (C.c_int, [_vp, _vp, _vp, _vp, C.POINTER(WeightSpec), C.c_int, _vp, _vp,
                                           C.POINTER(Stats)]),
    "tpcf_upweight_eval": (C.c_int, [C.POINTER(WeightSpec), _vp, C.c_int64, _vp]),
    "tpcf_count_backward": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_catalog_set_weights": (C.c_int, [_vp, _vp]),
    "tpcf_catalog_set_dither_masks": (C.c_int, [_vp, _vp]),
    "tpcf_binning_set_line_of_sight": (C.c_int, [_vp, C.c_int]),
    "tpcf_iip_weights": (C.c_int, [C.c_int64, C.c_int32, _vp, _vp, C.c_int32, _vp, _vp]),
    "tpcf_batch_create": (C.c_int, [_vp, _vp, C.c_int32, _vp, _vp, C.c_int, C.c_int32, C.c_int32, C.POINTER(_vp)]),
    "tpcf_batch_run": (C.c_int, [_vp, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_batch_n_outputs": (C.c_int, [_vp]),
    "tpcf_batch_refinement": (C.c_int, [_vp]),
    "tpcf_batch_order": (C.c_int, [C.c_void_p]),
    "tpcf_batch_destroy": (C.c_int, [_vp]),
    "tpcf_auto_pair_count": (C.c_int, [_vp, _vp, _vp, C.c_int, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_cross_pair_count": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _vp, _vp, C.POINTER(Stats)]),
    "tpcf_normalise_auto": (C.c_int, [_vp, C.c_int32, _vp, _vp]),
    "tpcf_normalise_cross": (C.c_int, [_vp, _vp, C.c_int32, _vp, _vp]),
    "tpcf_ls_estimator": (C.c_double, [C.c_double, C.c_double, C.c_double]),
    "tpcf_kernel_launches": (C.c_uint64, [_vp]),
    "tpcf_measure_peaks": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "tpcf_wait_selftest": (C.c_int, [_vp, C.c_int32, C.c_uint32]),
    "tpcf_debug_fail_allocations": (C.c_int, [C.c_int64]),
    "tpcf_debug_force_tile_timeout": (C.c_int, [C.c_int32]),
    # command-line flow (host only)
    "tpcf_host_last_error": (C.c_char_p, []),
    "tpcf_params_load": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "tpcf_params_parse": (C.c_int, [C.c_char_p, C.POINTER(_vp)]),
    "tpcf_params_destroy": (C.c_int, [_vp]),
    "tpcf_params_get_double": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_double)]),
    "tpcf_params_get_int": (C.c_int, [_vp, C.c_char_p, C.POINTER(C.c_int32)]),
    "tpcf_params_get_string": (C.c_int, [_vp, C.c_char_p, C.c_char_p, C.c_int32]),
    "tpcf_cosmology_create": (C.c_int, [C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int32,
                                        C.POINTER(_vp)]),
    "tpcf_cosmology_destroy": (C.c_int, [_vp]),
    "tpcf_cosmology_comov_dist": (C.c_int, [_vp, _vp, C.c_int64, _vp]),
    "tpcf_galaxy_set": (C.c_int, [C.c_int64, _vp, _vp, _vp, _vp, _vp]),
    "tpcf_cartesian_set": (C.c_int, [C.c_int64, _vp, _vp, _vp]),
    "tpcf_read_ascii": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int32, _vp, C.POINTER(_vp)]),
    "tpcf_host_catalog_size": (C.c_int64, [_vp]),
    "tpcf_host_catalog_arrays": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp),
                                           C.POINTER(_vp)]),
    "tpcf_host_catalog_destroy": (C.c_int, [_vp]),
    "tpcf_sub_filename": (C.c_int, [C.c_char_p, C.c_int64, C.c_char_p, C.c_int32]),
    "tpcf_write_xi_ascii": (C.c_int, [C.c_char_p, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "tpcf_run_param_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int]),
    "tpcf_set_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "tpcf_device_checks": (C.c_int, []),
    "tpcf_debug_corrupt_work_list": (C.c_int, [C.c_int]),
    "tpcf_set_kernel_config": (C.c_int, [C.c_void_p, C.c_int]),
    "tpcf_set_cross_order": (C.c_int, [C.c_void_p, C.c_int]),
    "tpcf_autotune_describe": (C.c_int64, [C.c_void_p, C.c_char_p, C.c_int64]),
    "tpcf_run_param_file_report": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_char_p]),
    "tpcf_run_invp": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, _vp, C.c_int]),
}

CARTESIAN, EQUATORIAL = 0, 1
PARTIAL_WORDS = 7

_LIB = None


def header_symbols(header_path: str | None = None) -> list[str]:
    """Function names declared in include/two_pcf_b200.h."""
    import re
    if header_path is None:
        header_path = os.path.join(os.path.dirname(os.path.dirname(LIB_PATH)), os.pardir, "include",
                                   "two_pcf_b200.h")
    src = open(os.path.normpath(header_path)).read()
    return sorted(set(re.findall(r"\b(tpcf_[a-z0-9_]+)\s*\(", src)))


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python two_pcf_b200/build.py` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB
