"""TEST INFRASTRUCTURE ONLY — ctypes access to the reference built in-process.

``oracle/build_ref.sh`` compiles the reference's own sources (``src/*.cpp``,
``src/healpix/*.cpp``) with ``oracle/ref_harness.cpp`` into
``oracle/_ref/libtwopcf_ref_{plain,invp}.so``.  This module wraps those entry
points for the tests, the golden-fixture generator and the CPU-baseline leg of
``bench.py``.  Nothing in the product imports it.

All counts come back as the reference leaves its histograms after
``invert_jk_hists()`` and, for auto counts, ``multiply_hists(2.0)``
(src/correlators.cpp:76-77, :124), before ``normalise()``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_PLAIN = None
_INVP = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")

MONOPOLE, SIGMA_PI, S_MU = 0, 1, 2


class RefAxisFields(C.Structure):
    _fields_ = [("n_bins", C.c_int), ("log_binning", C.c_int), ("min", C.c_float),
                ("minus_min", C.c_float), ("max", C.c_float), ("step", C.c_float),
                ("inv_step", C.c_float), ("base", C.c_float), ("inv_log_of_base", C.c_float),
                ("inv_log_step", C.c_float)]


def available(variant: str = "plain") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libtwopcf_ref_{variant}.so"))


def _opt(arr, dtype):
    """None -> NULL pointer, else a contiguous array of dtype."""
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype)


def _ptr(arr):
    return None if arr is None else arr.ctypes.data_as(C.c_void_p)


def plain():
    global _PLAIN
    if _PLAIN is None:
        path = os.path.join(REF_DIR, "libtwopcf_ref_plain.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        lib = C.CDLL(path)
        lib.ref_axis_fields.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, C.POINTER(RefAxisFields)]
        lib.ref_axis_bin_num.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, _fp, C.c_longlong, _fp]
        lib.ref_axis_centres.argtypes = [C.c_double, C.c_double, C.c_int, C.c_double, _dp, _dp]
        lib.ref_ls_estimator.argtypes = [C.c_double] * 3
        lib.ref_ls_estimator.restype = C.c_double
        lib.ref_comov_dist.argtypes = [C.c_double] * 4 + [_dp, C.c_longlong, _dp]
        lib.ref_galaxy_set.argtypes = [_dp, _dp, _dp, C.c_longlong, _dp, _dp]
        lib.ref_params_parse.argtypes = [C.c_char_p, _dp, _ip]
        lib.ref_normalise.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_int, C.c_int, C.c_int, _dp, _dp]
        vp = C.c_void_p
        lib.ref_count_3d.argtypes = [C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp,
                                     C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _ip]
        _PLAIN = lib
    return _PLAIN


def invp():
    global _INVP
    if _INVP is None:
        path = os.path.join(REF_DIR, "libtwopcf_ref_invp.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        lib = C.CDLL(path)
        vp = C.c_void_p
        lib.ref_n_mask_ints.restype = C.c_int
        lib.ref_invp_read.argtypes = [C.c_char_p, vp, vp, vp, vp, vp, vp, C.c_int, _dp, _dp, _dp, _fp, _fp,
                                      _ip, _lp]
        cat = [vp] * 7 + [C.c_int]
        lib.ref_invp_angular.argtypes = [C.c_char_p, C.c_int] + cat + cat + [C.c_int, _dp, _dp]
        lib.ref_invp_store_angular.argtypes = [C.c_char_p, C.c_char_p, _dp, _dp]
        lib.ref_invp_interp.argtypes = [C.c_char_p, C.c_char_p, _dp, C.c_longlong, _dp]
        lib.ref_invp_count_3d.argtypes = [C.c_char_p, C.c_int, C.c_int] + cat + cat + [C.c_int, _dp, _dp]
        _INVP = lib
    return _INVP


def axis_fields(vmin, vmax, n_bins, base) -> dict:
    out = RefAxisFields()
    plain().ref_axis_fields(vmin, vmax, n_bins, base, C.byref(out))
    return {k: getattr(out, k) for k, _ in RefAxisFields._fields_}


def axis_bin_num(vmin, vmax, n_bins, base, values) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.float32)
    out = np.empty_like(v)
    plain().ref_axis_bin_num(vmin, vmax, n_bins, base, v, v.size, out)
    return out


def axis_centres(vmin, vmax, n_bins, base):
    c = np.empty(n_bins)
    w = np.empty(n_bins)
    plain().ref_axis_centres(vmin, vmax, n_bins, base, c, w)
    return c, w


def comov_dist(omega_m, h, z_min, z_max, z) -> np.ndarray:
    z = np.ascontiguousarray(z, dtype=np.float64)
    out = np.empty_like(z)
    plain().ref_comov_dist(omega_m, h, z_min, z_max, z, z.size, out)
    return out


def galaxy_set(ra, dec, dcom):
    ra = np.ascontiguousarray(ra, np.float64)
    dec = np.ascontiguousarray(dec, np.float64)
    dcom = np.ascontiguousarray(dcom, np.float64)
    x = np.empty((ra.size, 3))
    xn = np.empty((ra.size, 3))
    plain().ref_galaxy_set(ra, dec, dcom, ra.size, x, xn)
    return x, xn


def params_parse(text: str):
    d = np.zeros(18)
    k = np.zeros(18, dtype=np.int32)
    rc = plain().ref_params_parse(text.encode(), d, k)
    if rc != 0:
        raise RuntimeError("ref_params_parse failed")
    return d, k


def normalise(is_auto, w1, jk1, w2, jk2, n_jk, full, sub):
    """In-place JKHists::normalise (src/hist.cpp:290-367) on copies; returns them."""
    full = np.array(full, dtype=np.float64, copy=True)
    sub = np.array(sub, dtype=np.float64, copy=True)
    w1 = _opt(w1, np.float32)
    jk1 = _opt(jk1, np.int32)
    w2 = _opt(w2, np.float32) if w2 is not None else None
    jk2 = _opt(jk2, np.int32) if jk2 is not None else None
    n2 = 0 if w2 is None else w2.size
    plain().ref_normalise(int(is_auto), _ptr(w1), _ptr(jk1), w1.size, _ptr(w2), _ptr(jk2), n2, n_jk,
                          full.size, full, sub.reshape(-1))
    return full, sub


def count_3d(mode, cat1, cat2=None, *, is_auto, n_jk=1, axes, n_threads=0):
    """Run one reference 3-D count.

    cat = dict(xyz=(N,3) f64, unit=(N,3) f64 or None, dcom=(N,) f64 or None,
    w=(N,) f32 or None, jk=(N,) i32 or None).  axes = (min1, max1, base1, nb1,
    min2, max2, base2, nb2) as Params values.  Returns (full[nb], sub[n_jk, nb],
    n_used).
    """
    min1, max1, base1, nb1, min2, max2, base2, nb2 = axes
    nb = nb1 if mode == MONOPOLE else nb1 * nb2
    axp = np.array([min1, max1, base1, min2, max2, base2], dtype=np.float64)

    def prep(cat):
        if cat is None:
            return [None] * 5, 0
        arrs = [_opt(cat["xyz"], np.float64), _opt(cat.get("unit"), np.float64),
                _opt(cat.get("dcom"), np.float64), _opt(cat.get("w"), np.float32),
                _opt(cat.get("jk"), np.int32)]
        return arrs, arrs[0].shape[0]

    a1, n1 = prep(cat1)
    a2, n2 = prep(cat2)
    full = np.zeros(nb)
    sub = np.zeros(nb * n_jk)
    used = np.zeros(2, dtype=np.int32)
    rc = plain().ref_count_3d(mode, int(is_auto), *[_ptr(a) for a in a1], n1, *[_ptr(a) for a in a2], n2,
                              n_jk, axp, nb1, nb2, n_threads, full, sub, used)
    if rc != 0:
        raise RuntimeError("ref_count_3d failed")
    return full, sub.reshape(n_jk, nb), used
