"""TEST INFRASTRUCTURE ONLY — ctypes access to the CPU restatement.

``oracle/tpcf_oracle.c`` restates the reference's pair-counting algorithm in
plain C (built by ``oracle/build_oracle.sh`` into ``oracle/lib/``).  The
tests use it as the parity checker for the CUDA path and pin it against the
reference itself (``oracle/refl.py``) and the committed golden fixtures.
Nothing in the product imports this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtpcf_oracle.so")
_LIB = None

MONOPOLE, SIGMA_PI, S_MU = 0, 1, 2
W_PLAIN, W_INVP_DD, W_INVP_DR = 0, 1, 2


class OrcAxis(C.Structure):
    _fields_ = [("n_bins", C.c_int), ("log_binning", C.c_int), ("min", C.c_float),
                ("minus_min", C.c_float), ("max", C.c_float), ("step", C.c_float),
                ("inv_step", C.c_float), ("base", C.c_float), ("inv_log_of_base", C.c_float),
                ("inv_log_step", C.c_float)]


class OrcCat(C.Structure):
    _fields_ = [("n", C.c_int), ("xyz", C.c_void_p), ("unit", C.c_void_p), ("dcom", C.c_void_p),
                ("w", C.c_void_p), ("iw", C.c_void_p), ("jk", C.c_void_p), ("masks", C.c_void_p),
                ("n_mask", C.c_int), ("dmasks", C.c_void_p)]


class OrcUpweight(C.Structure):
    _fields_ = [("ax", OrcAxis), ("bins", C.c_void_p), ("centre", C.c_void_p)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} missing: run oracle/build_oracle.sh")
        L = C.CDLL(LIB_PATH)
        L.orc_axis_init.argtypes = [C.POINTER(OrcAxis), C.c_double, C.c_double, C.c_int, C.c_double]
        L.orc_axis_bin_num.argtypes = [C.POINTER(OrcAxis), C.c_float]
        L.orc_axis_bin_num.restype = C.c_float
        L.orc_axis_bin_centre.argtypes = [C.POINTER(OrcAxis), C.c_int]
        L.orc_axis_bin_centre.restype = C.c_double
        L.orc_interp.argtypes = [C.POINTER(OrcUpweight), C.c_double]
        L.orc_interp.restype = C.c_double
        L.orc_count_3d.argtypes = [C.c_int, C.c_int, C.POINTER(OrcCat), C.POINTER(OrcCat), C.c_int,
                                   C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(OrcUpweight), C.c_int,
                                   C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_count_backward.argtypes = [C.c_int, C.c_int, C.POINTER(OrcCat), C.POINTER(OrcCat), C.c_void_p,
                                         C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_count_angular.argtypes = [C.c_int, C.POINTER(OrcCat), C.POINTER(OrcCat), C.c_int, C.c_double,
                                        C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_normalise_auto.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p]
        L.orc_normalise_cross.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                          C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_ls.argtypes = [C.c_double] * 3
        L.orc_ls.restype = C.c_double
        L.orc_partition.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_partition.restype = C.c_int
        L.orc_set_variant.argtypes = [C.c_int, C.c_int]
        _LIB = L
    return _LIB


def _arr(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return None if a is None else a.ctypes.data


class Cat:
    """Holds a catalogue's arrays alive and exposes the OrcCat view."""

    def __init__(self, xyz, unit=None, dcom=None, w=None, iw=None, jk=None, masks=None, dmasks=None):
        self.xyz = _arr(xyz, np.float64)
        n = self.xyz.shape[0]
        if unit is None:
            d = np.sqrt((self.xyz ** 2).sum(1))
            unit = self.xyz / d[:, None]
        self.unit = _arr(unit, np.float64)
        self.dcom = _arr(dcom, np.float64)
        self.w = _arr(w, np.float32)
        self.iw = _arr(iw, np.float32)
        self.jk = _arr(jk, np.int32)
        self.masks = _arr(masks, np.int64)
        self.dmasks = _arr(dmasks, np.int64)
        n_mask = 0 if self.masks is None else self.masks.reshape(n, -1).shape[1]
        self.c = OrcCat(n, _p(self.xyz), _p(self.unit), _p(self.dcom), _p(self.w), _p(self.iw), _p(self.jk),
                        _p(self.masks), n_mask, _p(self.dmasks))


class variant:
    """Context manager selecting a build variant of the reference for the
    oracle's counts: los_midpoint (pi without _ANGULAR_PI_DEFN) and/or
    dither (_USE_DITHER_WEIGHTS)."""

    def __init__(self, los_midpoint=False, dither=False):
        self.args = (int(los_midpoint), int(dither))

    def __enter__(self):
        lib().orc_set_variant(*self.args)
        return self

    def __exit__(self, *exc):
        lib().orc_set_variant(0, 0)
        return False


def axis(vmin, vmax, n_bins, base) -> OrcAxis:
    ax = OrcAxis()
    lib().orc_axis_init(C.byref(ax), vmin, vmax, n_bins, base)
    return ax


def partition(dcom) -> np.ndarray:
    d = np.ascontiguousarray(dcom, np.float64)
    perm = np.empty(d.size, np.int32)
    n = lib().orc_partition(d.ctypes.data, d.size, perm.ctypes.data)
    return perm[:n]


def make_upweight(vmin, vmax, n_bins, base, bins):
    """Up-weight table for orc_interp; one spare entry past the last bin."""
    ax = axis(vmin, vmax, n_bins, base)
    b = np.zeros(n_bins + 1)
    b[:n_bins] = bins
    b[n_bins] = bins[-1]
    cen = np.array([lib().orc_axis_bin_centre(C.byref(ax), i) for i in range(n_bins + 1)])
    up = OrcUpweight(ax, b.ctypes.data, cen.ctypes.data)
    up._keep = (b, cen)
    return up


def count_3d(mode, a: Cat, b: Cat | None, *, is_auto, n_jk=1, axes, weight_kind=W_PLAIN, up=None,
             n_runs=0, n_threads=0):
    """Same contract as oracle.refl.count_3d: histograms after inversion (and x2 for auto)."""
    min1, max1, base1, nb1, min2, max2, base2, nb2 = axes
    nb = nb1 if mode == MONOPOLE else nb1 * nb2
    axp = np.array([min1, max1, base1, min2, max2, base2], np.float64)
    full = np.zeros(nb)
    sub = np.zeros(nb * n_jk)
    used = np.zeros(2, np.int32)
    bc = b.c if b is not None else a.c
    lib().orc_count_3d(mode, int(is_auto), C.byref(a.c), C.byref(bc), n_jk, axp.ctypes.data, nb1, nb2,
                       weight_kind, C.byref(up) if up is not None else None, n_runs, n_threads, full.ctypes.data,
                       sub.ctypes.data, used.ctypes.data)
    return full, sub.reshape(n_jk, nb), used


def count_angular(kind, a: Cat, b: Cat | None, *, n_jk, theta_max, n_theta, theta_log_base, n_runs=0,
                  n_threads=0):
    full = np.zeros(n_theta)
    sub = np.zeros(n_theta * n_jk)
    bc = b.c if b is not None else a.c
    lib().orc_count_angular(kind, C.byref(a.c), C.byref(bc), n_jk, theta_max, n_theta, theta_log_base, n_runs,
                            n_threads, full.ctypes.data, sub.ctypes.data)
    return full, sub.reshape(n_jk, n_theta)


def count_backward(mode, a: Cat, b: Cat | None, *, is_auto, axes, G, n_threads=0):
    """FP64 CPU adjoint of a plain-weight 3-D count: per-object dL/dw for
    G = dL/d(raw full histogram, unordered pairs).  Returns (grad_a, grad_b)."""
    min1, max1, base1, nb1, min2, max2, base2, nb2 = axes
    axp = np.array([min1, max1, base1, min2, max2, base2], np.float64)
    G = np.ascontiguousarray(G, np.float64)
    ga = np.zeros(a.c.n)
    gb = np.zeros(b.c.n if b is not None else 1)
    bc = b.c if b is not None else a.c
    lib().orc_count_backward(mode, int(is_auto), C.byref(a.c), C.byref(bc), axp.ctypes.data, nb1, nb2,
                             G.ctypes.data, n_threads, ga.ctypes.data, gb.ctypes.data)
    return ga, (None if is_auto else gb)
