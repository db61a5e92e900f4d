"""The reference's command-line flow around the counts, over the C ABI
(include/two_pcf_b200.h, "command-line flow" part): parameter file,
cosmology, coordinate transforms, the ASCII catalogue reader, the ASCII
result writers and the whole program on a parameter file.

=============================================  ==========================================
reference (lstothert/two_pcf)                  here
=============================================  ==========================================
Params(filename)            src/io.cpp:16      Params.load(path) / Params.parse(text)
Cosmology(...).comov_dist   src/cosmology.cpp  Cosmology(...).comov_dist(z)
Galaxy::set(ra, dec)        src/galaxy.cpp:8   galaxy_set(ra, dec, d_comov)
cartesian reader transform  src/io.cpp:393     cartesian_set(xyz)
read_file(..., "ascii")     src/io.cpp:240     read_ascii(path, coord_system, ...)
generate_sub_filename       src/io.cpp:628     sub_filename(name, region)
output_xi_1D / output_xi_2D src/io.cpp:724     write_xi_ascii(name, binning, DD, DR, RR, ...)
main                        src/main.cpp:11    run_param_file(path)  /  two_pcf_b200/lib/two_pcf
main, inverse-p build       src/main.cpp:51    run_invp(ctx, params, data, randoms)
=============================================  ==========================================

All of it runs on the host except run_param_file, whose pair counts run on
the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import CARTESIAN, EQUATORIAL, FP32_GUARD

__all__ = ["Params", "Cosmology", "galaxy_set", "cartesian_set", "read_ascii", "sub_filename", "write_xi_ascii",
           "run_param_file", "run_invp", "CARTESIAN", "EQUATORIAL", "HostError"]


class HostError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _check(rc: int):
    if rc != 0:
        L = _capi.lib()
        raise HostError(rc, f"{L.tpcf_status_string(abs(rc)).decode()}: {L.tpcf_host_last_error().decode()}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Params:
    """Params (src/io.h:10-86): fields by parameter-file key, e.g. p["s_max"]."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load(cls, path: str) -> "Params":
        h = C.c_void_p()
        _check(_capi.lib().tpcf_params_load(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def parse(cls, text: str) -> "Params":
        h = C.c_void_p()
        _check(_capi.lib().tpcf_params_parse(text.encode(), C.byref(h)))
        return cls(h)

    def get_double(self, key: str) -> float:
        v = C.c_double()
        _check(_capi.lib().tpcf_params_get_double(self._h, key.encode(), C.byref(v)))
        return v.value

    def get_int(self, key: str) -> int:
        v = C.c_int32()
        _check(_capi.lib().tpcf_params_get_int(self._h, key.encode(), C.byref(v)))
        return v.value

    def get_string(self, key: str) -> str:
        L = _capi.lib()
        n = L.tpcf_params_get_string(self._h, key.encode(), None, 0)
        if n < 0:
            _check(n)
        buf = C.create_string_buffer(n + 1)
        L.tpcf_params_get_string(self._h, key.encode(), buf, n + 1)
        return buf.raw[:n].decode()

    def __getitem__(self, key: str):
        for get in (self.get_string, self.get_double, self.get_int):
            try:
                return get(key)
            except HostError:
                pass
        raise KeyError(key)

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_params_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Cosmology:
    """Cosmology(omega_m, h, z_min, z_max, z_save_step, z_oversample)
    (src/cosmology.cpp:11-71); the reference's program uses 1e-4 and 100."""

    def __init__(self, omega_m: float, h: float, z_min: float, z_max: float, z_save_step: float = 1e-4,
                 z_oversample: int = 100):
        hdl = C.c_void_p()
        _check(_capi.lib().tpcf_cosmology_create(float(omega_m), float(h), float(z_min), float(z_max),
                                                 float(z_save_step), int(z_oversample), C.byref(hdl)))
        self._h = hdl

    def comov_dist(self, z) -> np.ndarray:
        z = _f64(z)
        out = np.empty_like(z)
        _check(_capi.lib().tpcf_cosmology_comov_dist(self._h, _ptr(z), z.size, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_cosmology_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def galaxy_set(ra, dec, d_comov):
    """Galaxy::set over arrays: returns (xyz, x_norm)."""
    ra, dec, d = _f64(ra), _f64(dec), _f64(d_comov)
    n = ra.size
    if dec.size != n or d.size != n:
        raise ValueError("ra, dec and d_comov must have one length")
    xyz = np.empty((n, 3))
    xn = np.empty((n, 3))
    _check(_capi.lib().tpcf_galaxy_set(n, _ptr(ra), _ptr(dec), _ptr(d), _ptr(xyz), _ptr(xn)))
    return xyz, xn


def cartesian_set(xyz):
    """The cartesian reader's transform: returns (d_comov, x_norm)."""
    xyz = _f64(xyz).reshape(-1, 3)
    n = xyz.shape[0]
    d = np.empty(n)
    xn = np.empty((n, 3))
    _check(_capi.lib().tpcf_cartesian_set(n, _ptr(xyz), _ptr(d), _ptr(xn)))
    return d, xn


def read_ascii(path: str, coord_system: int = CARTESIAN, use_weights: bool = False, n_jk_regions: int = 1,
               cosmo: Cosmology | None = None) -> dict:
    """read_data_ascii: returns {"xyz", "x_norm", "d_comov", "weight", "jk"}
    (copies), the arguments Catalog takes."""
    L = _capi.lib()
    h = C.c_void_p()
    _check(L.tpcf_read_ascii(str(path).encode(), int(coord_system), int(bool(use_weights)), int(n_jk_regions),
                             cosmo._h if cosmo is not None else None, C.byref(h)))
    try:
        n = L.tpcf_host_catalog_size(h)
        p = [C.c_void_p() for _ in range(5)]
        _check(L.tpcf_host_catalog_arrays(h, *[C.byref(x) for x in p]))

        def view(ptr, ctype, count, dtype):
            if count == 0:
                return np.empty(0, dtype)
            arr = C.cast(ptr, C.POINTER(ctype * count)).contents
            return np.frombuffer(arr, dtype=dtype, count=count).copy()

        return {"xyz": view(p[0], C.c_double, 3 * n, np.float64).reshape(n, 3),
                "x_norm": view(p[1], C.c_double, 3 * n, np.float64).reshape(n, 3),
                "d_comov": view(p[2], C.c_double, n, np.float64),
                "weight": view(p[3], C.c_float, n, np.float32),
                "jk": view(p[4], C.c_int32, n, np.int32)}
    finally:
        L.tpcf_host_catalog_destroy(h)


def sub_filename(filename: str, region: int) -> str:
    L = _capi.lib()
    n = L.tpcf_sub_filename(filename.encode(), int(region), None, 0)
    if n < 0:
        _check(n)
    buf = C.create_string_buffer(n + 1)
    L.tpcf_sub_filename(filename.encode(), int(region), buf, n + 1)
    return buf.raw[:n].decode()


def write_xi_ascii(filename: str, binning, dd, dr, rr, dd_sub=None, dr_sub=None, rr_sub=None):
    """output_xi_1D / output_xi_2D with output type "ascii"."""
    arrs = [_f64(a).reshape(-1) if a is not None else None for a in (dd, dr, rr, dd_sub, dr_sub, rr_sub)]
    for a in arrs[:3]:
        if a.size != binning.nb:
            raise ValueError("full histograms must have binning.nb values")
    for a in arrs[3:]:
        if a is not None and a.size != binning.nb * binning.n_jk:
            raise ValueError("region histograms must have n_jk * nb values")
    _check(_capi.lib().tpcf_write_xi_ascii(str(filename).encode(), binning._h, *[_ptr(a) for a in arrs]))


def run_param_file(path: str, device: int = 0, precision: int = FP32_GUARD, log: bool = False,
                   check_fp64: bool = False, summary: str | None = None):
    """The reference's program on a parameter file, counts on the GPU.
    summary: path of a JSON run summary (tpcf_run_param_file_report);
    check_fp64: also count on the plain FP64 path and report every output's
    difference from it in the summary.  Returns the summary as a dict when
    one was written, else None."""
    L = _capi.lib()
    if summary is None and not check_fp64:
        _check(L.tpcf_run_param_file(str(path).encode(), int(device), int(precision), int(bool(log))))
        return None
    rc = L.tpcf_run_param_file_report(str(path).encode(), int(device), int(precision), int(bool(log)),
                                      int(bool(check_fp64)), None if summary is None else str(summary).encode())
    _check(rc)
    if summary is None:
        return None
    import json
    with open(summary) as f:
        return json.load(f)


def run_invp(ctx, params: Params, data, randoms, precision: int = FP32_GUARD, dither: bool = False,
             log: bool = False) -> dict:
    """The inverse-p program after reading (tpcf_run_invp): angular stage on
    the GPU, then the 3-D inverse-p counts and ASCII outputs the parameters
    ask for.  data / randoms are two_pcf_b200.Catalog objects with bitmasks.
    Returns the angular histograms {"dd", "dd_invp", "dr", "dr_invp"}, each
    (full[nt], regions[n_jk, nt]) in the reference's convention."""
    nt = params.get_int("theta_n_bins")
    n_jk = params.get_int("n_jk_regions")
    out = np.zeros((4, 1 + n_jk, nt))
    _check(_capi.lib().tpcf_run_invp(ctx._h, params._h, data._h, randoms._h, int(precision), int(bool(dither)),
                                     _ptr(out), int(bool(log))))
    return {k: (out[i, 0].copy(), out[i, 1:].copy()) for i, k in enumerate(("dd", "dd_invp", "dr", "dr_invp"))}
