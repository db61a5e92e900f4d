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
_PLAIN: dict = {}
_INVP: dict = {}

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
    """variant: plain, midpoint (plain build without _ANGULAR_PI_DEFN), invp,
    invp_dither (_USE_DITHER_WEIGHTS), invp4 (_N_MASK_INTS = 4)."""
    return os.path.exists(os.path.join(REF_DIR, f"libtwopcf_ref_{variant}.so"))


def _opt(arr, dtype):
    """None -> NULL pointer, else a contiguous array of dtype."""
    if arr is None:
        return None
    return np.ascontiguousarray(arr, dtype=dtype)


def _ptr(arr):
    return None if arr is None else arr.ctypes.data_as(C.c_void_p)


def plain(variant: str = "plain"):
    if variant not in _PLAIN:
        path = os.path.join(REF_DIR, f"libtwopcf_ref_{variant}.so")
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
        lib.ref_read_ascii.argtypes = [C.c_char_p, C.c_char_p, C.c_longlong, vp, vp, vp, vp, vp]
        lib.ref_read_ascii.restype = C.c_longlong
        lib.ref_write_xi.argtypes = [C.c_char_p, C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                     _dp]
        _PLAIN[variant] = lib
    return _PLAIN[variant]


def invp(variant: str = "invp"):
    if variant not in _INVP:
        path = os.path.join(REF_DIR, f"libtwopcf_ref_{variant}.so")
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
        lib.ref_invp_correlate.argtypes = [C.c_char_p] + cat + cat + [C.c_int]
        lib.ref_invp_set_dither.argtypes = [vp, vp]
        lib.ref_has_dither.restype = C.c_int
        _INVP[variant] = lib
    return _INVP[variant]


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


def read_ascii(param_text: str, path: str) -> dict:
    """read_file(path, "ascii", cosmo, Params(param_text)): the Galaxy fields."""
    L = plain()
    n = L.ref_read_ascii(param_text.encode(), str(path).encode(), -1, None, None, None, None, None)
    if n < 0:
        raise RuntimeError("ref_read_ascii failed")
    out = {"xyz": np.empty((n, 3)), "x_norm": np.empty((n, 3)), "d_comov": np.empty(n),
           "weight": np.empty(n, np.float32), "jk": np.empty(n, np.int32)}
    L.ref_read_ascii(param_text.encode(), str(path).encode(), n, *[_ptr(out[k]) for k in
                                                                  ("xyz", "x_norm", "d_comov", "weight", "jk")])
    return out


def write_xi(filename: str, mode: int, axp, nb1: int, nb2: int, n_jk: int, dd, dr, rr, dd_sub, dr_sub, rr_sub):
    """output_xi_1D (mode 0) / output_xi_2D (1 sigma-pi, 2 s-mu), file type "ascii"."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (dd, dr, rr, dd_sub, dr_sub, rr_sub)]
    plain().ref_write_xi(str(filename).encode(), int(mode), np.ascontiguousarray(axp, dtype=np.float64), nb1, nb2,
                         n_jk, *arrs)


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


def count_3d(mode, cat1, cat2=None, *, is_auto, n_jk=1, axes, n_threads=0, variant="plain"):
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
    rc = plain(variant).ref_count_3d(mode, int(is_auto), *[_ptr(a) for a in a1], n1, *[_ptr(a) for a in a2], n2,
                              n_jk, axp, nb1, nb2, n_threads, full, sub, used)
    if rc != 0:
        raise RuntimeError("ref_count_3d failed")
    return full, sub.reshape(n_jk, nb), used


# ----------------------------------------------------------- inverse-p build
# Every function takes variant = "invp" (the build with _N_MASK_INTS = 32),
# "invp_dither" (plus _USE_DITHER_WEIGHTS) or "invp4" (_N_MASK_INTS = 4).

N_MASK_INTS_INVP = 32  # _N_MASK_INTS of the default inverse-p build (oracle/build_ref.sh)


def n_mask_ints(variant: str = "invp") -> int:
    return int(invp(variant).ref_n_mask_ints())


def invp_params(*, n_jk=1, healpix_order=5, theta_max=0.175, theta_n_bins=40, theta_log_base=1.6,
                n_bitwise_runs=2048, monopole=(0.0, 100.0, 30, 1.3), sigma=(0.0, 50.0, 50, 1.0),
                pi=(0.0, 50.0, 50, 1.0), s=(0.0, 100.0, 40, 1.3), mu_n_bins=50,
                dd_file="ang_dd.hdf5", ddi_file="ang_dd_invp.hdf5", dr_file="ang_dr.hdf5",
                dri_file="ang_dr_invp.hdf5", plot=(0, 0, 0), calculate=(0, 0, 0, 0),
                out_files=("mono.txt", "sp.txt", "smu.txt"), coord_system="cartesian") -> str:
    """A parameter file for the inverse-p build with every key set (the
    reference leaves absent keys uninitialised, src/io.cpp:16-237)."""
    kv = {
        "data_filename": "data.hdf5", "data_file_type": "hdf5", "random_filename": "rand.hdf5",
        "random_file_type": "hdf5", "coord_system": coord_system, "ra_x_dataset_name": "x",
        "dec_y_dataset_name": "y", "z_z_dataset_name": "z", "weight_dataset_name": "w",
        "jk_dataset_name": "jk", "bitwise_weight_dataset_name": "bw", "dither_weight_dataset_name": "dw",
        "use_weights": 1, "n_jk_regions": n_jk, "omega_m": 0.25, "h": 1.0, "z_min": 0.0, "z_max": 1.0,
        "plot_monopole": plot[0], "plot_sigma_pi": plot[1], "plot_s_mu": plot[2],
        "monopole_filename": out_files[0],
        "monopole_output_type": "ascii", "monopole_min": monopole[0], "monopole_max": monopole[1],
        "monopole_n_bins": monopole[2], "monopole_log_base": monopole[3], "sigma_pi_filename": out_files[1],
        "sigma_pi_output_type": "ascii", "sigma_min": sigma[0], "sigma_max": sigma[1],
        "sigma_n_bins": sigma[2], "sigma_log_base": sigma[3], "pi_min": pi[0], "pi_max": pi[1],
        "pi_n_bins": pi[2], "pi_log_base": pi[3], "s_mu_filename": out_files[2], "s_mu_output_type": "ascii",
        "s_min": s[0], "s_max": s[1], "s_n_bins": s[2], "s_log_base": s[3], "mu_n_bins": mu_n_bins,
        "n_threads": 1, "healpix_order": healpix_order, "theta_max": repr(float(theta_max)),
        "theta_n_bins": theta_n_bins, "theta_log_base": theta_log_base, "n_bitwise_runs": n_bitwise_runs,
        "calculate_angular_dd": calculate[0], "calculate_angular_dd_invpweights": calculate[1],
        "calculate_angular_dr": calculate[2], "calculate_angular_dr_invpweights": calculate[3],
        "angular_dd_filename": dd_file,
        "angular_dd_invpweights_filename": ddi_file, "angular_dr_filename": dr_file,
        "angular_dr_invpweights_filename": dri_file,
    }
    return "".join(f"{k} = {v}\n" for k, v in kv.items())


def _invp_cat(cat, variant="invp"):
    """cat dict -> the 7 pointers + n of the harness (xyz, unit, dcom, w, iw,
    jk, masks[n x _N_MASK_INTS] object-major)."""
    if cat is None:
        return [None] * 7 + [0], []
    arrs = [_opt(cat["xyz"], np.float64), _opt(cat.get("unit"), np.float64), _opt(cat.get("dcom"), np.float64),
            _opt(cat.get("w"), np.float32), _opt(cat.get("iw"), np.float32), _opt(cat.get("jk"), np.int32),
            _opt(cat.get("masks"), np.int64)]
    if arrs[6] is not None:
        assert arrs[6].shape == (arrs[0].shape[0], n_mask_ints(variant))
    return [_ptr(a) for a in arrs] + [arrs[0].shape[0]], arrs


class _Dither:
    """Sets the harness's dither masks (cat dict key "dmasks") for one call."""

    def __init__(self, variant, cat1, cat2):
        self.L = invp(variant)
        self.on = bool(self.L.ref_has_dither())
        self.keep = [None if c is None or c.get("dmasks") is None else _opt(c["dmasks"], np.int64)
                     for c in (cat1, cat2)]

    def __enter__(self):
        if self.on:
            self.L.ref_invp_set_dither(_ptr(self.keep[0]), _ptr(self.keep[1]))
        return self

    def __exit__(self, *exc):
        if self.on:
            self.L.ref_invp_set_dither(None, None)
        return False


def invp_angular(params: str, kind, cat1, cat2=None, *, n_jk, n_bins, n_threads=0, variant="invp"):
    """Angular stage: kind 0 DD, 1 DD inverse-p, 2 DR, 3 DR inverse-p
    (src/correlators_invpweight.cpp:713-982).  Returns (full, sub[n_jk, nb])
    after invert_jk_hists and (auto) x2."""
    p1, keep1 = _invp_cat(cat1, variant)
    p2, keep2 = _invp_cat(cat2, variant)
    full = np.zeros(n_bins)
    sub = np.zeros(n_bins * n_jk)
    with _Dither(variant, cat1, cat2):
        rc = invp(variant).ref_invp_angular(params.encode(), int(kind), *p1, *p2, n_threads, full, sub)
    if rc != 0:
        raise RuntimeError("ref_invp_angular failed")
    return full, sub.reshape(n_jk, n_bins)


def invp_store_angular(params: str, fname: str, full, sub, variant="invp"):
    full = np.ascontiguousarray(full, np.float64)
    sub = np.ascontiguousarray(sub, np.float64).reshape(-1)
    if invp(variant).ref_invp_store_angular(params.encode(), fname.encode(), full, sub) != 0:
        raise RuntimeError("ref_invp_store_angular failed")


def invp_interp(num_file: str, den_file: str, values, variant="invp") -> np.ndarray:
    v = np.ascontiguousarray(values, np.float64)
    out = np.empty_like(v)
    if invp(variant).ref_invp_interp(num_file.encode(), den_file.encode(), v, v.size, out) != 0:
        raise RuntimeError("ref_invp_interp failed")
    return out


def invp_count_3d(params: str, mode, how, cat1, cat2=None, *, n_jk, nb, n_threads=0, variant="invp"):
    """3-D counts of the inverse-p build: how = 1 DD with inverse-p weights,
    0 DR with the angular DR up-weight, 2 plain auto count.  The angular
    histograms must have been stored under the params' file names."""
    p1, keep1 = _invp_cat(cat1, variant)
    p2, keep2 = _invp_cat(cat2, variant)
    full = np.zeros(nb)
    sub = np.zeros(nb * n_jk)
    with _Dither(variant, cat1, cat2):
        rc = invp(variant).ref_invp_count_3d(params.encode(), int(mode), int(how), *p1, *p2, n_threads, full, sub)
    if rc != 0:
        raise RuntimeError("ref_invp_count_3d failed")
    return full, sub.reshape(n_jk, nb)


def invp_correlate(params: str, data, randoms, *, n_threads=0, variant="invp"):
    """The inverse-p program after reading: calc_angular_upweight, then the
    auto_correlate_*_invpweights the params' plot flags select, writing the
    ASCII files the params name."""
    p1, keep1 = _invp_cat(data, variant)
    p2, keep2 = _invp_cat(randoms, variant)
    with _Dither(variant, data, randoms):
        rc = invp(variant).ref_invp_correlate(params.encode(), *p1, *p2, n_threads)
    if rc != 0:
        raise RuntimeError("ref_invp_correlate failed")


def invp_read(params: str, c1, c2, c3, w, jk, masks, dmasks=None, variant="invp"):
    """read_file(..., "hdf5", ...) of the inverse-p build on in-memory columns
    (src/io.cpp:418-593), including the bitwise-weight IIP rescaling.  masks
    and dmasks are object-major (n x _N_MASK_INTS).  Returns the Galaxy fields."""
    L = invp(variant)
    n = len(c1)
    nm = n_mask_ints(variant)
    m = np.ascontiguousarray(np.asarray(masks, np.int64).reshape(n, nm).T)  # dataset-major
    cols = [np.ascontiguousarray(c, np.float64) for c in (c1, c2, c3)]
    wv = None if w is None else np.ascontiguousarray(w, np.float64)
    jv = None if jk is None else np.ascontiguousarray(jk, np.int32)
    out = {"xyz": np.empty((n, 3)), "x_norm": np.empty((n, 3)), "d_comov": np.empty(n),
           "weight": np.empty(n, np.float32), "input_weight": np.empty(n, np.float32), "jk": np.empty(n, np.int32),
           "masks": np.empty((n, nm), np.int64)}
    d = {"dmasks": dmasks} if dmasks is not None else {}
    with _Dither(variant, d, None):
        rc = L.ref_invp_read(params.encode(), *[_ptr(c) for c in cols], _ptr(wv), _ptr(jv), _ptr(m), n, out["xyz"],
                             out["x_norm"], out["d_comov"], out["weight"], out["input_weight"], out["jk"],
                             out["masks"])
    if rc != 0:
        raise RuntimeError("ref_invp_read failed")
    return out


def invp_reset(variant="invp"):
    """Forget every in-memory HDF5 file of the stand-in library."""
    invp(variant).ref_h5_reset()
