"""two_pcf_b200 — B200-native grid-binned pair counting for the two-point
correlation function (the hot path of lstothert/two_pcf).

Python mirror of the reference's counting interface, over the C ABI of
include/two_pcf_b200.h:

===========================================  =====================================
reference (lstothert/two_pcf)                here
===========================================  =====================================
GalaxyBoxes(gals, n, other, n_other, rmax)   Catalog(ctx, xyz, ...)  (src/boxes.h:30)
Hist / Hist2D(min, max, n, base, ...)        Binning(ctx, mode, ax1, ax2, n_jk)
auto_pair_count_{monopole,sigma_pi,s_mu}     auto_pair_count(ctx, cat, binning)
cross_pair_count_{monopole,sigma_pi,s_mu}    cross_pair_count(ctx, a, b, binning)
JKHists::normalise                           normalise_auto / normalise_cross
ls_estimator                                 ls_estimator
===========================================  =====================================

The counting functions return (full_hist, sub_hist) exactly as the reference
leaves JKHists after invert_jk_hists() and, for auto counts, multiply_hists(2.0)
(src/correlators.cpp:76-77).  There is no CPU fallback: every count runs the
CUDA kernels in two_pcf_b200/lib/libtpcf_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import (ANGULAR, BATCH_AUTOTUNE, BATCH_DD, BATCH_DR, FP32_GUARD, FP64, LOS_ANGULAR, LOS_MIDPOINT,
                    MONOPOLE, S_MU, SIGMA_PI, WEIGHTS_INVP_DD, WEIGHTS_INVP_DD_DITHER, WEIGHTS_INVP_DR, WEIGHTS_PLAIN,
                    AxisSpec, Stats, WeightSpec)

__all__ = ["Context", "Catalog", "Binning", "TpcfError", "Weights", "count", "auto_pair_count", "cross_pair_count",
           "count_weighted", "pair_count_weighted", "upweight_eval", "count_backward", "normalise_auto",
           "normalise_cross",
           "ls_estimator", "MONOPOLE", "SIGMA_PI", "S_MU", "ANGULAR", "FP32_GUARD", "FP64", "WEIGHTS_PLAIN",
           "WEIGHTS_INVP_DD", "WEIGHTS_INVP_DR", "WEIGHTS_INVP_DD_DITHER", "LOS_ANGULAR", "LOS_MIDPOINT", "iip_weights",
           "Batch", "BATCH_DD", "BATCH_DR", "BATCH_AUTOTUNE", "count_shard", "shard_combine", "count_sharded",
           "count_many"]


class TpcfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def _check(rc: int, ctx=None):
    if rc != 0:
        L = _capi.lib()
        detail = L.tpcf_last_error(ctx._h).decode() if ctx is not None and ctx._h else ""
        raise TpcfError(rc, f"{L.tpcf_status_string(rc).decode()}: {detail}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One CUDA device; owns a stream.  Replaces the OpenMP set-up of src/main.cpp:29-35."""

    def __init__(self, device: int = 0, refinement: int = 0):
        L = _capi.lib()
        h = C.c_void_p()
        rc = L.tpcf_create(int(device), C.byref(h))
        if rc != 0:
            raise TpcfError(rc, f"tpcf_create(device={device}) failed: {L.tpcf_status_string(rc).decode()}")
        self._h = h
        if refinement:
            _check(L.tpcf_set_refinement(self._h, int(refinement)), self)

    def set_refinement(self, m: int):
        _check(_capi.lib().tpcf_set_refinement(self._h, int(m)), self)

    def set_autotune(self, on: bool = True):
        """Autotuning of counts (tpcf_set_autotune): the first count of each
        class probes the refinement and kernel configuration; later counts of
        the class use the fastest."""
        _check(_capi.lib().tpcf_set_autotune(self._h, int(bool(on))), self)

    def set_kernel_config(self, cfg: int):
        """Kernel configuration of the plain-weight FP32+guard kernels (0, 1;
        -1 automatic)."""
        _check(_capi.lib().tpcf_set_kernel_config(self._h, int(cfg)), self)

    def set_cross_order(self, order: int):
        """Order of plain-weight cross counts (tpcf_set_cross_order): 0 a's
        points against b's, 1 the reverse, -1 automatic."""
        _check(_capi.lib().tpcf_set_cross_order(self._h, int(order)), self)

    def autotune_table(self) -> list:
        """The autotuner's choices so far (tpcf_autotune_describe)."""
        import json
        L = _capi.lib()
        n = L.tpcf_autotune_describe(self._h, None, 0)
        if n < 0:
            _check(int(-n), self)
        buf = C.create_string_buffer(int(n) + 1)
        L.tpcf_autotune_describe(self._h, buf, int(n) + 1)
        return json.loads(buf.value.decode())

    def set_stream(self, stream_handle: int | None):
        _check(_capi.lib().tpcf_set_stream(self._h, C.c_void_p(stream_handle or 0)), self)

    def synchronize(self):
        _check(_capi.lib().tpcf_synchronize(self._h), self)

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Catalog:
    """A catalogue resident on the device (Galaxy fields of src/galaxy.h:16-35)."""

    def __init__(self, ctx: Context, xyz, x_norm=None, d_comov=None, weight=None, input_weight=None,
                 jk_region=None, n_jk_regions: int = 1, bitmask=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        n = xyz.shape[0]
        arrs = {
            "x_norm": None if x_norm is None else np.ascontiguousarray(x_norm, np.float64).reshape(n, 3),
            "d_comov": None if d_comov is None else np.ascontiguousarray(d_comov, np.float64).reshape(n),
            "weight": None if weight is None else np.ascontiguousarray(weight, np.float32).reshape(n),
            "input_weight": None if input_weight is None else np.ascontiguousarray(input_weight, np.float32).reshape(n),
            "jk": None if jk_region is None else np.ascontiguousarray(jk_region, np.int32).reshape(n),
            "mask": None if bitmask is None else np.ascontiguousarray(bitmask, np.int64).reshape(n, -1),
        }
        n_mask = 0 if arrs["mask"] is None else arrs["mask"].shape[1]
        h = C.c_void_p()
        rc = _capi.lib().tpcf_catalog_create(ctx._h, n, _ptr(xyz), _ptr(arrs["x_norm"]), _ptr(arrs["d_comov"]),
                                             _ptr(arrs["weight"]), _ptr(arrs["input_weight"]), _ptr(arrs["jk"]),
                                             int(n_jk_regions), _ptr(arrs["mask"]), n_mask, C.byref(h))
        _check(rc, ctx)
        self._h = h
        self.ctx = ctx
        self.n = n
        self.n_jk = int(n_jk_regions)

    @property
    def n_used(self) -> int:
        return int(_capi.lib().tpcf_catalog_n_used(self._h))

    def set_weights(self, weight):
        """Replace Galaxy::weight of every point (device copy and cached cell grids)."""
        w = np.ascontiguousarray(weight, np.float32).reshape(self.n)
        _check(_capi.lib().tpcf_catalog_set_weights(self._h, _ptr(w)), self.ctx)

    def set_dither_masks(self, dither_mask):
        """Galaxy::dither_mask (the _USE_DITHER_WEIGHTS build): n x n_mask_ints int64."""
        m = np.ascontiguousarray(dither_mask, np.int64).reshape(self.n, -1)
        _check(_capi.lib().tpcf_catalog_set_dither_masks(self._h, _ptr(m)), self.ctx)

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_catalog_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _axis(spec) -> AxisSpec:
    if isinstance(spec, AxisSpec):
        return spec
    vmin, vmax, base, n = spec
    return AxisSpec(float(vmin), float(vmax), float(base), int(n))


class Binning:
    """Histogram definition: mode plus (min, max, log_base, n_bins) axes."""

    def __init__(self, ctx: Context | None, mode: int, ax1, ax2=None, n_jk_regions: int = 1):
        a1 = _axis(ax1)
        a2 = _axis(ax2) if ax2 is not None else None
        h = C.c_void_p()
        rc = _capi.lib().tpcf_binning_create(ctx._h if ctx is not None else None, int(mode), C.byref(a1), C.byref(a2) if a2 is not None else None,
                                             int(n_jk_regions), C.byref(h))
        _check(rc, ctx)
        self._h = h
        self.ctx = ctx
        self.mode = mode
        self.n_jk = int(n_jk_regions)
        self.nb = int(_capi.lib().tpcf_binning_total_bins(h))
        self.shape = (a1.n_bins,) if mode in (MONOPOLE, ANGULAR) else (a1.n_bins, a2.n_bins)

    def set_line_of_sight(self, line_of_sight: int):
        """LOS_ANGULAR (the reference's default _ANGULAR_PI_DEFN build) or
        LOS_MIDPOINT (its build without it, src/correlators.cpp:172-182)."""
        _check(_capi.lib().tpcf_binning_set_line_of_sight(self._h, int(line_of_sight)), self.ctx)

    def thresholds(self, axis: int = 1) -> np.ndarray:
        n = _capi.lib().tpcf_binning_thresholds(self._h, axis, None, 0)
        out = np.empty(n, np.float32)
        _capi.lib().tpcf_binning_thresholds(self._h, axis, _ptr(out), n)
        return out

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_binning_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def count(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, precision: int = FP32_GUARD,
          with_regions: bool = True):
    """Raw count: (full[nb], regions[n_jk, nb] or None, stats dict), not inverted nor doubled."""
    full = np.zeros(binning.nb)
    reg = np.zeros((binning.n_jk, binning.nb)) if with_regions else None
    st = Stats()
    rc = _capi.lib().tpcf_count(ctx._h, a._h, b._h if b is not None else None, binning._h, int(precision),
                                _ptr(full), _ptr(reg), C.byref(st))
    _check(rc, ctx)
    return full, reg, st.as_dict()


def auto_pair_count(ctx: Context, cat: Catalog, binning: Binning, precision: int = FP32_GUARD):
    """auto_pair_count_{monopole,sigma_pi,s_mu} (src/correlators.cpp:11-78, :190-239, :345-393)."""
    full = np.zeros(binning.nb)
    sub = np.zeros((binning.n_jk, binning.nb))
    st = Stats()
    _check(_capi.lib().tpcf_auto_pair_count(ctx._h, cat._h, binning._h, int(precision), _ptr(full), _ptr(sub),
                                            C.byref(st)), ctx)
    return full, sub, st.as_dict()


def cross_pair_count(ctx: Context, a: Catalog, b: Catalog, binning: Binning, precision: int = FP32_GUARD):
    """cross_pair_count_{monopole,sigma_pi,s_mu} (src/correlators.cpp:80-125, :241-278, :395-430)."""
    full = np.zeros(binning.nb)
    sub = np.zeros((binning.n_jk, binning.nb))
    st = Stats()
    _check(_capi.lib().tpcf_cross_pair_count(ctx._h, a._h, b._h, binning._h, int(precision), _ptr(full), _ptr(sub),
                                             C.byref(st)), ctx)
    return full, sub, st.as_dict()


def normalise_auto(cat: Catalog, full, sub):
    """JKHists::normalise(cat, n_gals) (src/hist.cpp:290-321); returns normalised copies."""
    full = np.array(full, np.float64, copy=True)
    sub = np.array(sub, np.float64, copy=True)
    _check(_capi.lib().tpcf_normalise_auto(cat._h, full.size, _ptr(full), _ptr(sub)))
    return full, sub


def normalise_cross(a: Catalog, b: Catalog, full, sub):
    """JKHists::normalise(cat1, n1, cat2, n2) (src/hist.cpp:323-367); returns normalised copies."""
    full = np.array(full, np.float64, copy=True)
    sub = np.array(sub, np.float64, copy=True)
    _check(_capi.lib().tpcf_normalise_cross(a._h, b._h, full.size, _ptr(full), _ptr(sub)))
    return full, sub


def ls_estimator(dd, dr, rr):
    """Landy-Szalay estimator (src/io.cpp:643-651), elementwise."""
    dd, dr, rr = np.broadcast_arrays(np.asarray(dd, float), np.asarray(dr, float), np.asarray(rr, float))
    f = _capi.lib().tpcf_ls_estimator
    out = np.array([f(float(x), float(y), float(z)) for x, y, z in zip(dd.ravel(), dr.ravel(), rr.ravel())])
    return out.reshape(dd.shape)


class Weights:
    """Pair weighting of the inverse-p build (tpcf_weight_spec).

    weighting: WEIGHTS_PLAIN, WEIGHTS_INVP_DD or WEIGHTS_INVP_DR.  For 3-D
    inverse-p counts, theta_axis = (0, 1 - cos(theta_max), theta_log_base,
    theta_n_bins) and the angular up-weight is up_numerator / up_denominator
    bin by bin (the angular DD and DD-inverse-p full histograms for DD, DR and
    DR-inverse-p for DR)."""

    def __init__(self, weighting: int = WEIGHTS_PLAIN, n_bitwise_runs: int = 0, theta_axis=None,
                 up_numerator=None, up_denominator=None):
        self._num = None if up_numerator is None else np.ascontiguousarray(up_numerator, np.float64)
        self._den = None if up_denominator is None else np.ascontiguousarray(up_denominator, np.float64)
        ax = _axis(theta_axis) if theta_axis is not None else AxisSpec(0.0, 0.0, 0.0, 0)
        self.spec = WeightSpec(int(weighting), int(n_bitwise_runs), ax, _ptr(self._num), _ptr(self._den))


def count_weighted(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, weights: Weights | None,
                   precision: int = FP32_GUARD, with_regions: bool = True):
    """Raw weighted count (tpcf_count_weighted): (full, regions or None, stats)."""
    full = np.zeros(binning.nb)
    reg = np.zeros((binning.n_jk, binning.nb)) if with_regions else None
    st = Stats()
    rc = _capi.lib().tpcf_count_weighted(ctx._h, a._h, b._h if b is not None else None, binning._h,
                                         C.byref(weights.spec) if weights is not None else None, int(precision),
                                         _ptr(full), _ptr(reg), C.byref(st))
    _check(rc, ctx)
    return full, reg, st.as_dict()


def pair_count_weighted(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, weights: Weights | None,
                        precision: int = FP32_GUARD):
    """The *_invpweights / *_angular counting functions (src/correlators_invpweight.cpp): histograms after
    invert_jk_hists and, for auto counts (b None), multiply_hists(2.0)."""
    full = np.zeros(binning.nb)
    sub = np.zeros((binning.n_jk, binning.nb))
    st = Stats()
    rc = _capi.lib().tpcf_pair_count_weighted(ctx._h, a._h, b._h if b is not None else None, binning._h,
                                              C.byref(weights.spec) if weights is not None else None,
                                              int(precision), _ptr(full), _ptr(sub), C.byref(st))
    _check(rc, ctx)
    return full, sub, st.as_dict()


def iip_weights(bitmask, weight, n_bitwise_runs: int, dither_mask=None):
    """The inverse-p build's reading of bitwise weights (src/io.cpp:519-586):
    returns (weight, input_weight) as float32."""
    m = np.ascontiguousarray(bitmask, np.int64)
    n = m.shape[0]
    m = m.reshape(n, -1)
    d = None if dither_mask is None else np.ascontiguousarray(dither_mask, np.int64).reshape(n, m.shape[1])
    w = np.array(weight, dtype=np.float32, copy=True).reshape(n)
    iw = np.empty(n, np.float32)
    _check(_capi.lib().tpcf_iip_weights(n, m.shape[1], _ptr(m), _ptr(d), int(n_bitwise_runs), _ptr(w), _ptr(iw)))
    return w, iw


def count_many(ctx: Context, jobs, precision: int = FP32_GUARD, reference_form: bool = False):
    """Several counts in one call (tpcf_count_many): jobs is a list of
    (a, b or None, binning) or (a, b, binning, weights).  Results as one
    count() (reference_form: auto_/cross_pair_count) per job, in order; each
    count's host work overlaps the previous count's kernel.  Returns a list of
    (full, regions, stats)."""
    outs = []
    arr = (_capi.CountJob * max(1, len(jobs)))()
    for k, job in enumerate(jobs):
        a, b, binning = job[0], job[1], job[2]
        weights = job[3] if len(job) > 3 else None
        full = np.zeros(binning.nb)
        reg = np.zeros((binning.n_jk, binning.nb))
        st = Stats()
        outs.append((full, reg, st, weights))
        arr[k] = _capi.CountJob(a._h, b._h if b is not None else None, binning._h,
                                C.cast(C.pointer(weights.spec), C.c_void_p) if weights is not None else None,
                                int(precision), int(bool(reference_form)), _ptr(full), _ptr(reg),
                                C.cast(C.pointer(st), C.c_void_p))
    _check(_capi.lib().tpcf_count_many(ctx._h, arr, len(jobs)), ctx)
    return [(f, r, st.as_dict()) for f, r, st, _ in outs]


def count_shard(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, shard: int, n_shards: int,
                precision: int = FP32_GUARD, weights: Weights | None = None):
    """One shard of a count split across processes (tpcf_count_shard): returns
    (partial[(1 + n_jk) * nb, PARTIAL_WORDS] int64, scale_exp, stats).  Partials
    of all shards add word by word; shard_combine turns the sum into the
    count's histograms."""
    partial = np.zeros(((1 + binning.n_jk) * binning.nb, _capi.PARTIAL_WORDS), np.int64)
    se = C.c_int32()
    st = Stats()
    rc = _capi.lib().tpcf_count_shard(ctx._h, a._h, b._h if b is not None else None, binning._h,
                                      C.byref(weights.spec) if weights is not None else None, int(precision),
                                      int(shard), int(n_shards), _ptr(partial), C.byref(se), C.byref(st))
    _check(rc, ctx)
    return partial, se.value, st.as_dict()


def shard_combine(binning: Binning, partial, scale_exp: int):
    """Summed shard partials -> (full[nb], regions[n_jk, nb]) as count() returns them."""
    p = np.ascontiguousarray(partial, np.int64)
    if p.size != (1 + binning.n_jk) * binning.nb * _capi.PARTIAL_WORDS:
        raise ValueError("partial has the wrong size for this binning")
    full = np.empty(binning.nb)
    reg = np.empty((binning.n_jk, binning.nb))
    _check(_capi.lib().tpcf_shard_combine(binning._h, _ptr(p), int(scale_exp), _ptr(full), _ptr(reg)))
    return full, reg


def count_sharded(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, precision: int = FP32_GUARD,
                  weights: Weights | None = None, group=None):
    """One count split over the ranks of a torch.distributed process group,
    one GPU per rank: each rank runs its shard and one all-reduce (SUM over
    int64 limbs) adds the partial sums, so every rank returns exactly what
    count() returns.  Returns (full, regions, stats of this rank's shard)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        partial, se, st = count_shard(ctx, a, b, binning, 0, 1, precision, weights)
        return (*shard_combine(binning, partial, se), st)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    partial, se, st = count_shard(ctx, a, b, binning, rank, world, precision, weights)
    full, reg = shard_combine(binning, reduce_partials(partial, se, group), se)
    return full, reg, st


def reduce_partials(partial, scale_exp: int, group=None):
    """The exchange step of a sharded count: every rank's partial sums
    (int64 limbs, count_shard) added by one all-reduce SUM over the process
    group -- on the GPU for an NCCL group, on the host for gloo -- after
    checking that all ranks planned the same fixed-point scale.  Returns the
    summed limbs (as numpy) for shard_combine."""
    import torch
    import torch.distributed as dist
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(partial, np.int64)).to(dev)
    chk = torch.tensor([scale_exp, -scale_exp], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(chk, op=dist.ReduceOp.MAX, group=group)
    if int(chk[0]) != scale_exp or -int(chk[1]) != scale_exp:
        raise TpcfError(_capi.TPCF_E_INVALID_ARG, "shards disagree on the fixed-point scale: different inputs per rank")
    return t.cpu().numpy()


def upweight_eval(weights: Weights, values) -> np.ndarray:
    """The angular up-weight of a 3-D inverse-p spec at values of 1 - cos(theta), as the kernels form it."""
    v = np.ascontiguousarray(values, np.float64)
    out = np.empty_like(v)
    _check(_capi.lib().tpcf_upweight_eval(C.byref(weights.spec), _ptr(v), v.size, _ptr(out)))
    return out


def wait_selftest(ctx: Context, arrive: bool, limit: int = 1000) -> int:
    """The device give-up path (tpcf_wait_selftest): the pair kernels' bounded
    wait on a barrier that is completed first (arrive) or never; returns the
    status, TPCF_OK or TPCF_E_DEVICE_TIMEOUT (the context stays usable)."""
    return int(_capi.lib().tpcf_wait_selftest(ctx._h, int(bool(arrive)), int(limit)))


def count_backward(ctx: Context, a: Catalog, b: Catalog | None, binning: Binning, dL_dfull,
                   precision: int = FP32_GUARD):
    """Adjoint of count(): per-point dL/dw of a and b (b None: auto count,
    gradient of a only) for dL_dfull = dL/d(raw full histogram)."""
    G = np.ascontiguousarray(dL_dfull, np.float64).reshape(binning.nb)
    ga = np.zeros(a.n)
    gb = np.zeros(b.n) if b is not None else None
    st = Stats()
    rc = _capi.lib().tpcf_count_backward(ctx._h, a._h, b._h if b is not None else None, binning._h, int(precision),
                                         _ptr(G), _ptr(ga), _ptr(gb), C.byref(st))
    _check(rc, ctx)
    return ga, gb, st.as_dict()


class Batch:
    """DD and/or DR counts of many mock catalogues (DR against one shared random
    catalogue) in one persistent launch, planned once and replayed as a CUDA
    graph by run().  refinement: 1..3, 0 automatic, BATCH_AUTOTUNE to probe
    refinements 1, 2, 3 and both orders of the DR jobs and keep the fastest
    (.refinement, .order)."""

    def __init__(self, ctx: Context, mocks, randoms: Catalog | None, binning: Binning, precision: int = FP32_GUARD,
                 what: int = BATCH_DD | BATCH_DR, refinement: int = 0):
        arr = (C.c_void_p * len(mocks))(*[m._h.value for m in mocks])
        h = C.c_void_p()
        rc = _capi.lib().tpcf_batch_create(ctx._h, arr, len(mocks), randoms._h if randoms is not None else None,
                                           binning._h, int(precision), int(what), int(refinement), C.byref(h))
        _check(rc, ctx)
        self._h, self.ctx, self.binning = h, ctx, binning
        self._keep = (list(mocks), randoms)
        self.n_outputs = int(_capi.lib().tpcf_batch_n_outputs(h))
        self.refinement = int(_capi.lib().tpcf_batch_refinement(h))
        self.order = int(_capi.lib().tpcf_batch_order(h))

    def run(self, with_regions: bool = True):
        """(full[n_outputs, nb], regions[n_outputs, n_jk, nb] or None, stats)."""
        nb, nj = self.binning.nb, self.binning.n_jk
        full = np.zeros((self.n_outputs, nb))
        reg = np.zeros((self.n_outputs, nj, nb)) if with_regions else None
        st = Stats()
        _check(_capi.lib().tpcf_batch_run(self._h, _ptr(full), _ptr(reg), C.byref(st)), self.ctx)
        return full, reg, st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            _capi.lib().tpcf_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
