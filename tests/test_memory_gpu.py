"""Device memory of the engine: per-call scratch comes from the context's
stream-ordered pool and is reused, catalogue and grid memory is released in
stream order; neither leaks across repeated counts, and a catalogue may
outlive its context."""
import ctypes as C

import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import _capi, synthetic

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_repeated_counts_do_not_grow_device_memory():
    w = synthetic.survey_catalogue(seed=3, n_data=20_000, n_rand=60_000)
    ctx = tp.Context(0)
    d, r = w["data"], w["rand"]
    b = tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), w["n_jk"])
    L = _capi.lib()

    def cycle():
        D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
        R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
        out = []
        for a, bb in ((D, None), (D, R), (R, None)):
            out.append(tp.count(ctx, a, bb, b)[0])
        L.tpcf_catalog_release_cache(R._h)
        out.append(tp.count(ctx, R, None, b)[0])
        D.close()
        R.close()
        return out

    first = cycle()
    free0 = _free_bytes()
    for _ in range(8):
        again = cycle()
        for x, y in zip(first, again):
            np.testing.assert_allclose(x, y, rtol=1e-13)
    assert free0 - _free_bytes() < (64 << 20)
    ctx.close()


def test_catalogue_outlives_its_context():
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 200, (5000, 3))
    L = _capi.lib()
    h = C.c_void_p()
    assert L.tpcf_create(0, C.byref(h)) == 0
    cat = C.c_void_p()
    assert L.tpcf_catalog_create(h, 5000, x.ctypes.data_as(C.c_void_p), None, None, None, None, None, 1, None, 0,
                                 C.byref(cat)) == 0
    b = C.c_void_p()
    ax = tp.AxisSpec(0.0, 20.0, 1.0, 10)
    assert L.tpcf_binning_create(h, tp.MONOPOLE, C.byref(ax), None, 1, C.byref(b)) == 0
    full = np.zeros(10)
    st = tp.Stats()
    assert L.tpcf_count(h, cat, None, b, tp.FP32_GUARD, full.ctypes.data_as(C.c_void_p), None, C.byref(st)) == 0
    assert full.sum() > 0
    assert L.tpcf_destroy(h) == 0          # context first: its pool stays while the catalogue holds memory from it
    assert L.tpcf_catalog_destroy(cat) == 0   # frees into that pool, which then goes
    assert L.tpcf_binning_destroy(b) == 0
    _free_bytes()                          # a device-wide synchronisation completes the frees
    # the device is still healthy
    ctx = tp.Context(0)
    c2 = tp.Catalog(ctx, x)
    b2 = tp.Binning(ctx, tp.MONOPOLE, (0.0, 20.0, 1.0, 10))
    f2, _, _ = tp.count(ctx, c2, None, b2)
    assert np.array_equal(f2, full)
