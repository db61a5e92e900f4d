"""tpcf_count_noalloc — the count that allocates no device memory, its
scratch in a static device array — against tpcf_count, through the C ABI.

Each case counts once with tpcf_count (which also caches the cell grids the
allocation-free call needs) and then twice in a row with tpcf_count_noalloc:
the second call must not see the first call's leftovers in the shared array.
The two allocation-free calls run with every device allocation made to fail
(tpcf_debug_fail_allocations(0)), so they succeed only if they allocate
nothing; tpcf_count under the same setting fails with TPCF_E_OOM, which shows
the setting is in force.
Unit-weight counts must be identical; weighted sums agree to 1e-12 relative,
the tolerance of the other parity tests (both calls run the same kernel and
sum in the same fixed point, so they are in fact identical)."""
import ctypes as C

import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import _capi, synthetic

pytestmark = pytest.mark.gpu

W_RTOL = 1e-12
STATIC_SCRATCH_BYTES = 32 << 20


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def count_noalloc(ctx, a, b, binning, precision=tp.FP32_GUARD):
    full = np.full(binning.nb, np.nan)
    reg = np.full((binning.n_jk, binning.nb), np.nan)
    st = tp.Stats()
    L = _capi.lib()
    rc = L.tpcf_count_noalloc(ctx._h, a._h, b._h if b is not None else None, binning._h, int(precision), _ptr(full),
                              _ptr(reg), C.byref(st))
    msg = L.tpcf_last_error(ctx._h).decode() if rc else ""
    return rc, msg, full, reg, st.as_dict()


class allocations_fail:
    """Every device allocation of the engine fails inside the block."""

    def __enter__(self):
        assert _capi.lib().tpcf_debug_fail_allocations(0) == 0

    def __exit__(self, *exc):
        _capi.lib().tpcf_debug_fail_allocations(-1)


def same(x, y, weighted):
    if weighted:
        np.testing.assert_allclose(x, y, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.abs(y).max())))
    else:
        assert np.array_equal(x, y), np.flatnonzero(x != y)[:8]


@pytest.fixture(scope="module")
def survey(ctx):
    w = synthetic.survey_catalogue(seed=11, n_data=20_000, n_rand=60_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    U = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], None, None, r["jk"], w["n_jk"])
    return {"D": D, "R": R, "U": U, "n_jk": w["n_jk"]}


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("mode,ax1,ax2", [
    (tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50)),
    (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50)),
    (tp.MONOPOLE, (0.0, 100.0, 1.3, 30), None),
])
def test_noalloc_matches_count_twice(ctx, survey, mode, ax1, ax2, precision):
    b = tp.Binning(ctx, mode, ax1, ax2, survey["n_jk"])
    D, R, U = survey["D"], survey["R"], survey["U"]
    for a, bb, weighted in ((D, None, True), (D, R, True), (U, None, False)):
        full, reg, st = tp.count(ctx, a, bb, b, precision)
        assert full.sum() > 0
        with allocations_fail():
            runs = [count_noalloc(ctx, a, bb, b, precision) for _ in range(2)]
            with pytest.raises(tp.TpcfError) as refused:
                tp.count(ctx, a, bb, b, precision)
        assert refused.value.status == _capi.TPCF_E_OOM
        for rc, msg, f2, r2, st2 in runs:
            assert rc == 0, msg
            same(f2, full, weighted)
            same(r2, reg, weighted)
            assert st2["in_range"] == st["in_range"]
            assert st2["candidates"] == st["candidates"]


def test_noalloc_refuses_without_cached_grid(ctx):
    x = np.random.default_rng(2).uniform(100, 300, (3000, 3))
    A = tp.Catalog(ctx, x)
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 40.0, 1.0, 8))
    rc, msg, *_ = count_noalloc(ctx, A, None, b)
    assert rc == _capi.TPCF_E_INVALID_ARG
    assert "tpcf_count" in msg
    full, _, _ = tp.count(ctx, A, None, b)
    rc, msg, f2, _, _ = count_noalloc(ctx, A, None, b)
    assert rc == 0, msg
    same(f2, full, False)


def test_noalloc_refuses_oversized_scratch(ctx):
    """4096 bins x 1100 regions of 128-bit sums (16 bytes each) need more
    than the 32 MiB array."""
    n_jk = 1100
    assert 4096 * n_jk * 16 > STATIC_SCRATCH_BYTES
    rng = np.random.default_rng(4)
    x = rng.uniform(100, 300, (2000, 3))
    A = tp.Catalog(ctx, x, jk_region=rng.integers(0, n_jk, 2000).astype(np.int32), n_jk_regions=n_jk)
    b = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.0, 64), (0.0, 1.0, 0.0, 64), n_jk)
    rc, msg, *_ = count_noalloc(ctx, A, None, b)
    assert rc == _capi.TPCF_E_UNSUPPORTED
    assert str(STATIC_SCRATCH_BYTES) in msg and "tpcf_count" in msg
