"""Device give-up path: the pair kernels' bounded wait, run by a self-test
kernel on a barrier that nothing completes (a wait that must run out), gives
up after its iteration limit and reports TPCF_E_DEVICE_TIMEOUT; the context
keeps counting correctly afterwards.  Nothing here faults, traps or hangs the
GPU: the wait is bounded and no copy is pending on the barrier."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import _capi

pytestmark = pytest.mark.gpu


def test_bounded_wait_completes_when_the_barrier_is_completed(ctx):
    assert tp.wait_selftest(ctx, arrive=True, limit=1000) == _capi.TPCF_OK


def test_bounded_wait_gives_up_and_the_context_stays_usable(ctx):
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 200.0, (3000, 3))
    cat = tp.Catalog(ctx, x)
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 40.0, 1.3, 12), None)
    before = tp.count(ctx, cat, None, b)[0]
    for limit in (1, 1000):
        assert tp.wait_selftest(ctx, arrive=False, limit=limit) == _capi.TPCF_E_DEVICE_TIMEOUT
        assert b"iteration limit" in _capi.lib().tpcf_last_error(ctx._h)
    after = tp.count(ctx, cat, None, b)[0]
    assert np.array_equal(before, after) and before.sum() > 0


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_count_kernel_gives_up_on_its_own_tile_wait(ctx, precision):
    """The count kernels' own give-up path: with tpcf_debug_force_tile_timeout
    every wait for a staged tile of B, once its copy has completed, takes the
    branch of a wait that gave up, so the kernel raises the device-timeout
    flag, the other CTAs stop taking work items and the call returns
    TPCF_E_DEVICE_TIMEOUT with its results discarded.  No copy is ever left in
    flight.  With the switch off the same counts come out bit for bit as
    before, with and without jackknife regions."""
    lib = _capi.lib()
    w, D, R = _survey_pair(ctx, 37, 3000, 9000)
    b_jk = tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), w["n_jk"])
    x = np.random.default_rng(6).uniform(0.0, 200.0, (4000, 3))
    box = tp.Catalog(ctx, x)
    b_mono = tp.Binning(ctx, tp.MONOPOLE, (0.0, 40.0, 1.3, 12), None)
    cases = [(D, R, b_jk), (box, None, b_mono)]
    before = [tp.count(ctx, a, bb, b, precision) for a, bb, b in cases]
    try:
        assert lib.tpcf_debug_force_tile_timeout(1) == _capi.TPCF_OK
        for a, bb, b in cases:
            with pytest.raises(tp.TpcfError) as exc:
                tp.count(ctx, a, bb, b, precision)
            assert exc.value.status == _capi.TPCF_E_DEVICE_TIMEOUT
            assert "iteration limit" in str(exc.value)
    finally:
        lib.tpcf_debug_force_tile_timeout(0)
    for (a, bb, b), (f0, r0, s0) in zip(cases, before):
        f1, r1, s1 = tp.count(ctx, a, bb, b, precision)
        assert np.array_equal(f0, f1) and np.array_equal(r0, r1) and f0.sum() > 0
        assert s1["in_range"] == s0["in_range"]


def test_zero_limit_is_refused(ctx):
    assert tp.wait_selftest(ctx, arrive=True, limit=0) == _capi.TPCF_E_INVALID_ARG


def _survey_pair(ctx, seed, n_data, n_rand):
    from two_pcf_b200 import synthetic
    w = synthetic.survey_catalogue(seed=seed, n_data=n_data, n_rand=n_rand)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    return w, D, R


def test_allocation_failures_return_status_and_leave_the_context_usable(ctx):
    """Every device allocation of a catalogue, a cell grid or a count's
    scratch made to fail in turn (tpcf_debug_fail_allocations): the call
    fails with TPCF_E_OOM, and once the injection is off the same counts come
    out exactly as before."""
    lib = _capi.lib()
    w, D, R = _survey_pair(ctx, 31, 3000, 9000)
    b = tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), w["n_jk"])
    jobs = [(D, None, b), (D, R, b), (R, None, b)]
    for c in (D, R):
        lib.tpcf_catalog_release_cache(c._h)
    ref = tp.count_many(ctx, jobs)
    try:
        failed = 0
        for after in range(0, 40):
            for c in (D, R):
                lib.tpcf_catalog_release_cache(c._h)
            lib.tpcf_debug_fail_allocations(after)
            try:
                tp.count_many(ctx, jobs)
            except tp.TpcfError as ex:
                assert ex.status == _capi.TPCF_E_OOM, ex
                failed += 1
            finally:
                lib.tpcf_debug_fail_allocations(-1)
        assert failed > 5
        lib.tpcf_debug_fail_allocations(0)
        with pytest.raises(tp.TpcfError) as exc:
            tp.Catalog(ctx, np.zeros((10, 3)) + 5.0)
        assert exc.value.status == _capi.TPCF_E_OOM
    finally:
        lib.tpcf_debug_fail_allocations(-1)
    for c in (D, R):
        lib.tpcf_catalog_release_cache(c._h)
    again = tp.count_many(ctx, jobs)
    for (f, r, _), (f1, r1, _) in zip(ref, again):
        assert np.array_equal(f, f1)
        assert np.array_equal(r, r1)
