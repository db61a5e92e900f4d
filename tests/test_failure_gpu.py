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


def test_zero_limit_is_refused(ctx):
    assert tp.wait_selftest(ctx, arrive=True, limit=0) == _capi.TPCF_E_INVALID_ARG
