"""Angular counts and inverse-p (bitwise popcount) weights on the GPU, through
the C ABI, against the oracle (itself pinned to the reference's inverse-p
build in tests/test_oracle_invp.py and by tests/golden/sky_invp.npz).

Unit-weight angular counts must match bit for bit; inverse-p and weighted
sums to 1e-12 relative; bins the reference fills with NaN (0/0 up-weights of
empty angular bins) must be NaN here too."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import port
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu

W_RTOL = 1e-12
N_RUNS = 2048
THETA_MAX = 0.175
TMAX = 1.0 - np.cos(THETA_MAX)


def sky(seed, n, *, weights=True, masks=True, all_set=False, n_jk=4, negative=0, dup=10, ra_max=14.0,
        dec_lim=5.0):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0.0, ra_max, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-dec_lim)), np.sin(np.radians(dec_lim)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    unit[1:1 + dup] = unit[1 + dup:1 + 2 * dup]
    d = rng.uniform(400.0, 700.0, n)
    if negative:
        d[rng.choice(n, negative, replace=False)] = -1.0
    xyz = unit * np.where(d < 0, 0.0, d)[:, None]
    c = {"xyz": xyz, "unit": unit, "dcom": d, "jk": rng.integers(0, n_jk, n).astype(np.int32)}
    if weights:
        c["w"] = rng.lognormal(0, 0.2, n).astype(np.float32)
        c["iw"] = rng.lognormal(0, 0.3, n).astype(np.float32)
    if masks:
        c["masks"] = synthetic.bitwise_masks(seed + 77, n, n_runs=N_RUNS, all_set=all_set)
    return c


def engine_cat(ctx, c, n_jk):
    return tp.Catalog(ctx, c["xyz"], c["unit"], c["dcom"], c.get("w"), c.get("iw"), c["jk"], n_jk, c.get("masks"))


def oracle_cat(c):
    return port.Cat(c["xyz"], unit=c["unit"], dcom=c["dcom"], w=c.get("w"), iw=c.get("iw"), jk=c["jk"],
                    masks=c.get("masks"))


def close(a, b, exact):
    if exact:
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:8]
    else:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.nanmax(np.abs(b)))))


ANG_WEIGHTS = {0: None, 1: tp.Weights(tp.WEIGHTS_INVP_DD, N_RUNS), 2: None, 3: tp.Weights(tp.WEIGHTS_INVP_DR)}


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("weights", [False, True])
@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_angular_matches_oracle(ctx, kind, weights, precision):
    n_jk = 4
    d = sky(1, 2500, weights=weights, n_jk=n_jk, negative=25 if kind in (1, 3) else 0)
    r = sky(2, 4000, weights=weights, n_jk=n_jk, all_set=True, negative=30 if kind == 3 else 0)
    auto = kind in (0, 1)
    for base, nb in ((1.6, 40), (1.0, 30)):
        b = tp.Binning(ctx, tp.ANGULAR, (0.0, TMAX, base, nb), None, n_jk)
        D = engine_cat(ctx, d, n_jk)
        R = engine_cat(ctx, r, n_jk)
        full, sub, st = tp.pair_count_weighted(ctx, D, None if auto else R, b, ANG_WEIGHTS[kind], precision)
        of, os_ = port.count_angular(kind, oracle_cat(d), None if auto else oracle_cat(r), n_jk=n_jk,
                                     theta_max=THETA_MAX, n_theta=nb, theta_log_base=base, n_runs=N_RUNS)
        assert of.sum() > 0
        exact = not weights and kind != 1
        close(full, of, exact)
        close(sub, os_, exact)
        if auto:
            assert full[0] > 0  # identical directions: 1 - cos(theta) = 0 lands in bin 0


def test_angular_plain_count_entry_point(ctx):
    """tpcf_count on an angular binning is the plain angular DD."""
    d = sky(3, 2000, weights=False, masks=False, n_jk=1)
    D = engine_cat(ctx, d, 1)
    b = tp.Binning(ctx, tp.ANGULAR, (0.0, TMAX, 1.6, 40))
    full, _, st = tp.count(ctx, D, None, b)
    of, _ = port.count_angular(0, oracle_cat(d), None, n_jk=1, theta_max=THETA_MAX, n_theta=40, theta_log_base=1.6)
    assert np.array_equal(full * 2, of)
    assert st["in_range"] == of.sum() / 2


def angular_stage(d, r, n_jk, nb, base):
    """The angular DD / DD-invp / DR / DR-invp full histograms (oracle)."""
    out = {}
    for kind in range(4):
        auto = kind in (0, 1)
        f, _ = port.count_angular(kind, oracle_cat(d), None if auto else oracle_cat(r), n_jk=n_jk,
                                  theta_max=THETA_MAX, n_theta=nb, theta_log_base=base, n_runs=N_RUNS)
        out[kind] = f
    return out


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("theta_base", [1.0, 1.6])
@pytest.mark.parametrize("mode,axes", [
    (tp.S_MU, ((0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10))),
    (tp.SIGMA_PI, ((0.0, 40.0, 1.0, 20), (0.0, 40.0, 1.0, 20))),
    (tp.MONOPOLE, ((0.0, 60.0, 1.3, 15), None)),
])
def test_3d_invp_matches_oracle(ctx, mode, axes, theta_base, precision):
    n_jk = 4
    nb_t = 20 if theta_base == 1.0 else 40
    d = sky(11, 2500, n_jk=n_jk, negative=20)
    r = sky(12, 4000, n_jk=n_jk, all_set=True)
    ang = angular_stage(d, r, n_jk, nb_t, theta_base)
    with np.errstate(divide="ignore", invalid="ignore"):
        up_dd = port.make_upweight(0.0, TMAX, nb_t, theta_base, ang[0] / ang[1])
        up_dr = port.make_upweight(0.0, TMAX, nb_t, theta_base, ang[2] / ang[3])
    ax1, ax2 = axes
    oaxes = tuple(ax1) + (tuple(ax2) if ax2 is not None else (0, 0, 0, 0))
    b = tp.Binning(ctx, mode, ax1, ax2, n_jk)
    D = engine_cat(ctx, d, n_jk)
    R = engine_cat(ctx, r, n_jk)
    theta_axis = (0.0, TMAX, theta_base, nb_t)
    w_dd = tp.Weights(tp.WEIGHTS_INVP_DD, N_RUNS, theta_axis, ang[0], ang[1])
    w_dr = tp.Weights(tp.WEIGHTS_INVP_DR, N_RUNS, theta_axis, ang[2], ang[3])
    full, sub, _ = tp.pair_count_weighted(ctx, D, None, b, w_dd, precision)
    of, os_, _ = port.count_3d(mode, oracle_cat(d), None, is_auto=True, n_jk=n_jk, axes=oaxes,
                               weight_kind=port.W_INVP_DD, up=up_dd, n_runs=N_RUNS)
    assert np.nansum(of) > 0
    if theta_base == 1.0:
        assert np.isfinite(of).all()
    close(full, of, False)
    close(sub, os_, False)
    full, sub, _ = tp.pair_count_weighted(ctx, D, R, b, w_dr, precision)
    of, os_, _ = port.count_3d(mode, oracle_cat(d), oracle_cat(r), is_auto=False, n_jk=n_jk, axes=oaxes,
                               weight_kind=port.W_INVP_DR, up=up_dr)
    close(full, of, False)
    close(sub, os_, False)


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_nonfinite_upweights_propagate(ctx, precision):
    """Up-weight histograms with empty bins (0/0 = NaN, x/0 = inf), as a sparse
    angular stage writes them: the bins and regions those pairs reach become
    NaN or infinite exactly where the reference's double sums do."""
    n_jk = 3
    nb_t = 20
    d = sky(21, 2000, n_jk=n_jk)
    r = sky(22, 3000, n_jk=n_jk, all_set=True)
    ang = angular_stage(d, r, n_jk, nb_t, 1.0)
    num, den = ang[0].copy(), ang[1].copy()
    num[4], den[4] = 0.0, 0.0      # NaN
    den[9] = 0.0                   # +inf
    num[13], den[13] = -num[13], 0.0  # -inf
    with np.errstate(divide="ignore", invalid="ignore"):
        up = port.make_upweight(0.0, TMAX, nb_t, 1.0, num / den)
    b = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10), n_jk)
    D = engine_cat(ctx, d, n_jk)
    w = tp.Weights(tp.WEIGHTS_INVP_DD, N_RUNS, (0.0, TMAX, 1.0, nb_t), num, den)
    full, sub, _ = tp.pair_count_weighted(ctx, D, None, b, w, precision)
    of, os_, _ = port.count_3d(tp.S_MU, oracle_cat(d), None, is_auto=True, n_jk=n_jk,
                               axes=(0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 10), weight_kind=port.W_INVP_DD, up=up,
                               n_runs=N_RUNS)
    assert np.isnan(of).any() and np.isfinite(of).any()
    assert np.array_equal(np.isnan(full), np.isnan(of))
    assert np.array_equal(np.isinf(full), np.isinf(of))
    assert np.array_equal(np.isnan(sub), np.isnan(os_))
    assert np.array_equal(np.isinf(sub), np.isinf(os_))
    fin = np.isfinite(of)
    close(full[fin], of[fin], False)
    inf = np.isinf(of)
    assert np.array_equal(np.sign(full[inf]), np.sign(of[inf]))


def test_invp_rejects_missing_masks(ctx):
    d = sky(4, 500, masks=False)
    D = engine_cat(ctx, d, 4)
    b = tp.Binning(ctx, tp.ANGULAR, (0.0, TMAX, 1.6, 40), None, 4)
    with pytest.raises(tp.TpcfError) as e:
        tp.pair_count_weighted(ctx, D, None, b, tp.Weights(tp.WEIGHTS_INVP_DD, N_RUNS))
    assert e.value.status == 1
    b3 = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10), 4)
    with pytest.raises(tp.TpcfError):
        tp.pair_count_weighted(ctx, D, None, b3, tp.Weights(tp.WEIGHTS_INVP_DR))  # no up-weight histograms
