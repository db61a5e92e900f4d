"""The oracle's restatement of the inverse-p build (angular counts, popcount
weights, the angular up-weight and the 3-D inverse-p counts) against the
reference's own inverse-p build (oracle/_ref/libtwopcf_ref_invp.so, built
from its sources with an in-memory HDF5 stand-in), on fresh seeded inputs.

Unit-weight counts must agree bit for bit; weighted sums to 1e-12 relative
(both sum the same float pair weights in double, in different orders); the
up-weight interpolation exactly."""
import numpy as np
import pytest

from oracle import port, refl
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.skipif(not refl.available("invp"), reason="reference inverse-p build not present")

W_RTOL = 1e-12
THETA = dict(theta_max=0.175, n_theta=40, theta_log_base=1.6)
N_RUNS = 2048


def sky(seed, n, *, ra_max=14.0, dec_lim=5.0, dmin=400.0, dmax=700.0, weights=True, masks=True, n_jk=4,
        negative=0, dup=10):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0.0, ra_max, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-dec_lim)), np.sin(np.radians(dec_lim)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    unit[1:1 + dup] = unit[1 + dup:1 + 2 * dup]  # identical directions: 1 - cos = 0, binned in bin 0
    d = rng.uniform(dmin, dmax, n)
    if negative:
        d[rng.choice(n, negative, replace=False)] = -1.0
    xyz = unit * np.where(d < 0, 0.0, d)[:, None]  # Galaxy::set: x = 0 when d_comov < 0
    cat = {"xyz": xyz, "unit": unit, "dcom": d, "jk": rng.integers(0, n_jk, n).astype(np.int32)}
    if weights:
        cat["w"] = rng.lognormal(0, 0.2, n).astype(np.float32)
        cat["iw"] = rng.lognormal(0, 0.3, n).astype(np.float32)
    if masks:
        cat["masks"] = synthetic.bitwise_masks(seed + 77, n, n_runs=N_RUNS)
    return cat


def ocat(c):
    return port.Cat(c["xyz"], unit=c["unit"], dcom=c.get("dcom"), w=c.get("w"), iw=c.get("iw"), jk=c.get("jk"),
                    masks=c.get("masks"))


def close(a, b, weighted):
    if weighted:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.abs(b).max())))
    else:
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:8]


def params(n_jk, **kw):
    return refl.invp_params(n_jk=n_jk, theta_max=THETA["theta_max"], theta_n_bins=THETA["n_theta"],
                            theta_log_base=THETA["theta_log_base"], n_bitwise_runs=N_RUNS, **kw)


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
@pytest.mark.parametrize("weights", [False, True])
def test_angular_counts_match_reference(kind, weights):
    n_jk = 4
    d = sky(1, 1200, weights=weights, n_jk=n_jk, negative=25 if kind in (1, 3) else 0)
    r = sky(2, 2500, weights=weights, n_jk=n_jk, masks=False, negative=40 if kind == 3 else 0)
    r["masks"] = synthetic.bitwise_masks(0, 2500, all_set=True)
    p = params(n_jk)
    rf, rs = refl.invp_angular(p, kind, d, None if kind in (0, 1) else r, n_jk=n_jk, n_bins=THETA["n_theta"],
                               n_threads=2)
    of, os_ = port.count_angular(kind, ocat(d), None if kind in (0, 1) else ocat(r), n_jk=n_jk, n_runs=N_RUNS,
                                 **THETA)
    assert rf.sum() > 0
    # kind 1 weights are n_runs / popcount: not integers even with unit input weights
    exact = not weights and kind != 1
    close(of, rf, not exact)
    close(os_, rs, not exact)
    if kind in (0, 1):
        assert of[0] > 0  # identical directions land in bin 0


def test_upweight_interp_matches_reference():
    """JKHists::interp of divide_by_hist(DD, DD_invp) (src/hist.cpp:224-231,
    :369-391) at values across and beyond the theta axis."""
    n_jk = 3
    d = sky(5, 1500, n_jk=n_jk)
    p = params(n_jk)
    refl.invp_reset()
    nb = THETA["n_theta"]
    num_f, num_s = refl.invp_angular(p, 0, d, None, n_jk=n_jk, n_bins=nb)
    den_f, den_s = refl.invp_angular(p, 1, d, None, n_jk=n_jk, n_bins=nb)
    refl.invp_store_angular(p, "num.h5", num_f, num_s)
    refl.invp_store_angular(p, "den.h5", den_f, den_s)
    tmax = 1.0 - np.cos(THETA["theta_max"])
    rng = np.random.default_rng(0)
    v = np.concatenate([np.linspace(-1e-3, tmax * 1.1, 20001), rng.uniform(0, tmax, 20000),
                        np.geomspace(1e-14, tmax, 5000), [0.0, tmax, -0.0]])
    ref = refl.invp_interp("num.h5", "den.h5", v)
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = num_f / den_f
    up = port.make_upweight(0.0, tmax, nb, THETA["theta_log_base"], ratio)
    got = np.array([port.lib().orc_interp(up, float(x)) for x in v])
    # empty angular bins make 0/0 ratios: NaN on both sides
    assert np.isfinite(ref).mean() > 0.9
    assert np.array_equal(got, ref, equal_nan=True)


@pytest.mark.parametrize("theta_base", [1.0, 1.6])
@pytest.mark.parametrize("mode", [port.MONOPOLE, port.SIGMA_PI, port.S_MU])
def test_3d_invp_counts_match_reference(mode, theta_base):
    """With log theta bins the narrow first bins stay empty and their 0/0
    up-weights are NaN, which the reference carries into the 3-D sums; the
    oracle must carry them identically."""
    n_jk = 4
    th = dict(THETA, theta_log_base=theta_base, n_theta=20 if theta_base == 1.0 else 40)
    d = sky(11, 1500, n_jk=n_jk, negative=20)
    r = sky(12, 3000, n_jk=n_jk, masks=False)
    r["masks"] = synthetic.bitwise_masks(0, 3000, all_set=True)
    nb_t = th["n_theta"]
    p = refl.invp_params(n_jk=n_jk, theta_max=th["theta_max"], theta_n_bins=nb_t, theta_log_base=theta_base,
                         n_bitwise_runs=N_RUNS, monopole=(0.0, 60.0, 15, 1.3), sigma=(0.0, 40.0, 20, 1.0),
                         pi=(0.0, 40.0, 20, 1.0), s=(0.0, 60.0, 20, 1.3), mu_n_bins=10)
    refl.invp_reset()
    # the angular stage, stored where the 3-D stage reads it
    dd, dds = refl.invp_angular(p, 0, d, None, n_jk=n_jk, n_bins=nb_t)
    ddi, ddis = refl.invp_angular(p, 1, d, None, n_jk=n_jk, n_bins=nb_t)
    dr, drs = refl.invp_angular(p, 2, d, r, n_jk=n_jk, n_bins=nb_t)
    dri, dris = refl.invp_angular(p, 3, d, r, n_jk=n_jk, n_bins=nb_t)
    for f, a, b in (("ang_dd.hdf5", dd, dds), ("ang_dd_invp.hdf5", ddi, ddis), ("ang_dr.hdf5", dr, drs),
                    ("ang_dr_invp.hdf5", dri, dris)):
        refl.invp_store_angular(p, f, a, b)
    axes = {port.MONOPOLE: (0.0, 60.0, 1.3, 15, 0, 0, 0, 0), port.SIGMA_PI: (0.0, 40.0, 1.0, 20, 0.0, 40.0, 1.0, 20),
            port.S_MU: (0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 10)}[mode]
    nb = axes[3] if mode == port.MONOPOLE else axes[3] * axes[7]
    tmax = 1.0 - np.cos(th["theta_max"])
    with np.errstate(divide="ignore", invalid="ignore"):
        up_dd = port.make_upweight(0.0, tmax, nb_t, theta_base, dd / ddi)
        up_dr = port.make_upweight(0.0, tmax, nb_t, theta_base, dr / dri)
    # DD with inverse-p weights
    rf, rs = refl.invp_count_3d(p, mode, 1, d, None, n_jk=n_jk, nb=nb, n_threads=2)
    of, os_, _ = port.count_3d(mode, ocat(d), None, is_auto=True, n_jk=n_jk, axes=axes, weight_kind=port.W_INVP_DD,
                               up=up_dd, n_runs=N_RUNS)
    assert np.nansum(rf) > 0
    if theta_base == 1.0:
        assert np.isfinite(rf).all()
    close(of, rf, True)
    close(os_, rs, True)
    # DR with the angular DR up-weight
    rf, rs = refl.invp_count_3d(p, mode, 0, d, r, n_jk=n_jk, nb=nb, n_threads=2)
    of, os_, _ = port.count_3d(mode, ocat(d), ocat(r), is_auto=False, n_jk=n_jk, axes=axes,
                               weight_kind=port.W_INVP_DR, up=up_dr)
    close(of, rf, True)
    close(os_, rs, True)


@pytest.mark.parametrize("theta_base", [1.6, 1.0, 1.02, 1.3])
def test_engine_upweight_tables_match_reference(theta_base):
    """The engine's host-built interpolation tables (tpcf_upweight_eval, the
    arithmetic the kernels run) give the reference's JKHists::interp exactly."""
    import two_pcf_b200 as tp
    n_jk = 2
    nb = 25
    d = sky(7, 1500, n_jk=n_jk)
    p = refl.invp_params(n_jk=n_jk, theta_max=0.175, theta_n_bins=nb, theta_log_base=theta_base,
                         n_bitwise_runs=N_RUNS)
    refl.invp_reset()
    num_f, num_s = refl.invp_angular(p, 0, d, None, n_jk=n_jk, n_bins=nb)
    den_f, den_s = refl.invp_angular(p, 1, d, None, n_jk=n_jk, n_bins=nb)
    refl.invp_store_angular(p, "n.h5", num_f, num_s)
    refl.invp_store_angular(p, "d.h5", den_f, den_s)
    tmax = 1.0 - np.cos(0.175)
    rng = np.random.default_rng(1)
    v = np.concatenate([np.linspace(-1e-3, tmax * 1.1, 20001), rng.uniform(0, tmax, 20000),
                        np.geomspace(1e-14, tmax, 5000), [0.0, tmax, -0.0, np.float32(tmax), 2.0, -2.0]])
    ref = refl.invp_interp("n.h5", "d.h5", v)
    w = tp.Weights(tp.WEIGHTS_INVP_DD, N_RUNS, (0.0, tmax, theta_base, nb), num_f, den_f)
    got = tp.upweight_eval(w, v)
    assert np.array_equal(got, ref, equal_nan=True)
