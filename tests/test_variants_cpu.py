"""Build variants of the reference — pi along x1 + x2 (no _ANGULAR_PI_DEFN),
_USE_DITHER_WEIGHTS, _N_MASK_INTS = 4 — and the inverse-p build's reading of
bitwise weights: the oracle's restatement (and the engine's host-side
tpcf_iip_weights) against the reference compiled with each variant's flags
(oracle/build_ref.sh).  Unit-weight counts bit for bit; weighted sums to
1e-12 relative; the IIP weights exactly."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import port, refl
from two_pcf_b200 import synthetic

W_RTOL = 1e-12
N_RUNS = 2048


def close(a, b, weighted):
    if weighted:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.nanmax(np.abs(b)))))
    else:
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:8]


def survey_like(seed, n, weights):
    """A slab of sky at 400-700 Mpc/h with clustered points: lines of sight
    that differ between the angular and the midpoint definitions."""
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0, 20, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-6)), np.sin(np.radians(6)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    d = rng.uniform(400, 700, n)
    xyz = unit * d[:, None]
    pick = rng.choice(n, n // 3, replace=False)
    xyz[pick] = xyz[rng.choice(pick, pick.size)] + rng.normal(0, 3.0, (pick.size, 3))
    d = np.sqrt((xyz ** 2).sum(1))
    unit = xyz / d[:, None]
    c = {"xyz": xyz, "unit": unit, "dcom": d, "jk": rng.integers(0, 5, n).astype(np.int32)}
    if weights:
        c["w"] = rng.lognormal(0, 0.3, n).astype(np.float32)
    return c


@pytest.mark.skipif(not refl.available("midpoint"), reason="reference midpoint build not present")
@pytest.mark.parametrize("mode,axes", [
    (port.SIGMA_PI, (0.0, 40.0, 1.0, 20, 0.0, 40.0, 1.0, 20)),
    (port.S_MU, (0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 25)),
])
@pytest.mark.parametrize("weights", [False, True])
def test_oracle_midpoint_pi_matches_reference(mode, axes, weights):
    d = survey_like(1, 3000, weights)
    r = survey_like(2, 5000, weights)
    for cat2, is_auto in ((None, True), (r, False)):
        rf, rs, _ = refl.count_3d(mode, d, cat2, is_auto=is_auto, n_jk=5, axes=axes, n_threads=2, variant="midpoint")
        with port.variant(los_midpoint=True):
            of, os_, _ = port.count_3d(mode, port.Cat(d["xyz"], d["unit"], d["dcom"], d.get("w"), None, d["jk"]),
                                       None if cat2 is None else port.Cat(r["xyz"], r["unit"], r["dcom"], r.get("w"),
                                                                          None, r["jk"]),
                                       is_auto=is_auto, n_jk=5, axes=axes, n_threads=2)
        assert rf.sum() > 0
        close(of, rf, weights)
        close(os_, rs, weights)
        # the two definitions bin differently on this geometry
        af, _, _ = refl.count_3d(mode, d, cat2, is_auto=is_auto, n_jk=5, axes=axes, n_threads=2)
        assert not np.array_equal(af, rf)


def sky(seed, n, n_mask, *, dither=False, masks=True):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0.0, 14.0, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    d = rng.uniform(400.0, 700.0, n)
    c = {"xyz": unit * d[:, None], "unit": unit, "dcom": d, "jk": rng.integers(0, 3, n).astype(np.int32),
         "w": rng.lognormal(0, 0.2, n).astype(np.float32), "iw": rng.lognormal(0, 0.3, n).astype(np.float32)}
    runs = 64 * n_mask if n_mask < 32 else N_RUNS
    c["masks"] = synthetic.bitwise_masks(seed + 7, n, n_runs=runs, n_mask_ints=n_mask) if masks else \
        synthetic.bitwise_masks(0, n, n_mask_ints=n_mask, all_set=True)
    if dither:
        c["dmasks"] = synthetic.bitwise_masks(seed + 9, n, n_runs=runs, n_mask_ints=n_mask, p_lo=0.0, p_hi=0.6)
    return c


def ocat(c):
    return port.Cat(c["xyz"], unit=c["unit"], dcom=c["dcom"], w=c.get("w"), iw=c.get("iw"), jk=c["jk"],
                    masks=c.get("masks"), dmasks=c.get("dmasks"))


VARIANTS = [("invp_dither", 32, True), ("invp4", 4, False)]


@pytest.mark.parametrize("variant,n_mask,dither", VARIANTS)
def test_oracle_invp_variants_match_reference(variant, n_mask, dither):
    if not refl.available(variant):
        pytest.skip(f"reference {variant} build not present")
    assert refl.n_mask_ints(variant) == n_mask
    n_runs = 64 * n_mask if n_mask < 32 else N_RUNS
    n_jk, nt, tmax_ang = 3, 30, 0.175
    d = sky(3, 1500, n_mask, dither=dither)
    r = sky(4, 2500, n_mask, dither=dither, masks=False)
    p = refl.invp_params(n_jk=n_jk, theta_max=tmax_ang, theta_n_bins=nt, theta_log_base=1.0, n_bitwise_runs=n_runs,
                         s=(0.0, 60.0, 20, 1.3), mu_n_bins=10)
    refl.invp_reset(variant)
    th = dict(theta_max=tmax_ang, n_theta=nt, theta_log_base=1.0)
    ang = {}
    with port.variant(dither=dither):
        for kind in range(4):
            rf, rs = refl.invp_angular(p, kind, d, None if kind < 2 else r, n_jk=n_jk, n_bins=nt, variant=variant)
            of, os_ = port.count_angular(kind, ocat(d), None if kind < 2 else ocat(r), n_jk=n_jk, n_runs=n_runs,
                                         **th)
            close(of, rf, True)
            close(os_, rs, True)
            ang[kind] = (rf, rs)
        for f, k in (("ang_dd.hdf5", 0), ("ang_dd_invp.hdf5", 1), ("ang_dr.hdf5", 2), ("ang_dr_invp.hdf5", 3)):
            refl.invp_store_angular(p, f, *ang[k], variant=variant)
        tmax = 1.0 - np.cos(tmax_ang)
        up = port.make_upweight(0.0, tmax, nt, 1.0, ang[0][0] / ang[1][0])
        axes = (0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 10)
        rf, rs = refl.invp_count_3d(p, port.S_MU, 1, d, None, n_jk=n_jk, nb=200, n_threads=2, variant=variant)
        of, os_, _ = port.count_3d(port.S_MU, ocat(d), None, is_auto=True, n_jk=n_jk, axes=axes,
                                   weight_kind=port.W_INVP_DD, up=up, n_runs=n_runs)
    assert rf.sum() > 0
    close(of, rf, True)
    close(os_, rs, True)


@pytest.mark.parametrize("variant,n_mask,dither", [("invp", 32, False)] + VARIANTS)
def test_iip_weights_match_reference_reader(variant, n_mask, dither):
    """tpcf_iip_weights against read_data_hdf5's bitwise-weight handling
    (src/io.cpp:519-586), run through the reference's own reader."""
    if not refl.available(variant):
        pytest.skip(f"reference {variant} build not present")
    rng = np.random.default_rng(11)
    n = 4000
    runs = 64 * n_mask if n_mask < 32 else N_RUNS
    masks = synthetic.bitwise_masks(5, n, n_runs=runs, n_mask_ints=n_mask, p_lo=0.0, p_hi=1.0)
    masks[:50] = 0                      # no bit set: total 0 -> 1
    masks[50:100] = synthetic.bitwise_masks(0, 50, n_mask_ints=n_mask, all_set=True)  # total == n_runs?
    dmasks = synthetic.bitwise_masks(6, n, n_runs=runs, n_mask_ints=n_mask, p_lo=0.0, p_hi=1.0) if dither else None
    w = rng.lognormal(0, 0.4, n)
    xyz = rng.uniform(100, 300, (n, 3))
    p = refl.invp_params(n_jk=1, n_bitwise_runs=runs)
    ref = refl.invp_read(p, xyz[:, 0], xyz[:, 1], xyz[:, 2], w, None, masks, dmasks=dmasks, variant=variant)
    got_w, got_iw = tp.iip_weights(masks, w.astype(np.float32), runs, dither_mask=dmasks)
    assert np.array_equal(got_iw, ref["input_weight"])
    assert np.array_equal(got_w, ref["weight"])
    assert np.array_equal(ref["masks"], masks)
