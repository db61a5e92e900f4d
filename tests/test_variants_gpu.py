"""Build variants of the reference on the GPU, through the C ABI, against the
oracle's restatement of each (itself pinned to the reference compiled with
the variant's flags in tests/test_variants_cpu.py):

* TPCF_LOS_MIDPOINT — pi along x1 + x2 (the build without _ANGULAR_PI_DEFN);
* TPCF_WEIGHTS_INVP_DD_DITHER — _USE_DITHER_WEIGHTS;
* bitmasks of 4 words (_N_MASK_INTS = 4).

And the whole inverse-p flow (tpcf_run_invp) against the reference's own
calc_angular_upweight + auto_correlate_*_invpweights on the same catalogues,
output file by output file.

Unit-weight counts bit for bit, weighted sums to 1e-12 relative."""
import os

import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import port, refl
from two_pcf_b200 import ingest, synthetic

pytestmark = pytest.mark.gpu

W_RTOL = 1e-12
N_RUNS = 2048
THETA_MAX = 0.175
TMAX = 1.0 - np.cos(THETA_MAX)


def close(a, b, weighted):
    if weighted:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.nanmax(np.abs(b)))))
    else:
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:8]


def survey_like(seed, n, weights, n_jk=5):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0, 20, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-6)), np.sin(np.radians(6)), n)))
    xyz = synthetic.radec_to_unit(ra, dec) * rng.uniform(400, 700, n)[:, None]
    pick = rng.choice(n, n // 3, replace=False)
    xyz[pick] = xyz[rng.choice(pick, pick.size)] + rng.normal(0, 3.0, (pick.size, 3))
    d = np.sqrt((xyz ** 2).sum(1))
    c = {"xyz": xyz, "unit": xyz / d[:, None], "dcom": d, "jk": rng.integers(0, n_jk, n).astype(np.int32)}
    if weights:
        c["w"] = rng.lognormal(0, 0.3, n).astype(np.float32)
    return c


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("weights", [False, True])
@pytest.mark.parametrize("mode,ax1,ax2", [
    (tp.SIGMA_PI, (0.0, 40.0, 1.0, 20), (0.0, 40.0, 1.0, 20)),
    (tp.S_MU, (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 25)),
])
def test_midpoint_line_of_sight(ctx, mode, ax1, ax2, weights, precision):
    n_jk = 5
    d = survey_like(1, 6000, weights)
    r = survey_like(2, 9000, weights)
    D = tp.Catalog(ctx, d["xyz"], d["unit"], d["dcom"], d.get("w"), None, d["jk"], n_jk)
    R = tp.Catalog(ctx, r["xyz"], r["unit"], r["dcom"], r.get("w"), None, r["jk"], n_jk)
    b = tp.Binning(ctx, mode, ax1, ax2, n_jk)
    b.set_line_of_sight(tp.LOS_MIDPOINT)
    axes = (ax1[0], ax1[1], ax1[2], ax1[3], ax2[0], ax2[1], ax2[2], ax2[3])
    omode = {tp.SIGMA_PI: port.SIGMA_PI, tp.S_MU: port.S_MU}[mode]
    for other, oc in ((None, None), (R, r)):
        full, sub, _ = (tp.auto_pair_count(ctx, D, b, precision) if other is None
                        else tp.cross_pair_count(ctx, D, R, b, precision))
        with port.variant(los_midpoint=True):
            of, os_, _ = port.count_3d(omode, port.Cat(d["xyz"], d["unit"], d["dcom"], d.get("w"), None, d["jk"]),
                                       None if oc is None else port.Cat(oc["xyz"], oc["unit"], oc["dcom"],
                                                                        oc.get("w"), None, oc["jk"]),
                                       is_auto=other is None, n_jk=n_jk, axes=axes)
        assert of.sum() > 0
        close(full, of, weights)
        close(sub, os_, weights)
    # the default line of sight differs on this geometry
    b2 = tp.Binning(ctx, mode, ax1, ax2, n_jk)
    f2, _, _ = tp.auto_pair_count(ctx, D, b2, precision)
    f1, _, _ = tp.auto_pair_count(ctx, D, b, precision)
    assert not np.array_equal(f1, f2)


def sky(seed, n, n_mask, *, dither=False, masks=True, n_jk=3):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0.0, 14.0, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    d = rng.uniform(400.0, 700.0, n)
    runs = 64 * n_mask if n_mask < 32 else N_RUNS
    c = {"xyz": unit * d[:, None], "unit": unit, "dcom": d, "jk": rng.integers(0, n_jk, n).astype(np.int32),
         "w": rng.lognormal(0, 0.2, n).astype(np.float32), "iw": rng.lognormal(0, 0.3, n).astype(np.float32),
         "masks": (synthetic.bitwise_masks(seed + 7, n, n_runs=runs, n_mask_ints=n_mask) if masks else
                   synthetic.bitwise_masks(0, n, n_mask_ints=n_mask, all_set=True))}
    if dither:
        c["dmasks"] = synthetic.bitwise_masks(seed + 9, n, n_runs=runs, n_mask_ints=n_mask, p_lo=0.0, p_hi=0.6)
    return c


def engine_cat(ctx, c, n_jk):
    C = tp.Catalog(ctx, c["xyz"], c["unit"], c["dcom"], c["w"], c["iw"], c["jk"], n_jk, c["masks"])
    if "dmasks" in c:
        C.set_dither_masks(c["dmasks"])
    return C


def ocat(c):
    return port.Cat(c["xyz"], unit=c["unit"], dcom=c["dcom"], w=c["w"], iw=c["iw"], jk=c["jk"], masks=c["masks"],
                    dmasks=c.get("dmasks"))


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("n_mask,dither", [(32, True), (4, False), (4, True)])
def test_inverse_p_variants(ctx, n_mask, dither, precision):
    n_jk, nt = 3, 30
    runs = 64 * n_mask if n_mask < 32 else N_RUNS
    d = sky(3, 3000, n_mask, dither=dither, n_jk=n_jk)
    D = engine_cat(ctx, d, n_jk)
    wdd = tp.WEIGHTS_INVP_DD_DITHER if dither else tp.WEIGHTS_INVP_DD
    ab = tp.Binning(ctx, tp.ANGULAR, (0.0, TMAX, 1.0, nt), None, n_jk)
    with port.variant(dither=dither):
        of, os_ = port.count_angular(1, ocat(d), None, n_jk=n_jk, theta_max=THETA_MAX, n_theta=nt,
                                     theta_log_base=1.0, n_runs=runs)
        full, sub, _ = tp.pair_count_weighted(ctx, D, None, ab, tp.Weights(wdd, runs), precision)
        close(full, of, True)
        close(sub, os_, True)
        num, _, _ = tp.pair_count_weighted(ctx, D, None, ab, None, precision)
        up = port.make_upweight(0.0, TMAX, nt, 1.0, num / full)
        axes = (0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 10)
        of, os_, _ = port.count_3d(port.S_MU, ocat(d), None, is_auto=True, n_jk=n_jk, axes=axes,
                                   weight_kind=port.W_INVP_DD, up=up, n_runs=runs)
    b = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.3, 20), (0.0, 1.0, 0.0, 10), n_jk)
    f3, s3, _ = tp.pair_count_weighted(ctx, D, None, b, tp.Weights(wdd, runs, (0.0, TMAX, 1.0, nt), num, full),
                                       precision)
    assert np.nansum(of) > 0
    close(f3, of, True)
    close(s3, os_, True)


def test_dither_needs_masks(ctx):
    d = sky(5, 500, 4)
    D = engine_cat(ctx, d, 3)
    ab = tp.Binning(ctx, tp.ANGULAR, (0.0, TMAX, 1.0, 10), None, 3)
    with pytest.raises(tp.TpcfError) as e:
        tp.pair_count_weighted(ctx, D, None, ab, tp.Weights(tp.WEIGHTS_INVP_DD_DITHER, 256))
    assert e.value.status == 1


@pytest.mark.skipif(not refl.available("invp"), reason="reference inverse-p build not present")
@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_inverse_p_flow_matches_reference_program(ctx, tmp_path, precision):
    """tpcf_run_invp against calc_angular_upweight + auto_correlate_*_invpweights."""
    n_jk, nt = 4, 30
    d = sky(21, 2500, 32, n_jk=n_jk)
    r = sky(22, 6000, 32, masks=False, n_jk=n_jk)
    # the weights as the inverse-p reader leaves them: IIP-rescaled, input weights kept
    d["w"], d["iw"] = tp.iip_weights(d["masks"], d["w"], N_RUNS)
    r["w"], r["iw"] = tp.iip_weights(r["masks"], r["w"], N_RUNS)
    names = {}
    for who in ("ref", "ours"):
        (tmp_path / who).mkdir()
        names[who] = tuple(str(tmp_path / who / f) for f in ("mono.txt", "sp.txt", "smu.txt"))

    def params(who):
        return refl.invp_params(n_jk=n_jk, theta_max=THETA_MAX, theta_n_bins=nt, theta_log_base=1.6,
                                n_bitwise_runs=N_RUNS, monopole=(0.0, 40.0, 12, 1.3), sigma=(0.0, 30.0, 10, 1.0),
                                pi=(0.0, 30.0, 10, 1.0), s=(0.0, 40.0, 12, 1.3), mu_n_bins=8, plot=(1, 1, 1),
                                calculate=(1, 1, 1, 1), out_files=names[who])

    refl.invp_reset()
    refl.invp_correlate(params("ref"), d, r, n_threads=4)
    D = engine_cat(ctx, d, n_jk)
    R = engine_cat(ctx, r, n_jk)
    ang = ingest.run_invp(ctx, ingest.Params.parse(params("ours")), D, R, precision)
    # the angular stage against the reference's own counts
    for kind, key in enumerate(("dd", "dd_invp", "dr", "dr_invp")):
        rf, rs = refl.invp_angular(params("ref"), kind, d, None if kind < 2 else r, n_jk=n_jk, n_bins=nt)
        close(ang[key][0], rf, True)
        close(ang[key][1], rs, True)
    n_diff = n_lines = 0
    for a, b in zip(names["ours"], names["ref"]):
        for k in [None] + list(range(n_jk)):
            fa = a if k is None else ingest.sub_filename(a, k)
            fb = b if k is None else ingest.sub_filename(b, k)
            la, lb = open(fa).read().splitlines(), open(fb).read().splitlines()
            assert len(la) == len(lb)
            n_lines += len(lb)
            for x, y in zip(la, lb):
                if x != y:
                    n_diff += 1
                    np.testing.assert_allclose([float(t) for t in x.split("\t")], [float(t) for t in y.split("\t")],
                                               rtol=2e-6, equal_nan=True)
    assert n_diff <= max(3, n_lines // 100), (n_diff, n_lines)
    assert os.path.getsize(names["ours"][2]) > 0
