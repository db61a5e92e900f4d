"""tpcf_count_many: several counts in one call, each count's host planning
overlapping the previous kernel, must give exactly what one tpcf_count (or,
with reference_form, tpcf_pair_count_weighted) per job gives — across
binnings, weightings, precisions, angular and 3-D counts, with grids built
inside the call or already cached."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import _capi, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def survey(ctx):
    w = synthetic.survey_catalogue(seed=21, n_data=12_000, n_rand=36_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    return {"D": D, "R": R, "n_jk": w["n_jk"]}


def binnings(ctx, n_jk):
    return [tp.Binning(ctx, tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50), n_jk),
            tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), n_jk),
            tp.Binning(ctx, tp.MONOPOLE, (0.0, 80.0, 1.3, 20), None, n_jk)]


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("cached", [False, True])
def test_count_many_matches_single_counts(ctx, survey, precision, cached):
    D, R = survey["D"], survey["R"]
    bins = binnings(ctx, survey["n_jk"])
    jobs = [(a, b, bn) for bn in bins for a, b in ((D, None), (D, R), (R, None))]
    if not cached:
        for c in (D, R):
            _capi.lib().tpcf_catalog_release_cache(c._h)
    many = tp.count_many(ctx, jobs, precision)
    for (a, b, bn), (f, r, st) in zip(jobs, many):
        f1, r1, st1 = tp.count(ctx, a, b, bn, precision)
        assert np.array_equal(f, f1)
        assert np.array_equal(r, r1)
        assert st["in_range"] == st1["in_range"] and st["candidates"] == st1["candidates"]


def test_count_many_reference_form_and_weightings(ctx):
    rng = np.random.default_rng(4)
    n, n_jk, nt = 3000, 3, 20
    ra = rng.uniform(0, 14, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n)))
    unit = synthetic.radec_to_unit(ra, dec)
    d = rng.uniform(400, 700, n)
    jk = rng.integers(0, n_jk, n).astype(np.int32)
    masks = synthetic.bitwise_masks(3, n, n_runs=256, n_mask_ints=4)
    A = tp.Catalog(ctx, unit * d[:, None], unit, d, rng.lognormal(0, 0.2, n).astype(np.float32),
                   rng.lognormal(0, 0.3, n).astype(np.float32), jk, n_jk, masks)
    tmax = 1.0 - np.cos(0.175)
    ab = tp.Binning(ctx, tp.ANGULAR, (0.0, tmax, 1.0, nt), None, n_jk)
    b3 = tp.Binning(ctx, tp.S_MU, (0.0, 60.0, 1.3, 12), (0.0, 1.0, 0.0, 6), n_jk)
    num, _, _ = tp.pair_count_weighted(ctx, A, None, ab, None)
    den, _, _ = tp.pair_count_weighted(ctx, A, None, ab, tp.Weights(tp.WEIGHTS_INVP_DD, 256))
    spec = tp.Weights(tp.WEIGHTS_INVP_DD, 256, (0.0, tmax, 1.0, nt), num, den)
    jobs = [(A, None, ab), (A, None, ab, tp.Weights(tp.WEIGHTS_INVP_DD, 256)), (A, None, b3, spec), (A, None, b3)]
    many = tp.count_many(ctx, jobs, reference_form=True)
    singles = [tp.pair_count_weighted(ctx, A, None, ab, None),
               tp.pair_count_weighted(ctx, A, None, ab, tp.Weights(tp.WEIGHTS_INVP_DD, 256)),
               tp.pair_count_weighted(ctx, A, None, b3, spec),
               tp.auto_pair_count(ctx, A, b3)]
    for (f, r, _), (f1, r1, _) in zip(many, singles):
        assert np.array_equal(f, f1, equal_nan=True)
        assert np.array_equal(r, r1, equal_nan=True)


def test_count_many_empty_and_errors(ctx, survey):
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 50.0, 1.0, 10), None, survey["n_jk"])
    far = tp.Catalog(ctx, np.zeros((10, 3)) + 100.0, d_comov=np.full(10, -1.0),
                     jk_region=np.zeros(10, np.int32), n_jk_regions=survey["n_jk"])  # every point dropped
    res = tp.count_many(ctx, [(far, None, b), (survey["D"], None, b)])
    assert not res[0][0].any()
    assert np.array_equal(res[1][0], tp.count(ctx, survey["D"], None, b)[0])
    with pytest.raises(tp.TpcfError):
        tp.count_many(ctx, [(survey["D"], None, b)], precision=7)
    assert tp.count_many(ctx, []) == []


def test_count_many_trace_leaves_counts_unchanged(ctx, survey, capfd, monkeypatch):
    """TPCF_TRACE=1 prints one timeline line per count (and per grid built)
    on stderr; the counts are those of an untraced call."""
    D, R = survey["D"], survey["R"]
    b = binnings(ctx, survey["n_jk"])[1]
    jobs = [(D, None, b), (D, R, b), (R, None, b)]
    for c in (D, R):
        _capi.lib().tpcf_catalog_release_cache(c._h)
    plain = tp.count_many(ctx, jobs)
    capfd.readouterr()
    monkeypatch.setenv("TPCF_TRACE", "1")
    for c in (D, R):
        _capi.lib().tpcf_catalog_release_cache(c._h)
    traced = tp.count_many(ctx, jobs)
    err = capfd.readouterr().err
    assert "[tpcf trace] 3 counts: grids built" in err
    assert all(f"count {k}:" in err for k in range(3))
    assert "[tpcf trace] grid of" in err
    for (f, r, _), (f1, r1, _) in zip(plain, traced):
        assert np.array_equal(f, f1)
        assert np.array_equal(r, r1)
