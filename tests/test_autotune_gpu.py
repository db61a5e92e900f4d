"""The count autotuner and the choices it makes (tpcf_set_autotune,
tpcf_set_kernel_config, tpcf_set_refinement): every refinement (1-3 cells per
maximum separation) and both kernel configurations give the histograms of
the default count bit for bit -- weighted jackknife survey counts and
unit-weight box counts, FP32+guard and FP64 -- and an autotuned context
probes each count class once, keeps its fastest choice and counts the same
histograms with it."""
import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu

SMU = (tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50))
SIGPI = (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50))


@pytest.fixture(scope="module")
def cats():
    c = tp.Context(0)
    w = synthetic.survey_catalogue(seed=13, n_data=20_000, n_rand=60_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(c, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(c, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    _SRC[id(D)] = (d["xyz"], d["x_norm"], d["d_comov"], d["weight"])
    _SRC[id(R)] = (r["xyz"], r["x_norm"], r["d_comov"], r["weight"])
    bx = synthetic.box_catalogue(seed=3, n_data=30_000, n_rand=60_000, box=300.0, n_centres=600)
    BD, BR = tp.Catalog(c, bx["data"]["xyz"]), tp.Catalog(c, bx["rand"]["xyz"])
    yield {"ctx": c, "D": D, "R": R, "n_jk": w["n_jk"], "BD": BD, "BR": BR}
    for cat in (D, R, BD, BR):
        cat.close()
    c.close()


def cases(s):
    c = s["ctx"]
    out = []
    for mode, a1, a2 in (SMU, SIGPI):
        b = tp.Binning(c, mode, a1, a2, s["n_jk"])
        out += [(s["D"], None, b), (s["D"], s["R"], b), (s["R"], None, b)]
    b1 = tp.Binning(c, *SMU, 1)
    out += [(s["BD"], None, b1), (s["BD"], s["BR"], b1)]
    return out


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64], ids=["fp32_guard", "fp64"])
def test_every_choice_counts_the_same(cats, precision):
    c = cats["ctx"]
    for a, b, bn in cases(cats):
        c.set_refinement(0)
        c.set_kernel_config(-1)
        c.set_cross_order(-1)
        full, reg, st = tp.count(c, a, b, bn, precision)
        assert st["in_range"] > 0
        for m in (1, 2, 3):
            for cfg in (0, 1):
                for order in ((0, 1) if b is not None else (0,)):
                    c.set_refinement(m)
                    c.set_kernel_config(cfg)
                    c.set_cross_order(order)
                    f2, r2, st2 = tp.count(c, a, b, bn, precision)
                    assert np.array_equal(f2, full), (m, cfg, order)
                    assert np.array_equal(r2, reg), (m, cfg, order)
                    assert st2["in_range"] == st["in_range"]
    c.set_refinement(0)
    c.set_kernel_config(-1)
    c.set_cross_order(-1)


def test_autotuned_counts_and_table(cats):
    c = cats["ctx"]
    jobs = cases(cats)
    ref = [tp.count(c, a, b, bn) for a, b, bn in jobs]
    ref64 = tp.count(c, jobs[0][0], jobs[0][1], jobs[0][2], tp.FP64)
    c.set_autotune(True)
    try:
        got = tp.count_many(c, [(a, b, bn) for a, b, bn in jobs])
        table = c.autotune_table()
        assert len(table) >= 3
        for e in table:
            assert e["refinement"] in (1, 2, 3) and e["kernel_config"] in (0, 1) and e["order"] in (0, 1)
            rates = e["pairs_per_s"]
            cross = "auto 0" in e["class"]
            # plain-weight FP32+guard: 3 refinements x 2 configurations, x 2 orders for a cross count
            assert len(rates) == 12 and sum(r > 0 for r in rates) == (12 if cross else 6)
            assert rates[(e["refinement"] - 1) + 3 * e["kernel_config"] + 6 * e["order"]] == max(rates)
        for (f, r, _), (f2, r2, _) in zip(ref, got):
            assert np.array_equal(f, f2) and np.array_equal(r, r2)
        # a second pass meets known classes: no new probes
        got2 = [tp.count(c, a, b, bn) for a, b, bn in jobs]
        assert len(c.autotune_table()) == len(table)
        for (f, r, _), (f2, r2, _) in zip(ref, got2):
            assert np.array_equal(f, f2) and np.array_equal(r, r2)
        # the FP64 path tunes the refinement only
        f64, r64, _ = tp.count(c, jobs[0][0], jobs[0][1], jobs[0][2], tp.FP64)
        assert np.array_equal(f64, ref64[0]) and np.array_equal(r64, ref64[1])
        e64 = [e for e in c.autotune_table() if "fp64 1" in e["class"]]
        assert len(e64) == 1 and e64[0]["kernel_config"] == 0 and e64[0]["pairs_per_s"][3:6] == [0, 0, 0]
    finally:
        c.set_autotune(False)


def test_fixed_choice_turns_tuning_off(cats):
    c = cats["ctx"]
    a, b, bn = cases(cats)[1]
    c.set_autotune(True)
    c.set_refinement(2)
    try:
        n0 = len(c.autotune_table())
        tp.count(c, a, b, bn)
        assert len(c.autotune_table()) == n0
    finally:
        c.set_autotune(False)
        c.set_refinement(0)


def test_autotuned_adjoint(cats):
    """The adjoint tunes its refinement only (its gradients are per catalogue,
    so the order stays): gradients equal the untuned ones to the adjoint's
    fixed-point resolution."""
    c = cats["ctx"]
    D, R = cats["D"], cats["R"]
    b = tp.Binning(c, *SMU, 1)
    D1 = tp.Catalog(c, *[np.asarray(x) for x in _xyz_of(D)])
    R1 = tp.Catalog(c, *[np.asarray(x) for x in _xyz_of(R)])
    G = np.random.default_rng(3).standard_normal(b.nb)
    ga, gb, _ = tp.count_backward(c, D1, R1, b, G)
    c.set_autotune(True)
    try:
        ga2, gb2, _ = tp.count_backward(c, D1, R1, b, G)
        e = [x for x in c.autotune_table() if "weight kind 6" in x["class"]]
        assert len(e) == 1 and e[0]["order"] == 0 and sum(r > 0 for r in e[0]["pairs_per_s"]) == 3
    finally:
        c.set_autotune(False)
    scale = np.abs(ga).max()
    np.testing.assert_allclose(ga2, ga, rtol=1e-11, atol=1e-12 * scale)
    np.testing.assert_allclose(gb2, gb, rtol=1e-11, atol=1e-12 * np.abs(gb).max())
    D1.close()
    R1.close()


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64], ids=["fp32_guard", "fp64"])
def test_invp_dr_counts_the_same_in_either_order(cats, precision):
    """Inverse-p DR weights are symmetric in the two points (the product of
    the two weights, and for 3-D counts times the angular up-weight of
    1 - cos(theta)): both orders give the same histograms."""
    c = cats["ctx"]
    D, R, n_jk = cats["D"], cats["R"], cats["n_jk"]
    nt = 20
    theta_axis = (0.0, 1.0 - np.cos(0.05), 1.6, nt)
    rng = np.random.default_rng(8)
    num = rng.uniform(1.0, 2.0, (1 + n_jk) * nt)
    den = rng.uniform(0.5, 1.0, (1 + n_jk) * nt)
    cases_ = [(tp.Binning(c, tp.ANGULAR, theta_axis, None, n_jk), tp.Weights(tp.WEIGHTS_INVP_DR)),
              (tp.Binning(c, *SMU, n_jk), tp.Weights(tp.WEIGHTS_INVP_DR, 64, theta_axis, num, den))]
    try:
        for b, wts in cases_:
            out = []
            for order in (0, 1):
                c.set_cross_order(order)
                f, r, st = tp.count_weighted(c, D, R, b, wts, precision)
                assert st["in_range"] > 0
                out.append((f, r))
            assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    finally:
        c.set_cross_order(-1)


_SRC = {}


def _xyz_of(cat):
    return _SRC[id(cat)]
