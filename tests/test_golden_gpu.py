"""The CUDA engine, through the C ABI, against the golden fixtures made by
the reference itself (tests/golden/make_golden.py), plus edge cases and
size-independent properties.  Unit-weight counts are bit-exact; weighted
sums agree to 1e-12 relative (the engine sums the reference's float pair
weights exactly in 64-bit fixed point; the reference sums them in double in
thread order); xi within 1e-10 relative."""
import glob
import os

import numpy as np
import pytest

import two_pcf_b200 as tp

pytestmark = pytest.mark.gpu

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("sky_", "full_")))  # 3-D plain-build fixtures
W_RTOL = 1e-12
MODES = {0: tp.MONOPOLE, 1: tp.SIGMA_PI, 2: tp.S_MU}


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def catalog(ctx, g, tag, n_jk):
    return tp.Catalog(ctx, g[f"{tag}_xyz"], g.get(f"{tag}_unit"), g.get(f"{tag}_dcom"), g.get(f"{tag}_w"), None,
                      g.get(f"{tag}_jk"), n_jk)


def binning(ctx, g):
    mode = MODES[int(g["mode"])]
    a = g["axes"]
    ax1 = (a[0], a[1], a[2], int(a[3]))
    ax2 = None if mode == tp.MONOPOLE else (a[4], a[5], a[6], int(a[7]))
    return tp.Binning(ctx, mode, ax1, ax2, int(g["n_jk"]))


def close(a, b, weighted):
    if weighted:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.abs(b).max())))
    else:
        assert np.array_equal(a, b), np.flatnonzero(a != b)[:8]


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_engine_matches_golden(ctx, path, precision):
    g = load(path)
    n_jk = int(g["n_jk"])
    D, R = catalog(ctx, g, "d", n_jk), catalog(ctx, g, "r", n_jk)
    b = binning(ctx, g)
    weighted = "d_w" in g
    assert D.n_used == g["dd_used"][0]
    out = {}
    for lab, fn in (("dd", lambda: tp.auto_pair_count(ctx, D, b, precision)),
                    ("dr", lambda: tp.cross_pair_count(ctx, D, R, b, precision)),
                    ("rr", lambda: tp.auto_pair_count(ctx, R, b, precision))):
        full, sub, st = fn()
        close(full, g[f"{lab}_full"], weighted)
        close(sub, g[f"{lab}_sub"], weighted)
        out[lab] = (full, sub)
    # normalisation (JKHists::normalise) and the LS estimator
    nd, nsd = tp.normalise_auto(D, *out["dd"])
    ndr, nsdr = tp.normalise_cross(D, R, *out["dr"])
    nr, nsr = tp.normalise_auto(R, *out["rr"])
    np.testing.assert_allclose(nd, g["dd_norm_full"], rtol=1e-12)
    np.testing.assert_allclose(ndr, g["dr_norm_full"], rtol=1e-12)
    np.testing.assert_allclose(nr, g["rr_norm_full"], rtol=1e-12)
    np.testing.assert_allclose(nsd[0], g["dd_norm_sub0"], rtol=1e-12, equal_nan=True)
    xi = tp.ls_estimator(nd, ndr, nr)
    np.testing.assert_allclose(xi, g["xi_full"], rtol=1e-10, atol=1e-12)


def test_fp32_guard_equals_fp64_at_scale(ctx):
    """Size-independent property: both paths give identical histograms
    (integer counts and exact fixed-point weighted sums) on a clustered
    catalogue of 120k points with jackknife regions."""
    from two_pcf_b200 import synthetic
    w = synthetic.survey_catalogue(seed=5, n_data=40_000, n_rand=120_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    for mode, ax1, ax2 in ((tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50)),
                           (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50))):
        b = tp.Binning(ctx, mode, ax1, ax2, w["n_jk"])
        for a, bb in ((D, None), (D, R)):
            f32, s32, st32 = tp.count(ctx, a, bb, b, tp.FP32_GUARD)
            f64, s64, st64 = tp.count(ctx, a, bb, b, tp.FP64)
            assert np.array_equal(f32, f64)
            assert np.array_equal(s32, s64)
            assert st32["in_range"] == st64["in_range"]
            assert st32["candidates"] == st64["candidates"]


def test_empty_and_single_point(ctx):
    b = tp.Binning(ctx, tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), 1)
    E = tp.Catalog(ctx, np.zeros((0, 3)))
    one = tp.Catalog(ctx, np.array([[100.0, 200.0, 300.0]]))
    for a, bb in ((E, None), (one, None), (E, one), (one, E), (one, one)):
        full, sub, st = tp.count(ctx, a, bb, b)
        if a is one and bb is one:
            assert full.sum() == 0  # zero separation is never counted
        else:
            assert full.sum() == 0


def test_duplicates_never_counted(ctx):
    x = np.tile(np.array([[10.0, 20.0, 30.0]]), (500, 1))
    D = tp.Catalog(ctx, x)
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 100.0, 1.3, 30))
    full, sub, st = tp.count(ctx, D, None, b)
    assert full.sum() == 0
    assert st["in_range"] == 0
    assert st["guard_evals"] > 0  # every s^2 = 0 pair sits on the range edge


def test_partition_drops_like_reference(ctx):
    """Points with d_comov < 0 are removed by the reference's loop, which stops
    early and drops some good points too (src/boxes.cpp:15-26)."""
    from oracle import port
    rng = np.random.default_rng(3)
    n = 300
    xyz = rng.uniform(100, 200, (n, 3))
    dcom = np.sqrt((xyz ** 2).sum(1))
    dcom[rng.choice(n, 40, replace=False)] = -1.0
    D = tp.Catalog(ctx, xyz, None, dcom)
    kept = port.partition(dcom)
    assert D.n_used == kept.size
    assert kept.size < n - 40  # good points lost as in the reference
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 60.0, 1.0, 12))
    full, _, _ = tp.count(ctx, D, None, b)
    of, _, _ = port.count_3d(port.MONOPOLE, port.Cat(xyz, dcom=dcom), None, is_auto=True, n_jk=1,
                             axes=(0.0, 60.0, 1.0, 12, 0, 0, 0, 0))
    assert np.array_equal(full * 2, of)


def test_invalid_inputs_rejected(ctx):
    x = np.random.default_rng(1).uniform(0, 1, (10, 3))
    bad = x.copy()
    bad[3, 1] = np.nan
    with pytest.raises(tp.TpcfError) as e:
        tp.Catalog(ctx, bad)
    assert e.value.status == 1
    with pytest.raises(tp.TpcfError):
        tp.Catalog(ctx, x, jk_region=np.full(10, 5, np.int32), n_jk_regions=5)
    D = tp.Catalog(ctx, x, jk_region=np.zeros(10, np.int32), n_jk_regions=2)
    b = tp.Binning(ctx, tp.MONOPOLE, (0.0, 1.0, 1.0, 4), None, 3)
    with pytest.raises(tp.TpcfError):
        tp.count(ctx, D, None, b)


INVP = os.path.join(os.path.dirname(__file__), "golden", "sky_invp.npz")


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64])
def test_engine_matches_invp_golden(ctx, precision):
    """Angular stage (DD, DD inverse-p, DR, DR inverse-p, linear and log theta
    bins) and the 3-D s-mu inverse-p DD / DR of the reference's inverse-p
    build (tests/golden/sky_invp.npz)."""
    g = load(INVP)
    n_jk, n_runs = int(g["n_jk"]), int(g["n_runs"])

    def cat(tag):
        return tp.Catalog(ctx, g[f"{tag}_xyz"], g[f"{tag}_unit"], g[f"{tag}_dcom"], g[f"{tag}_w"], g[f"{tag}_iw"],
                          g[f"{tag}_jk"], n_jk, g[f"{tag}_masks"])

    D, R = cat("d"), cat("r")
    kinds = {0: None, 1: tp.Weights(tp.WEIGHTS_INVP_DD, n_runs), 2: None, 3: tp.Weights(tp.WEIGHTS_INVP_DR)}
    for pre, th in (("ang", g["theta"]), ("anglog", g["theta_log"])):
        b = tp.Binning(ctx, tp.ANGULAR, (0.0, 1.0 - np.cos(th[0]), th[2], int(th[1])), None, n_jk)
        for kind, w in kinds.items():
            full, sub, _ = tp.pair_count_weighted(ctx, D, None if kind < 2 else R, b, w, precision)
            close(full, g[f"{pre}{kind}_full"], True)
            close(sub, g[f"{pre}{kind}_sub"], True)
    th = g["theta"]
    axis = (0.0, 1.0 - np.cos(th[0]), th[2], int(th[1]))
    ax = g["smu_axes"]
    b = tp.Binning(ctx, tp.S_MU, (ax[0], ax[1], ax[2], int(ax[3])), (ax[4], ax[5], ax[6], int(ax[7])), n_jk)
    w_dd = tp.Weights(tp.WEIGHTS_INVP_DD, n_runs, axis, g["ang0_full"], g["ang1_full"])
    w_dr = tp.Weights(tp.WEIGHTS_INVP_DR, n_runs, axis, g["ang2_full"], g["ang3_full"])
    full, sub, _ = tp.pair_count_weighted(ctx, D, None, b, w_dd, precision)
    close(full, g["dd_invp_full"], True)
    close(sub, g["dd_invp_sub"], True)
    full, sub, _ = tp.pair_count_weighted(ctx, D, R, b, w_dr, precision)
    close(full, g["dr_invp_full"], True)
    close(sub, g["dr_invp_sub"], True)
