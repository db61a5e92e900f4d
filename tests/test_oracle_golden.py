"""The oracle restatement (oracle/tpcf_oracle.c) against the golden fixtures
produced by the reference build (tests/golden/make_golden.py) and, where the
reference build is present, against the reference directly on fresh inputs.

Unit-weight counts must agree bit for bit; weighted sums to 1e-12 relative
(both sum the same float pair weights in double, in different orders)."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from oracle import port, refl

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("sky_", "full_")))  # 3-D plain-build fixtures
W_RTOL = 1e-12


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def oracle_cat(g, tag):
    get = lambda k: g.get(f"{tag}_{k}")
    return port.Cat(get("xyz"), unit=get("unit"), dcom=get("dcom"), w=get("w"), jk=get("jk"))


def close(a, b, weighted):
    if weighted:
        np.testing.assert_allclose(a, b, rtol=W_RTOL, atol=1e-9 * max(1.0, float(np.abs(b).max())))
    else:
        assert np.array_equal(a, b)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_golden_counts(path):
    g = load(path)
    mode, axes, n_jk = int(g["mode"]), tuple(g["axes"]), int(g["n_jk"])
    axes = (axes[0], axes[1], axes[2], int(axes[3]), axes[4], axes[5], axes[6], int(axes[7]))
    d, r = oracle_cat(g, "d"), oracle_cat(g, "r")
    weighted = "d_w" in g
    for lab, a, b, auto in (("dd", d, None, True), ("dr", d, r, False), ("rr", r, None, True)):
        full, sub, used = port.count_3d(mode, a, b, is_auto=auto, n_jk=n_jk, axes=axes)
        assert full.sum() > 0
        close(full, g[f"{lab}_full"], weighted)
        close(sub, g[f"{lab}_sub"], weighted)
        assert used[0] == g[f"{lab}_used"][0]


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_normalisation_and_xi(path):
    g = load(path)
    n_jk = int(g["n_jk"])
    L = port.lib()
    normed = {}
    for lab, ta, tb in (("dd", "d", None), ("dr", "d", "r"), ("rr", "r", None)):
        full = np.array(g[f"{lab}_full"], np.float64)
        sub = np.array(g[f"{lab}_sub"], np.float64)
        nb = full.size

        def kept(tag):
            n = g[f"{tag}_xyz"].shape[0]
            idx = port.partition(g[f"{tag}_dcom"]) if f"{tag}_dcom" in g else np.arange(n)
            w = g.get(f"{tag}_w", np.ones(n, np.float32))[idx].astype(np.float32)
            jk = g.get(f"{tag}_jk", np.zeros(n, np.int32))[idx].astype(np.int32)
            return np.ascontiguousarray(w), np.ascontiguousarray(jk)

        wa, ja = kept(ta)
        if tb is None:
            L.orc_normalise_auto(wa.ctypes.data, ja.ctypes.data, wa.size, n_jk, nb, full.ctypes.data, sub.ctypes.data)
        else:
            wb, jb = kept(tb)
            L.orc_normalise_cross(wa.ctypes.data, ja.ctypes.data, wa.size, wb.ctypes.data, jb.ctypes.data, wb.size,
                                  n_jk, nb, full.ctypes.data, sub.ctypes.data)
        np.testing.assert_allclose(full, g[f"{lab}_norm_full"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(sub[0], g[f"{lab}_norm_sub0"], rtol=1e-12, atol=0, equal_nan=True)
        normed[lab] = full
    xi = np.array([L.orc_ls(a, b, c) for a, b, c in zip(normed["dd"], normed["dr"], normed["rr"])])
    np.testing.assert_allclose(xi, g["xi_full"], rtol=1e-10, atol=1e-12)


@pytest.mark.skipif(not refl.available("plain"), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("mode,axes", [
    (refl.MONOPOLE, (0.0, 80.0, 1.5, 20, 0, 0, 0, 0)),
    (refl.SIGMA_PI, (1.0, 40.0, 1.0, 13, 0.0, 30.0, 1.0, 7)),
    (refl.S_MU, (0.0, 90.0, 1.2, 25, 0.0, 1.0, 0.0, 9)),
])
@pytest.mark.parametrize("seed", [3, 4])
def test_oracle_matches_reference_fresh_inputs(mode, axes, seed):
    rng = np.random.default_rng(seed)
    n1, n2, n_jk = 1800, 2200, 5
    x1 = rng.uniform(0, 200, (n1, 3)) + 400
    x2 = rng.uniform(0, 200, (n2, 3)) + 400
    x1[1:40] = x1[40:79]  # duplicates
    x1[0] = x1[1:].min(axis=0) + 1.0  # keep point 0 off the per-axis maxima
    x2[0] = x2[1:].min(axis=0) + 1.0
    w1 = rng.lognormal(0, 0.3, n1).astype(np.float32)
    w2 = rng.lognormal(0, 0.3, n2).astype(np.float32)
    j1 = rng.integers(0, n_jk, n1).astype(np.int32)
    j2 = rng.integers(0, n_jk, n2).astype(np.int32)
    c1 = {"xyz": x1, "w": w1, "jk": j1}
    c2 = {"xyz": x2, "w": w2, "jk": j2}
    for auto in (True, False):
        rf, rs, _ = refl.count_3d(mode, c1, c2, is_auto=auto, n_jk=n_jk, axes=axes, n_threads=2)
        of, os_, _ = port.count_3d(mode, port.Cat(x1, w=w1, jk=j1), None if auto else port.Cat(x2, w=w2, jk=j2),
                                   is_auto=auto, n_jk=n_jk, axes=axes)
        close(of, rf, True)
        close(os_, rs, True)


@pytest.mark.skipif(not refl.available("plain"), reason="reference build (oracle/_ref) not present")
def test_axis_restatement_matches_reference_fields():
    for spec in [(0.0, 100.0, 30, 1.3), (0.0, 1.0, 50, 0.0), (0.0, 50.0, 50, 1.0), (2.5, 60.0, 29, 1.0),
                 (0.0, 1.0 - np.cos(0.175), 40, 1.6), (0.1, 10.0, 7, 1.021), (0.0, 10.0, 7, 1.02)]:
        vmin, vmax, n, base = spec
        ref = refl.axis_fields(vmin, vmax, n, base)
        ax = port.axis(vmin, vmax, n, base)
        for k in ("n_bins", "log_binning", "min", "minus_min", "max", "step", "inv_step", "base", "inv_log_of_base",
                  "inv_log_step"):
            assert np.float32(getattr(ax, k)).tobytes() == np.float32(ref[k]).tobytes() or getattr(ax, k) == ref[k], k
        vals = np.linspace(-5, vmax * 1.2, 3001).astype(np.float32)
        rb = refl.axis_bin_num(vmin, vmax, n, base, vals)
        ob = np.array([port.lib().orc_axis_bin_num(C.byref(ax), float(v)) for v in vals], np.float32)
        assert np.array_equal(rb.view(np.uint32), ob.view(np.uint32))


INVP = os.path.join(os.path.dirname(__file__), "golden", "sky_invp.npz")


def invp_cat(g, tag):
    return port.Cat(g[f"{tag}_xyz"], unit=g[f"{tag}_unit"], dcom=g[f"{tag}_dcom"], w=g[f"{tag}_w"],
                    iw=g[f"{tag}_iw"], jk=g[f"{tag}_jk"], masks=g[f"{tag}_masks"])


def test_oracle_matches_invp_golden():
    """Angular stage, up-weight interpolation and 3-D s-mu inverse-p counts of
    the reference's inverse-p build (tests/golden/make_golden.py)."""
    g = load(INVP)
    n_jk, n_runs = int(g["n_jk"]), int(g["n_runs"])
    d, r = invp_cat(g, "d"), invp_cat(g, "r")
    for pre, th in (("ang", g["theta"]), ("anglog", g["theta_log"])):
        for kind in range(4):
            f, s = port.count_angular(kind, d, None if kind < 2 else r, n_jk=n_jk, theta_max=th[0], n_theta=int(th[1]),
                                      theta_log_base=th[2], n_runs=n_runs)
            close(f, g[f"{pre}{kind}_full"], True)  # weighted: non-unit input weights
            close(s, g[f"{pre}{kind}_sub"], True)
    th = g["theta"]
    tmax = 1.0 - np.cos(th[0])
    up_dd = port.make_upweight(0.0, tmax, int(th[1]), th[2], g["ang0_full"] / g["ang1_full"])
    up_dr = port.make_upweight(0.0, tmax, int(th[1]), th[2], g["ang2_full"] / g["ang3_full"])
    L = port.lib()
    for up, key in ((up_dd, "up_dd"), (up_dr, "up_dr")):
        got = np.array([L.orc_interp(up, float(x)) for x in g["up_v"]])
        assert np.array_equal(got, g[key], equal_nan=True)
    ax = tuple(float(x) for x in g["smu_axes"])
    ax = (ax[0], ax[1], ax[2], int(ax[3]), ax[4], ax[5], ax[6], int(ax[7]))
    f, s, _ = port.count_3d(port.S_MU, d, None, is_auto=True, n_jk=n_jk, axes=ax, weight_kind=port.W_INVP_DD,
                            up=up_dd, n_runs=n_runs)
    close(f, g["dd_invp_full"], True)
    close(s, g["dd_invp_sub"], True)
    f, s, _ = port.count_3d(port.S_MU, d, r, is_auto=False, n_jk=n_jk, axes=ax, weight_kind=port.W_INVP_DR, up=up_dr)
    close(f, g["dr_invp_full"], True)
    close(s, g["dr_invp_sub"], True)


def test_engine_upweight_matches_invp_golden():
    """The engine's host-built interpolation tables against the reference's
    JKHists::interp values stored in the fixture (no GPU needed)."""
    import two_pcf_b200 as tp
    g = load(INVP)
    th = g["theta"]
    axis = (0.0, 1.0 - np.cos(th[0]), th[2], int(th[1]))
    for num, den, key in (("ang0_full", "ang1_full", "up_dd"), ("ang2_full", "ang3_full", "up_dr")):
        w = tp.Weights(tp.WEIGHTS_INVP_DD, int(g["n_runs"]), axis, g[num], g[den])
        assert np.array_equal(tp.upweight_eval(w, g["up_v"]), g[key], equal_nan=True)
