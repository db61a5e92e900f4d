"""The CUDA engine against the reference at the benchmark's full sizes.

The fixtures (tests/golden/full_*.npz, made by tests/golden/make_fullsize.py
from the reference build) hold only outputs; the catalogues are regenerated
here from their seeds and checked against the digest the fixture recorded.
Each fixture is counted on both engine paths (FP32+guard and FP64) through
the C ABI in the reference's convention (invert_jk_hists, x2 for auto):

* full_box: 100k clustered data, 300k randoms, unit weights, monopole 30 log
  and s-mu 40 x 50 bins -- every count bit for bit;
* full_survey_unit: 1M data, 5M randoms, unit weights, 100 jackknife regions,
  sigma-pi 50 x 50 and s-mu 40 x 50 -- every count and every region's count
  bit for bit;
* full_survey_w: the same with lognormal weights -- sums within W_RTOL of the
  reference's (the engine's sums of the float pair weights are exact; the
  reference adds them to doubles in thread order).

The normalised full histograms agree to 1e-12 and xi to 1e-10 relative in
every case (src/hist.cpp:290-367, :512-589; src/io.cpp:643-651).
"""
import os

import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import synthetic

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = [n for n in ("full_box", "full_survey_unit", "full_survey_w")
         if os.path.exists(os.path.join(HERE, "golden", n + ".npz"))]
MODES = {0: tp.MONOPOLE, 1: tp.SIGMA_PI, 2: tp.S_MU}
W_RTOL = 1e-12
NORM_RTOL = 1e-12
XI_RTOL = 1e-10

_inputs = {}


def load(name):
    z = np.load(os.path.join(HERE, "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


def regenerate(name, g):
    """The fixture's catalogues from its seed (as make_fullsize.py made them)."""
    if name not in _inputs:
        if name == "full_box":
            w = synthetic.box_catalogue(seed=int(g["gen_seed"]), n_data=int(g["gen_n_data"]),
                                        n_rand=int(g["gen_n_rand"]))
            cat = {"data": {"xyz": w["data"]["xyz"]}, "rand": {"xyz": w["rand"]["xyz"]}, "n_jk": 1}
        else:
            cat = synthetic.survey_catalogue(seed=int(g["gen_seed"]), n_data=int(g["gen_n_data"]),
                                             n_rand=int(g["gen_n_rand"]))
            if name == "full_survey_unit":
                for c in (cat["data"], cat["rand"]):
                    c["weight"] = np.ones_like(c["weight"])
        _inputs.clear()   # one catalogue pair held at a time
        _inputs[name] = cat
    return _inputs[name]


def catalog(ctx, c, n_jk):
    return tp.Catalog(ctx, c["xyz"], c.get("x_norm"), c.get("d_comov"), c.get("weight"), None, c.get("jk"), n_jk)


def binning(ctx, g, tag):
    mode = MODES[int(g[f"{tag}_mode"])]
    a = g[f"{tag}_axes"]
    ax2 = None if mode == tp.MONOPOLE else (a[4], a[5], a[6], int(a[7]))
    return tp.Binning(ctx, mode, (a[0], a[1], a[2], int(a[3])), ax2, int(g["n_jk"]))


def check_sums(ours, ref, weighted, what):
    if weighted:
        np.testing.assert_allclose(ours, ref, rtol=W_RTOL, atol=0, err_msg=what)
    else:
        bad = np.flatnonzero(ours != ref)
        assert bad.size == 0, f"{what}: {bad.size} bins differ, first {bad[:8]}"


@pytest.mark.parametrize("precision", [tp.FP32_GUARD, tp.FP64], ids=["fp32_guard", "fp64"])
@pytest.mark.parametrize("name", NAMES)
def test_fullsize_matches_reference(ctx, name, precision):
    g = load(name)
    cat = regenerate(name, g)
    assert synthetic.catalogue_digest(cat["data"]) == str(g["digest_data"]), \
        "the seed regenerated different data than the fixture was made from"
    assert synthetic.catalogue_digest(cat["rand"]) == str(g["digest_rand"]), \
        "the seed regenerated different randoms than the fixture was made from"
    n_jk = int(g["n_jk"])
    weighted = name == "full_survey_w"
    D, R = catalog(ctx, cat["data"], n_jk), catalog(ctx, cat["rand"], n_jk)
    tags = [t for t in ("mono", "sigpi", "smu") if f"{t}_mode" in g]
    try:
        for tag in tags:
            b = binning(ctx, g, tag)
            out = {}
            for lab, fn in (("dd", lambda: tp.auto_pair_count(ctx, D, b, precision)),
                            ("dr", lambda: tp.cross_pair_count(ctx, D, R, b, precision)),
                            ("rr", lambda: tp.auto_pair_count(ctx, R, b, precision))):
                full, sub, st = fn()
                assert st["in_range"] > 0
                check_sums(full, g[f"{tag}_{lab}_full"], weighted, f"{name} {tag} {lab} full")
                check_sums(sub, g[f"{tag}_{lab}_sub"], weighted, f"{name} {tag} {lab} regions")
                out[lab] = (full, sub)
            assert D.n_used == int(g[f"{tag}_dd_used"][0]) and R.n_used == int(g[f"{tag}_rr_used"][0])
            nd, nsd = tp.normalise_auto(D, *out["dd"])
            ndr, nsdr = tp.normalise_cross(D, R, *out["dr"])
            nr, nsr = tp.normalise_auto(R, *out["rr"])
            for lab, f in (("dd", nd), ("dr", ndr), ("rr", nr)):
                np.testing.assert_allclose(f, g[f"{tag}_{lab}_norm_full"], rtol=NORM_RTOL, atol=0)
            xi = tp.ls_estimator(nd, ndr, nr)
            np.testing.assert_allclose(xi, g[f"{tag}_xi_full"], rtol=XI_RTOL, atol=1e-12)
            b.close()
    finally:
        D.close()
        R.close()
