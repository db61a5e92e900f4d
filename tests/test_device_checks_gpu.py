"""The checked build (device bounds checks, TPCF_DEVICE_CHECKS) on the GPU.

A child process loads two_pcf_b200/lib/checked/ (TPCF_CHECKED=1) and counts:
survey-slab counts with weights and jackknife regions (sigma-pi, s-mu; DD,
DR, RR), a unit-weight box monopole without regions, an angular count, on
both paths.  No check may fire, and every histogram must equal the release
build's bit for bit.  Then one bad index is planted on the host
(tpcf_debug_corrupt_work_list: the next count's first segment gets a region
past the histogram rows): that count must return TPCF_E_DEVICE_CHECK naming
the segment's region, its kernel skips the item before staging any tile, so
nothing is read or written out of bounds, and the next count on the same
context must again equal the release build's."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMU = ((0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50))
SIGPI = ((0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50))


def counts(out_path=None):
    """Every case's histograms with the library this process loaded; in the
    child also the planted-index check.  Returns {name: array}."""
    import two_pcf_b200 as tp
    from two_pcf_b200 import _capi, synthetic
    ctx = tp.Context(0)
    w = synthetic.survey_catalogue(seed=17, n_data=15_000, n_rand=45_000)
    d, r = w["data"], w["rand"]
    D = tp.Catalog(ctx, d["xyz"], d["x_norm"], d["d_comov"], d["weight"], None, d["jk"], w["n_jk"])
    R = tp.Catalog(ctx, r["xyz"], r["x_norm"], r["d_comov"], r["weight"], None, r["jk"], w["n_jk"])
    bx = synthetic.box_catalogue(seed=5, n_data=20_000, n_rand=40_000, box=250.0, n_centres=400)
    BD, BR = tp.Catalog(ctx, bx["data"]["xyz"]), tp.Catalog(ctx, bx["rand"]["xyz"])
    res = {}
    for prec, pn in ((tp.FP32_GUARD, "f32"), (tp.FP64, "f64")):
        for mode, axes, mn in ((tp.S_MU, SMU, "smu"), (tp.SIGMA_PI, SIGPI, "sigpi")):
            b = tp.Binning(ctx, mode, *axes, w["n_jk"])
            for lab, a, bb in (("dd", D, None), ("dr", D, R), ("rr", R, None)):
                f, g, _ = tp.count(ctx, a, bb, b, prec)
                res[f"{pn}_{mn}_{lab}_full"], res[f"{pn}_{mn}_{lab}_reg"] = f, g
        bm = tp.Binning(ctx, tp.MONOPOLE, (0.0, 60.0, 1.3, 20))
        res[f"{pn}_box_dd"] = tp.count(ctx, BD, None, bm, prec)[0]
        res[f"{pn}_box_dr"] = tp.count(ctx, BD, BR, bm, prec)[0]
        ba = tp.Binning(ctx, tp.ANGULAR, (0.0, 1.0 - np.cos(0.05), 1.6, 20), None, w["n_jk"])
        f, g, _ = tp.count(ctx, D, None, ba, prec)
        res[f"{pn}_ang_full"], res[f"{pn}_ang_reg"] = f, g
    if out_path is not None:
        L = _capi.lib()
        report = {"checks": int(L.tpcf_device_checks())}
        b = tp.Binning(ctx, tp.S_MU, *SMU, w["n_jk"])
        assert L.tpcf_debug_corrupt_work_list(1) == 0
        try:
            tp.count(ctx, D, R, b)
            report["planted"] = {"status": 0, "msg": ""}
        except tp.TpcfError as e:
            report["planted"] = {"status": e.status, "msg": str(e)}
        f, g, _ = tp.count(ctx, D, R, b)
        res["after_full"], res["after_reg"] = f, g
        np.savez(out_path, **res)
        with open(str(out_path) + ".json", "w") as fh:
            json.dump(report, fh)
    for cat in (D, R, BD, BR):
        cat.close()
    ctx.close()
    return res


def test_checked_build_counts_like_release_and_catches_a_planted_index(tmp_path):
    from two_pcf_b200 import _capi
    if not os.path.exists(_capi.CHECKED_LIB_PATH):
        pytest.skip("checked build absent (TPCF_DEVICE_CHECKS=1 python two_pcf_b200/build.py)")
    out = tmp_path / "checked.npz"
    code = (f"import sys; sys.path.insert(0, {ROOT!r}); sys.path.insert(0, {os.path.join(ROOT, 'tests')!r}); "
            f"import test_device_checks_gpu as t; t.counts({str(out)!r})")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900, cwd=ROOT,
                       env=dict(os.environ, TPCF_CHECKED="1"))
    assert r.returncode == 0, r.stderr[-3000:]
    report = json.load(open(str(out) + ".json"))
    assert report["checks"] == 1
    assert report["planted"]["status"] == _capi.TPCF_E_DEVICE_CHECK
    assert "segment's region" in report["planted"]["msg"]
    got = np.load(out)
    ref = counts()
    for k, v in ref.items():
        assert np.array_equal(got[k], v), k
    assert np.array_equal(got["after_full"], ref["f32_smu_dr_full"])
    assert np.array_equal(got["after_reg"], ref["f32_smu_dr_reg"])
