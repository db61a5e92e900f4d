"""Full-size parity fixtures from the reference itself.

Runs the reference's own counting code (built from its sources by
oracle/build_ref.sh into oracle/_ref/) on the benchmark catalogues at their
full sizes and stores only the outputs; the inputs regenerate from their
seeds (two_pcf_b200/synthetic.py forms positions with correctly rounded
operations only) and each fixture records a sha256 digest of them, so a test
can tell that it counts the same catalogue.

    python tests/golden/make_fullsize.py [box] [survey_w] [survey_unit]

* full_box.npz -- the cartesian box: 100k Neyman-Scott data (2000 centres,
  Poisson(50) members, sigma 5 Mpc/h, L = 500 Mpc/h), 300k uniform randoms,
  unit weights, no jackknife; monopole 30 log bins (base 1.3, 0-100) and s-mu
  40 log bins (base 1.3, 0-100) x 50 mu bins.  Every count is an integer.
* full_survey_w.npz -- the survey slab: 1M clustered data and 5M randoms,
  lognormal(0, 0.2) weights, 100 jackknife regions (10 x 10 in ra/dec);
  sigma-pi 50 x 50 linear bins over 0-50 and s-mu 40 log (1.3, 0-100) x 50.
* full_survey_unit.npz -- the same catalogues and bins with unit weights, so
  the 100-region counts can be compared bit for bit.

Per count (DD auto, DR cross, RR auto) the fixture holds the histograms as
the reference leaves them after invert_jk_hists and (auto) x2 -- the full
histogram and every jackknife region's slice -- and the number of points the
grid kept; per mode, the normalised full histograms (JKHists::normalise,
src/hist.cpp:290-367, :512-589) and the Landy-Szalay xi (src/io.cpp:643-651)
of the full sample.  (The normalised slices and their xi follow from the
stored histograms and would triple the file.)  On 8
host threads the box takes under a minute and each survey fixture about
three quarters of an hour.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refl  # noqa: E402
from two_pcf_b200 import synthetic  # noqa: E402

MONO_AXES = (0.0, 100.0, 1.3, 30, 0.0, 0.0, 0.0, 0)
SMU_AXES = (0.0, 100.0, 1.3, 40, 0.0, 1.0, 0.0, 50)
SIGPI_AXES = (0.0, 50.0, 1.0, 50, 0.0, 50.0, 1.0, 50)

BOX = {"seed": 1, "n_data": 100_000, "n_rand": 300_000}
SURVEY = {"seed": 2, "n_data": 1_000_000, "n_rand": 5_000_000}


def box_inputs():
    """The cartesian box catalogues, as the tests regenerate them."""
    w = synthetic.box_catalogue(**BOX)
    return {"data": {"xyz": w["data"]["xyz"]}, "rand": {"xyz": w["rand"]["xyz"]}, "n_jk": 1}


def survey_inputs(unit_weights: bool):
    """The survey-slab catalogues, as the tests regenerate them."""
    w = synthetic.survey_catalogue(**SURVEY)
    if unit_weights:
        for c in (w["data"], w["rand"]):
            c["weight"] = np.ones_like(c["weight"])
    return w


def ls(dd, dr, rr):
    return np.where(rr == 0, 0.0, dd / np.where(rr == 0, 1, rr) - 2.0 * dr / np.where(rr == 0, 1, rr) + 1.0)


def ref_cat(c):
    return {"xyz": c["xyz"], "unit": c.get("x_norm"), "dcom": c.get("d_comov"), "w": c.get("weight"),
            "jk": c.get("jk")}


def run(cat, modes, n_threads):
    d, r = ref_cat(cat["data"]), ref_cat(cat["rand"])
    n_jk = cat["n_jk"]
    out = {"n_jk": n_jk, "digest_data": synthetic.catalogue_digest(cat["data"]),
           "digest_rand": synthetic.catalogue_digest(cat["rand"])}
    nd, nr = d["xyz"].shape[0], r["xyz"].shape[0]
    wd = d["w"] if d["w"] is not None else np.ones(nd, np.float32)
    wr = r["w"] if r["w"] is not None else np.ones(nr, np.float32)
    jd = d["jk"] if d["jk"] is not None else np.zeros(nd, np.int32)
    jr = r["jk"] if r["jk"] is not None else np.zeros(nr, np.int32)
    for tag, mode, axes in modes:
        out[f"{tag}_mode"] = mode
        out[f"{tag}_axes"] = np.array(axes, dtype=np.float64)
        res = {}
        for lab, a, b, auto in (("dd", d, r, True), ("dr", d, r, False), ("rr", r, d, True)):
            t0 = time.time()
            full, sub, used = refl.count_3d(mode, a, b, is_auto=auto, n_jk=n_jk, axes=axes, n_threads=n_threads)
            print(f"{tag} {lab}: {time.time() - t0:.1f} s", flush=True)
            out[f"{tag}_{lab}_full"] = full
            out[f"{tag}_{lab}_sub"] = sub
            out[f"{tag}_{lab}_used"] = used
            res[lab] = (full, sub)
        # normalisation as the drivers do it (src/correlators.cpp:141-150); no
        # point of these catalogues has d_comov < 0, so every point is kept
        ndd, nsdd = refl.normalise(True, wd, jd, None, None, n_jk, *res["dd"])
        ndr, nsdr = refl.normalise(False, wd, jd, wr, jr, n_jk, *res["dr"])
        nrr, nsrr = refl.normalise(True, wr, jr, None, None, n_jk, *res["rr"])
        for lab, v in (("dd", ndd), ("dr", ndr), ("rr", nrr)):
            out[f"{tag}_{lab}_norm_full"] = v
        with np.errstate(divide="ignore", invalid="ignore"):
            out[f"{tag}_xi_full"] = ls(ndd, ndr, nrr)
    return out


def main(which):
    n_threads = os.cpu_count() or 1
    jobs = {
        "box": ("full_box.npz", box_inputs, [("mono", refl.MONOPOLE, MONO_AXES), ("smu", refl.S_MU, SMU_AXES)],
                BOX),
        "survey_w": ("full_survey_w.npz", lambda: survey_inputs(False),
                     [("sigpi", refl.SIGMA_PI, SIGPI_AXES), ("smu", refl.S_MU, SMU_AXES)], SURVEY),
        "survey_unit": ("full_survey_unit.npz", lambda: survey_inputs(True),
                        [("sigpi", refl.SIGMA_PI, SIGPI_AXES), ("smu", refl.S_MU, SMU_AXES)], SURVEY),
    }
    for name in which:
        fname, make, modes, gen = jobs[name]
        t0 = time.time()
        out = run(make(), modes, n_threads)
        out.update({f"gen_{k}": v for k, v in gen.items()})
        out["ref_threads"] = n_threads
        out["ref_seconds"] = time.time() - t0
        np.savez_compressed(os.path.join(HERE, fname), **out)
        print(f"wrote {fname} in {time.time() - t0:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["box", "survey_w", "survey_unit"])
