"""Generate the golden fixtures from the reference itself.

Runs the reference's own counting code (built from its sources by
oracle/build_ref.sh into oracle/_ref/) on small seeded catalogues and stores
inputs and outputs in tests/golden/*.npz.  The fixtures pin the oracle
restatement (oracle/tpcf_oracle.c) and the CUDA engine in the CPU and GPU
suites, on machines where the reference sources are absent.

    python tests/golden/make_golden.py

Each fixture holds, per count (DD auto, DR cross, RR auto), the histograms as
the reference leaves them after invert_jk_hists and (auto) x2, plus the
normalised histograms (JKHists::normalise) and the Landy-Szalay xi.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import refl  # noqa: E402

MONO, SIGPI, SMU = refl.MONOPOLE, refl.SIGMA_PI, refl.S_MU


def clustered(rng, n, box, offset, sigma=4.0, per=30):
    nc = max(1, n // per)
    c = rng.uniform(0, box, (nc, 3))
    p = np.repeat(c, per, axis=0)[:n] + rng.normal(0, sigma, (n, 3))
    p = np.mod(p, box) + offset
    return p


def unit_of(xyz):
    d = np.sqrt((xyz ** 2).sum(1))
    return xyz / d[:, None], d


def fix_first_point(xyz):
    # The reference's bounding-box scan never tests point 0 against the
    # maximum (src/boxes.cpp:37-40); keep point 0 off the maximum so its
    # cell indexing stays in bounds.
    for _ in range(3):
        if not np.any(xyz[0] >= xyz.max(axis=0)):
            break
        k = 1 + int(np.argmin(xyz[1:, 0]))
        xyz[[0, k]] = xyz[[k, 0]]
    return xyz


def case_box(seed):
    rng = np.random.default_rng(seed)
    d = fix_first_point(clustered(rng, 1500, 250.0, 100.0))
    r = fix_first_point(rng.uniform(0, 250.0, (3000, 3)) + 100.0)
    # edge cases: exact duplicates (s^2 = 0, never counted), points on the
    # faces of a side-100 lattice, a radial pair (mu = 1), a tiny separation
    d[10:20] = d[20:30]
    d[40:50, 0] = 200.0
    d[60] = d[61] * (1.0 + 1e-3)
    d[70] = d[71] + np.array([1e-4, 0, 0])
    return {"data": {"xyz": d}, "rand": {"xyz": r}, "n_jk": 1}


def case_survey(seed, n_jk=9, weights=True, with_negative=False):
    rng = np.random.default_rng(seed)
    n_d, n_r = 1200, 2500
    ra_d = rng.uniform(0, 20, n_d)
    dec_d = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n_d)))
    dist_d = rng.uniform(300, 420, n_d)
    ra_r = rng.uniform(0, 20, n_r)
    dec_r = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n_r)))
    dist_r = rng.uniform(300, 420, n_r)

    def build(ra, dec, dist, n):
        u = np.stack([np.cos(np.radians(dec)) * np.cos(np.radians(ra)),
                      np.cos(np.radians(dec)) * np.sin(np.radians(ra)), np.sin(np.radians(dec))], 1)
        xyz = u * dist[:, None]
        w = rng.lognormal(0, 0.2, n).astype(np.float32) if weights else None
        side = int(round(np.sqrt(n_jk)))
        jk = (np.minimum((ra / (20.0 / side)).astype(int), side - 1) * side
              + np.minimum(((dec + 5) / (10.0 / side)).astype(int), side - 1)).astype(np.int32)
        return {"xyz": fix_first_point(xyz), "unit": u, "dcom": dist.copy(), "w": w, "jk": jk}

    d = build(ra_d, dec_d, dist_d, n_d)
    r = build(ra_r, dec_r, dist_r, n_r)
    # clustered data: pull 40% of the points towards a few centres along the line of sight
    k = n_d * 2 // 5
    d["dcom"][:k] = 350 + rng.normal(0, 3, k)
    d["xyz"][:k] = d["unit"][:k] * d["dcom"][:k, None]
    if with_negative:
        # points without a redshift: d_comov < 0 (src/io.cpp:458-463); the
        # reference's partition loop stops early and drops some good points too
        neg = rng.choice(n_d, 25, replace=False)
        d["dcom"][neg] = -1.0
        d["xyz"][neg] = 0.0
    return {"data": d, "rand": r, "n_jk": n_jk}


AXES = {
    "mono_log": (MONO, (0.0, 100.0, 1.3, 30, 0.0, 0.0, 0.0, 0)),
    "smu_log": (SMU, (0.0, 100.0, 1.3, 40, 0.0, 1.0, 0.0, 50)),
    "sigpi_lin": (SIGPI, (0.0, 50.0, 1.0, 50, 0.0, 50.0, 1.0, 50)),
    "smu_lin_min": (SMU, (2.0, 60.0, 1.0, 29, 0.0, 1.0, 0.0, 10)),
}

CASES = {
    "box_mono": (case_box, 11, "mono_log"),
    "box_smu": (case_box, 11, "smu_log"),
    "box_sigpi": (case_box, 12, "sigpi_lin"),
    "survey_sigpi_jk_w": (lambda s: case_survey(s), 21, "sigpi_lin"),
    "survey_smu_jk_w": (lambda s: case_survey(s), 21, "smu_log"),
    "survey_smu_min_neg": (lambda s: case_survey(s, n_jk=4, weights=True, with_negative=True), 22, "smu_lin_min"),
    "survey_mono_unit_jk": (lambda s: case_survey(s, n_jk=4, weights=False), 23, "mono_log"),
}


def ls(dd, dr, rr):
    return np.where(rr == 0, 0.0, dd / np.where(rr == 0, 1, rr) - 2.0 * dr / np.where(rr == 0, 1, rr) + 1.0)


def make(name):
    fn, seed, axname = CASES[name]
    cat = fn(seed)
    mode, axes = AXES[axname]
    n_jk = cat["n_jk"]
    d, r = cat["data"], cat["rand"]
    out = {"mode": mode, "axes": np.array(axes, dtype=np.float64), "n_jk": n_jk}
    for tag, c in (("d", d), ("r", r)):
        for k in ("xyz", "unit", "dcom", "w", "jk"):
            if c.get(k) is not None:
                out[f"{tag}_{k}"] = c[k]
    res = {}
    for lab, a, b, auto in (("dd", d, r, True), ("dr", d, r, False), ("rr", r, d, True)):
        full, sub, used = refl.count_3d(mode, a, b, is_auto=auto, n_jk=n_jk, axes=axes, n_threads=1)
        out[f"{lab}_full"] = full
        out[f"{lab}_sub"] = sub
        out[f"{lab}_used"] = used
        res[lab] = (full, sub, used)
    # normalisation as the drivers do it (src/correlators.cpp:141-150) and xi
    from oracle import port
    for lab, a, b, auto in (("dd", d, None, True), ("dr", d, r, False), ("rr", r, None, True)):
        full, sub, used = res[lab]
        pa = port.partition(a["dcom"]) if a.get("dcom") is not None else np.arange(a["xyz"].shape[0])
        wa = (a["w"] if a.get("w") is not None else np.ones(a["xyz"].shape[0], np.float32))[pa]
        ja = (a["jk"] if a.get("jk") is not None else np.zeros(a["xyz"].shape[0], np.int32))[pa]
        if auto:
            nf, ns = refl.normalise(True, wa, ja, None, None, n_jk, full, sub)
        else:
            pb = port.partition(b["dcom"]) if b.get("dcom") is not None else np.arange(b["xyz"].shape[0])
            wb = (b["w"] if b.get("w") is not None else np.ones(b["xyz"].shape[0], np.float32))[pb]
            jb = (b["jk"] if b.get("jk") is not None else np.zeros(b["xyz"].shape[0], np.int32))[pb]
            nf, ns = refl.normalise(False, wa, ja, wb, jb, n_jk, full, sub)
        out[f"{lab}_norm_full"] = nf
        out[f"{lab}_norm_sub0"] = ns[0]  # one jackknife row of the normalised histogram
    out["xi_full"] = np.array([refl.plain().ref_ls_estimator(x, y, z) for x, y, z in
                               zip(out["dd_norm_full"], out["dr_norm_full"], out["rr_norm_full"])])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    return out


if __name__ == "__main__":
    if not refl.available("plain"):
        sys.exit("oracle/_ref not built: run oracle/build_ref.sh")
    for nm in CASES:
        o = make(nm)
        print(nm, {k: float(o[k].sum()) for k in ("dd_full", "dr_full", "rr_full")})
