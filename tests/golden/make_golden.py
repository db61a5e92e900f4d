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


# ---------------------------------------------------------- inverse-p build

INVP_THETA = (0.175, 20, 1.0)   # theta_max, n_bins, log base (linear: every bin filled)
INVP_THETA_LOG = (0.175, 40, 1.6)
INVP_SMU = (0.0, 60.0, 1.3, 20, 0.0, 1.0, 0.0, 10)
N_RUNS = 2048


def case_sky(seed, n, n_jk, *, masks_all_set=False):
    rng = np.random.default_rng(seed)
    ra = rng.uniform(0.0, 14.0, n)
    dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-5)), np.sin(np.radians(5)), n)))
    u = np.stack([np.cos(np.radians(dec)) * np.cos(np.radians(ra)),
                  np.cos(np.radians(dec)) * np.sin(np.radians(ra)), np.sin(np.radians(dec))], 1)
    u[1:11] = u[11:21]  # identical directions
    d = rng.uniform(400.0, 700.0, n)
    xyz = u * d[:, None]
    from two_pcf_b200 import synthetic
    masks = synthetic.bitwise_masks(seed + 5, n, n_runs=N_RUNS, all_set=masks_all_set)
    return {"xyz": xyz, "unit": u, "dcom": d, "w": rng.lognormal(0, 0.2, n).astype(np.float32),
            "iw": rng.lognormal(0, 0.3, n).astype(np.float32), "jk": rng.integers(0, n_jk, n).astype(np.int32),
            "masks": masks}


def make_invp():
    """tests/golden/sky_invp.npz: the angular stage (DD, DD inverse-p, DR, DR
    inverse-p; linear and log theta bins), the 3-D s-mu inverse-p DD and DR
    that read it back, and the up-weight JKHists::interp at sample values.
    Every point has a redshift: for points without one (x = 0) the plain
    angular counts' pixel lookup (vec2pix of a zero vector) is undefined in
    the reference."""
    n_jk = 4
    d = case_sky(41, 1000, n_jk)
    r = case_sky(42, 2000, n_jk, masks_all_set=True)
    out = {"n_jk": n_jk, "n_runs": N_RUNS, "theta": np.array(INVP_THETA), "theta_log": np.array(INVP_THETA_LOG),
           "smu_axes": np.array(INVP_SMU)}
    for tag, c in (("d", d), ("r", r)):
        for k, v in c.items():
            out[f"{tag}_{k}"] = v
    refl.invp_reset()
    tmax, nb, base = INVP_THETA
    p = refl.invp_params(n_jk=n_jk, theta_max=tmax, theta_n_bins=nb, theta_log_base=base, n_bitwise_runs=N_RUNS,
                         s=(INVP_SMU[0], INVP_SMU[1], INVP_SMU[3], INVP_SMU[2]), mu_n_bins=INVP_SMU[7])
    files = ("ang_dd.hdf5", "ang_dd_invp.hdf5", "ang_dr.hdf5", "ang_dr_invp.hdf5")
    for kind in range(4):
        f, sb = refl.invp_angular(p, kind, d, None if kind < 2 else r, n_jk=n_jk, n_bins=nb)
        out[f"ang{kind}_full"], out[f"ang{kind}_sub"] = f, sb
        refl.invp_store_angular(p, files[kind], f, sb)
    pl = refl.invp_params(n_jk=n_jk, theta_max=INVP_THETA_LOG[0], theta_n_bins=INVP_THETA_LOG[1],
                          theta_log_base=INVP_THETA_LOG[2], n_bitwise_runs=N_RUNS, dd_file="l0", ddi_file="l1",
                          dr_file="l2", dri_file="l3")
    for kind in range(4):
        f, sb = refl.invp_angular(pl, kind, d, None if kind < 2 else r, n_jk=n_jk, n_bins=INVP_THETA_LOG[1])
        out[f"anglog{kind}_full"], out[f"anglog{kind}_sub"] = f, sb
    nb3 = INVP_SMU[3] * INVP_SMU[7]
    out["dd_invp_full"], out["dd_invp_sub"] = refl.invp_count_3d(p, SMU, 1, d, None, n_jk=n_jk, nb=nb3)
    out["dr_invp_full"], out["dr_invp_sub"] = refl.invp_count_3d(p, SMU, 0, d, r, n_jk=n_jk, nb=nb3)
    t = 1.0 - np.cos(tmax)
    v = np.concatenate([np.linspace(-1e-4, t * 1.05, 4001), np.geomspace(1e-12, t, 1000)])
    out["up_v"] = v
    out["up_dd"] = refl.invp_interp(files[0], files[1], v)
    out["up_dr"] = refl.invp_interp(files[2], files[3], v)
    np.savez_compressed(os.path.join(HERE, "sky_invp.npz"), **out)
    return out


if __name__ == "__main__":
    if not refl.available("plain"):
        sys.exit("oracle/_ref not built: run oracle/build_ref.sh")
    for nm in CASES:
        o = make(nm)
        print(nm, {k: float(o[k].sum()) for k in ("dd_full", "dr_full", "rr_full")})
    if refl.available("invp"):
        o = make_invp()
        print("sky_invp", {k: float(np.nansum(o[k])) for k in ("ang0_full", "ang1_full", "dd_invp_full",
                                                                "dr_invp_full")})
