"""Golden outputs of the reference's own command-line program
(oracle/_ref/twopcf_ref, built from its sources by oracle/build_ref.sh) on
two small parameter-file cases, for the end-to-end driver test
(tests/test_driver_gpu.py) on machines without the reference build.

    python tests/golden/make_driver_golden.py

writes tests/golden/driver_outputs.json: for each case, the SHA-256 of the
generated input files (the test regenerates them from the same seeds and
checks the digest) and the text of every output file.

The inputs are seeded synthetic catalogues (no external data):
  box_weighted_jk  cartesian, 1200 clustered points + 3000 randoms in a
                   150 Mpc/h box, lognormal weights, 3 jackknife regions,
                   monopole + sigma-pi + s-mu
  sky_unit         equatorial (flat LCDM, omega_m 0.25, h 1), 900 + 2500
                   points on a 30 x 16 deg patch at 0.1 < z < 0.2, unit
                   weights, no jackknife, monopole + s-mu
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "driver_outputs.json")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "twopcf_ref")

CASES = ("box_weighted_jk", "sky_unit")


def _fmt(v):
    return repr(float(v))


def _clustered_box(rng, n, box, n_centres, sigma):
    centres = rng.uniform(0, box, (n_centres, 3))
    pick = rng.integers(0, n_centres, n)
    return np.mod(centres[pick] + rng.normal(0, sigma, (n, 3)), box)


def write_inputs(case: str, d: str, out_dir: str) -> tuple[str, list[str]]:
    """Writes data.txt, rand.txt and params.ini for a case under d, with the
    outputs going to out_dir.  Returns (param path, output base names)."""
    rng = np.random.default_rng(20240 + CASES.index(case))
    if case == "box_weighted_jk":
        box = 150.0
        data = _clustered_box(rng, 1200, box, 60, 4.0)
        rand = rng.uniform(0, box, (3000, 3))
        wd = rng.lognormal(0, 0.25, len(data))
        wr = rng.lognormal(0, 0.1, len(rand))
        jd = (data[:, 0] // (box / 3)).astype(int).clip(0, 2)
        jr = (rand[:, 0] // (box / 3)).astype(int).clip(0, 2)
        rows = [(data, wd, jd), (rand, wr, jr)]
        coord, use_w, n_jk = "cartesian", 1, 3
        modes = {"monopole": 1, "sigma_pi": 1, "s_mu": 1}
    else:
        def sky(n):
            ra = rng.uniform(10, 40, n)
            dec = np.degrees(np.arcsin(rng.uniform(np.sin(np.radians(-8)), np.sin(np.radians(8)), n)))
            z = rng.uniform(0.1, 0.2, n)
            return np.stack([ra, dec, z], 1)
        rows = [(sky(900), None, None), (sky(2500), None, None)]
        coord, use_w, n_jk = "equatorial", 0, 1
        modes = {"monopole": 1, "sigma_pi": 0, "s_mu": 1}
    names = []
    for fname, (xyz, w, jk) in zip(("data.txt", "rand.txt"), rows):
        with open(os.path.join(d, fname), "w") as f:
            f.write("# seeded synthetic catalogue\n")
            for i in range(len(xyz)):
                toks = [_fmt(v) for v in xyz[i]]
                if w is not None:
                    toks.append(_fmt(w[i]))
                if jk is not None:
                    toks.append(str(int(jk[i])))
                f.write(" ".join(toks) + "\n")
    outs = {"monopole": "xi_mono.txt", "sigma_pi": "xi_sigpi.txt", "s_mu": "xi_smu.txt"}
    p = f"""# end-to-end case {case}
data_filename = {os.path.join(d, 'data.txt')}
data_file_type = ascii
random_filename = {os.path.join(d, 'rand.txt')}
random_file_type = ascii
coord_system = {coord}
use_weights = {use_w}
n_threads = 2
n_jk_regions = {n_jk}
omega_m = 0.25
h = 1.0
z_min = 0.0
z_max = 1.0
plot_monopole = {modes['monopole']}
monopole_filename = {os.path.join(out_dir, outs['monopole'])}
monopole_output_type = ascii
monopole_log_base = 1.3
monopole_min = 0.0
monopole_max = 30.0
monopole_n_bins = 15
plot_sigma_pi = {modes['sigma_pi']}
sigma_pi_filename = {os.path.join(out_dir, outs['sigma_pi'])}
sigma_pi_output_type = ascii
sigma_log_base = 1.0
sigma_min = 0.0
sigma_max = 20.0
sigma_n_bins = 8
pi_log_base = 1.0
pi_min = 0.0
pi_max = 20.0
pi_n_bins = 8
plot_s_mu = {modes['s_mu']}
s_mu_filename = {os.path.join(out_dir, outs['s_mu'])}
s_mu_output_type = ascii
s_log_base = 1.3
s_min = 0.0
s_max = 30.0
s_n_bins = 10
mu_n_bins = 5
"""
    path = os.path.join(d, "params.ini")
    with open(path, "w") as f:
        f.write(p)
    return path, [outs[m] for m in outs if modes[m]]


def input_digest(d: str) -> str:
    h = hashlib.sha256()
    for fname in ("data.txt", "rand.txt"):
        with open(os.path.join(d, fname), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def main():
    if not os.path.exists(REF_CLI):
        sys.exit(f"{REF_CLI} missing: run oracle/build_ref.sh")
    result = {}
    for case in CASES:
        with tempfile.TemporaryDirectory() as d:
            out_dir = os.path.join(d, "out")
            os.makedirs(out_dir)
            params, _ = write_inputs(case, d, out_dir)
            subprocess.run([REF_CLI, params], check=True, stdout=subprocess.DEVNULL)
            files = {n: open(os.path.join(out_dir, n)).read() for n in sorted(os.listdir(out_dir))}
            result[case] = {"inputs_sha256": input_digest(d), "files": files}
    with open(OUT, "w") as f:
        json.dump(result, f, indent=0, sort_keys=True)
    print(OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
