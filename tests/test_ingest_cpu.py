"""The command-line flow around the counts (parameter file, cosmology table,
Galaxy::set, the ASCII reader and the ASCII writers) against the reference's
own code, built from its sources into oracle/_ref (refl).  All host-side:
every comparison is exact (bit for bit, or byte for byte for files)."""
import os
import zlib

import numpy as np
import pytest

import two_pcf_b200 as tp
from oracle import refl
from two_pcf_b200 import ingest

pytestmark = pytest.mark.skipif(not refl.available("plain"), reason="reference build not present")

# The numeric fields ref_params_parse returns, in its order.
DBL_KEYS = ["omega_m", "h", "z_min", "z_max", "monopole_log_base", "monopole_min", "monopole_max", "sigma_log_base",
            "sigma_min", "sigma_max", "pi_log_base", "pi_min", "pi_max", "s_log_base", "s_min", "s_max",
            "theta_max", "theta_log_base"]
INT_KEYS = ["use_weights", "n_threads", "n_jk_regions", "plot_monopole", "monopole_n_bins", "plot_sigma_pi",
            "sigma_n_bins", "pi_n_bins", "plot_s_mu", "s_n_bins", "mu_n_bins", "calculate_angular_dd",
            "calculate_angular_dd_invpweights", "calculate_angular_dr", "calculate_angular_dr_invpweights",
            "theta_n_bins", "healpix_order", "n_bitwise_runs"]
STR_KEYS = ["data_filename", "data_file_type", "random_filename", "random_file_type", "coord_system",
            "monopole_filename", "monopole_output_type", "sigma_pi_filename", "s_mu_filename"]


def param_text(rng, values):
    """A parameter file setting every key, with the formatting the
    reference's parser tolerates: spaces anywhere, trailing comments, comment
    and junk lines, unknown keys, repeated keys (the last one wins)."""
    lines = ["# two_pcf parameter file", "", "this line has no equals sign", "unknown_key = 3"]
    for k, v in values.items():
        txt = f"{v!r}" if isinstance(v, float) else str(v)
        style = rng.integers(0, 5)
        if style == 0:
            lines.append(f"{k}={txt}")
        elif style == 1:
            lines.append(f"  {k}  =  {txt}   # comment = with equals")
        elif style == 2:
            lines.append(f"{k[:2]} {k[2:]} = {txt[:1]} {txt[1:]}")  # spaces inside key and value vanish
        elif style == 3:
            lines.append(f"{k} = 12345")
            lines.append(f"{k} ={txt}")  # repeated: last wins
        elif isinstance(v, str):
            lines.append(f"{k}={txt}#x")
        else:
            lines.append(f"{k} =\t{txt}#x")  # std::stod / std::stoi skip the leading tab
    lines.append("#n_threads = 77")
    return "\n".join(lines) + "\n"


def random_values(rng):
    v = {}
    for k in DBL_KEYS:
        v[k] = float(rng.choice([rng.uniform(-5, 200), 0.25, 1.0, 1e-3, 1.3]))
    for k in INT_KEYS:
        v[k] = int(rng.integers(-3, 60))
    for k in STR_KEYS:
        v[k] = "file_" + str(int(rng.integers(0, 1000))) + ".txt"
    return v


@pytest.mark.parametrize("seed", range(6))
def test_params_match_reference(seed):
    rng = np.random.default_rng(seed)
    values = random_values(rng)
    text = param_text(rng, values)
    d_ref, i_ref = refl.params_parse(text)
    p = ingest.Params.parse(text)
    got_d = np.array([p.get_double(k) for k in DBL_KEYS])
    got_i = np.array([p.get_int(k) for k in INT_KEYS], dtype=np.int32)
    assert np.array_equal(got_d, d_ref)
    assert np.array_equal(got_i, i_ref), (got_i, i_ref)
    for k in STR_KEYS:
        assert p.get_string(k) == values[k]


def test_params_quirks():
    p = ingest.Params.parse("n_jk_regions = -4\ndata_filename = a b.txt # c\ns_max = 1e2xyz\nmu_n_bins = 7.9\n")
    assert p.get_int("n_jk_regions") == 1  # <= 1 becomes 1
    assert p.get_string("data_filename") == "ab.txt"  # spaces removed
    assert p.get_double("s_max") == 100.0  # std::stod ignores trailing characters
    assert p.get_int("mu_n_bins") == 7  # std::stoi stops at the '.'
    for bad in ("s_max = abc\n", "mu_n_bins = \n", "n_threads = 99999999999\n"):
        with pytest.raises(ingest.HostError):
            ingest.Params.parse(bad)


@pytest.mark.parametrize("om,h,zmin,zmax", [(0.25, 1.0, 0.0, 1.0), (0.31, 0.7, 0.0, 0.5), (0.3, 0.68, 0.05, 0.8),
                                            (0.25, 1.0, 0.2, 0.6)])
def test_comov_dist_matches_reference(om, h, zmin, zmax):
    rng = np.random.default_rng(1)
    z = np.concatenate([rng.uniform(zmin - 0.1, zmax + 0.1, 20000), np.linspace(zmin, zmax, 1001),
                        [zmin, zmax, zmin - 1.0, zmax + 5.0, np.nextafter(zmin, 1), np.inf, -np.inf]])
    ref = refl.comov_dist(om, h, zmin, zmax, z)
    c = ingest.Cosmology(om, h, zmin, zmax)
    got = c.comov_dist(z)
    assert np.array_equal(got, ref)


def test_galaxy_set_matches_reference():
    rng = np.random.default_rng(2)
    n = 50000
    ra = rng.uniform(-30, 400, n)
    dec = rng.uniform(-90, 90, n)
    d = rng.uniform(-50, 3000, n)
    x_ref, xn_ref = refl.galaxy_set(ra, dec, d)
    x, xn = ingest.galaxy_set(ra, dec, d)
    assert np.array_equal(x, x_ref)
    assert np.array_equal(xn, xn_ref)
    assert (x[d < 0] == 0).all()


def _write_catalogue(path, cols, sep, rng, comments=True):
    lines = []
    if comments:
        lines += ["# header comment", ""]
    for row in zip(*cols):
        toks = []
        for v in row:
            if isinstance(v, (np.floating, float)):
                toks.append(repr(float(v)) if rng.random() < 0.5 else f"{float(v):.6f}")
            else:
                toks.append(str(v))
        if sep == " ":
            line = "".join(t + " " * int(rng.integers(1, 4)) for t in toks).rstrip()
            if rng.random() < 0.3:
                line = "  " + line
        elif sep == ",":
            line = ", ".join(toks)
        else:
            line = "\t".join(toks)
        lines.append(line)
        if comments and rng.random() < 0.01:
            lines.append("#interleaved comment")
    with open(path, "w") as f:
        f.write("\n".join(lines))  # no newline after the last line


@pytest.mark.parametrize("sep", [" ", "\t", ","])
@pytest.mark.parametrize("coords,weights,n_jk", [("cartesian", True, 5), ("cartesian", False, 1),
                                                 ("equatorial", True, 8), ("equatorial", False, 1)])
def test_read_ascii_matches_reference(tmp_path, sep, coords, weights, n_jk):
    rng = np.random.default_rng(zlib.crc32(f"{sep}|{coords}|{weights}|{n_jk}".encode()))
    n = 3000
    if coords == "cartesian":
        cols = [rng.uniform(-500, 500, n), rng.uniform(-500, 500, n), rng.uniform(-500, 500, n)]
    else:
        cols = [rng.uniform(0, 360, n), rng.uniform(-80, 80, n), rng.uniform(0.0, 0.6, n)]
    if weights:
        cols.append(rng.lognormal(0, 0.3, n))
    if n_jk > 1:
        cols.append(rng.integers(0, n_jk, n))
    if coords == "cartesian":
        cols.append(rng.integers(0, 9, n))  # an extra column the reader ignores
    path = tmp_path / "cat.txt"
    _write_catalogue(path, cols, sep, rng)
    ptext = (f"coord_system = {coords}\nuse_weights = {int(weights)}\nn_jk_regions = {n_jk}\n"
             "omega_m = 0.25\nh = 1.0\nz_min = 0.0\nz_max = 1.0\n")
    ref = refl.read_ascii(ptext, str(path))
    cosmo = ingest.Cosmology(0.25, 1.0, 0.0, 1.0) if coords == "equatorial" else None
    got = ingest.read_ascii(str(path), ingest.EQUATORIAL if coords == "equatorial" else ingest.CARTESIAN, weights,
                            n_jk, cosmo)
    assert got["d_comov"].size == n
    for k in ("xyz", "x_norm", "d_comov", "weight", "jk"):
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


def test_read_ascii_errors(tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("1 2 3\n4 5\n")
    with pytest.raises(ingest.HostError, match="line 2"):
        ingest.read_ascii(str(bad))
    bad.write_text("1 2 3 0.5\n4 5 6 x\n")
    with pytest.raises(ingest.HostError, match="weight"):
        ingest.read_ascii(str(bad), use_weights=True)
    bad.write_text("1,2,3,\n")  # trailing separator: the jackknife field is missing
    with pytest.raises(ingest.HostError, match="jk_region"):
        ingest.read_ascii(str(bad), n_jk_regions=3)
    with pytest.raises(ingest.HostError):
        ingest.read_ascii(str(tmp_path / "missing.txt"))
    with pytest.raises(ingest.HostError):
        ingest.read_ascii(str(bad), coord_system=ingest.EQUATORIAL)  # no cosmology


def test_sub_filename():
    assert ingest.sub_filename("out/xi_smu.txt", 3) == "out/xi_smu3.txt"
    assert ingest.sub_filename("./xi", 0) == "0./xi"  # the last '.' of the whole path
    assert ingest.sub_filename("a.b.c", 12) == "a.b12.c"
    with pytest.raises(ingest.HostError):
        ingest.sub_filename("noext", 1)


@pytest.mark.parametrize("mode,ax1,ax2", [
    (tp.MONOPOLE, (0.0, 100.0, 1.3, 30), None),
    (tp.MONOPOLE, (1.0, 40.0, 1.0, 13), None),
    (tp.SIGMA_PI, (0.0, 50.0, 1.0, 20), (0.0, 30.0, 1.5, 12)),
    (tp.S_MU, (0.0, 150.0, 1.3, 40), (0.0, 1.0, 0.0, 50)),
])
def test_write_xi_ascii_matches_reference(tmp_path, mode, ax1, ax2):
    n_jk = 3
    b = tp.Binning(None, mode, ax1, ax2, n_jk)
    rng = np.random.default_rng(int(mode) + 10 * ax1[3])
    nb = b.nb

    def hist(shape):
        h = rng.lognormal(0, 2, shape) * rng.choice([1e-9, 1e-3, 1.0, 1e6], shape)
        h[rng.random(shape) < 0.1] = 0.0
        return h

    dd, dr, rr = hist(nb), hist(nb), hist(nb)
    rr[:3] = 0.0  # ls_estimator gives 0 where RR == 0
    dd[5] = np.nan
    dr[6] = np.inf
    subs = [hist(n_jk * nb) for _ in range(3)]
    subs[0][7] = -np.inf
    ours = tmp_path / "ours" / "xi.dat"
    refs = tmp_path / "ref" / "xi.dat"
    ours.parent.mkdir()
    refs.parent.mkdir()
    ingest.write_xi_ascii(str(ours), b, dd, dr, rr, *subs)
    axp = [ax1[0], ax1[1], ax1[2]] + ([ax2[0], ax2[1], ax2[2]] if ax2 is not None else [0.0, 0.0, 0.0])
    nb2 = ax2[3] if ax2 is not None else 1
    refl.write_xi(str(refs), int(mode), axp, ax1[3], nb2, n_jk, dd, dr, rr, *subs)
    names = sorted(os.listdir(refs.parent))
    assert names == sorted(os.listdir(ours.parent)) == ["xi.dat", "xi0.dat", "xi1.dat", "xi2.dat"]
    for name in names:
        a = (ours.parent / name).read_bytes()
        r = (refs.parent / name).read_bytes()
        assert a == r, name


def test_write_xi_refuses_angular(tmp_path):
    b = tp.Binning(None, tp.ANGULAR, (0.0, 0.01, 1.6, 10), None, 1)
    z = np.zeros(10)
    with pytest.raises(ingest.HostError):
        ingest.write_xi_ascii(str(tmp_path / "a.txt"), b, z, z, z)
