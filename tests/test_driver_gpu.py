"""End to end through the command-line program: parameter file -> ASCII
catalogues -> DD, DR, RR on the GPU -> normalised ASCII outputs, against the
reference's own program (oracle/_ref/twopcf_ref, built from its sources) on
the same files, or, where that build is absent, against its committed outputs
(tests/golden/driver_outputs.json, made by tests/golden/make_driver_golden.py).

Unit-weight outputs must be byte-identical.  Weighted sums agree to about
1e-12 relative (both sum the same float pair weights, in different orders),
so a printed 6-significant-digit value may differ in its last digit where it
sits on a rounding boundary: such lines are compared numerically to 2e-6
relative, and must be rare."""
import importlib.util
import json
import os
import subprocess

import numpy as np
import pytest

from two_pcf_b200 import _capi, ingest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(os.path.dirname(_capi.LIB_PATH), "two_pcf")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "twopcf_ref")
GOLDEN = os.path.join(ROOT, "tests", "golden", "driver_outputs.json")


def _gen():
    spec = importlib.util.spec_from_file_location("make_driver_golden",
                                                  os.path.join(ROOT, "tests", "golden", "make_driver_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _compare(ours: str, ref: str, weighted: bool, name: str):
    if ours == ref:
        return 0
    assert weighted, f"{name}: unit-weight output differs from the reference"
    lo, lr = ours.splitlines(), ref.splitlines()
    assert len(lo) == len(lr), name
    n_diff = 0
    for a, b in zip(lo, lr):
        if a == b:
            continue
        n_diff += 1
        va = np.array([float(t) for t in a.split("\t")])
        vb = np.array([float(t) for t in b.split("\t")])
        np.testing.assert_allclose(va, vb, rtol=2e-6, atol=0, equal_nan=True, err_msg=f"{name}: {a!r} vs {b!r}")
    return n_diff


def _run_ours(params, *extra):
    r = subprocess.run([CLI, params, "--quiet", *extra], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("case", ["box_weighted_jk", "sky_unit"])
def test_cli_matches_reference_outputs(tmp_path, case):
    g = _gen()
    out_dir = tmp_path / "out"
    out_dir.mkdir()
    params, names = g.write_inputs(case, str(tmp_path), str(out_dir))
    _run_ours(params)
    ours = {n: (out_dir / n).read_text() for n in sorted(os.listdir(out_dir))}
    if os.path.exists(REF_CLI):
        ref_dir = tmp_path / "ref"
        ref_dir.mkdir()
        ref_params, _ = g.write_inputs(case, str(tmp_path), str(ref_dir))
        subprocess.run([REF_CLI, ref_params], check=True, stdout=subprocess.DEVNULL, timeout=300)
        ref = {n: (ref_dir / n).read_text() for n in sorted(os.listdir(ref_dir))}
    else:
        gold = json.load(open(GOLDEN))[case]
        assert g.input_digest(str(tmp_path)) == gold["inputs_sha256"], "regenerated inputs differ from the fixture's"
        ref = gold["files"]
    assert sorted(ours) == sorted(ref)
    weighted = case == "box_weighted_jk"
    n_lines = sum(len(t.splitlines()) for t in ref.values())
    n_diff = sum(_compare(ours[n], ref[n], weighted, n) for n in ref)
    assert n_diff <= max(2, n_lines // 100)


def test_cli_golden_fixture_matches(tmp_path):
    """The committed fixture itself, whatever reference build is present."""
    g = _gen()
    gold = json.load(open(GOLDEN))
    for case in ("box_weighted_jk", "sky_unit"):
        d = tmp_path / case
        out_dir = d / "out"
        out_dir.mkdir(parents=True)
        params, _ = g.write_inputs(case, str(d), str(out_dir))
        assert g.input_digest(str(d)) == gold[case]["inputs_sha256"]
        ingest.run_param_file(params)
        for n, text in gold[case]["files"].items():
            _compare((out_dir / n).read_text(), text, case == "box_weighted_jk", n)


def test_cli_fp64_path_same_counts(tmp_path):
    g = _gen()
    a, b = tmp_path / "a", tmp_path / "b"
    for d in (a, b):
        (d / "out").mkdir(parents=True)
    pa, _ = g.write_inputs("sky_unit", str(a), str(a / "out"))
    pb, _ = g.write_inputs("sky_unit", str(b), str(b / "out"))
    _run_ours(pa)
    _run_ours(pb, "--fp64")
    for n in os.listdir(a / "out"):
        assert (a / "out" / n).read_bytes() == (b / "out" / n).read_bytes()


def test_cli_errors(tmp_path):
    g = _gen()
    params, _ = g.write_inputs("sky_unit", str(tmp_path), str(tmp_path))
    text = open(params).read()
    bad = tmp_path / "hdf5.ini"
    bad.write_text(text.replace("data_file_type = ascii", "data_file_type = hdf5"))
    r = subprocess.run([CLI, str(bad), "--quiet"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2 and "HDF5" in r.stderr
    with pytest.raises(ingest.HostError) as e:
        ingest.run_param_file(str(bad))
    assert e.value.status == _capi.TPCF_E_UNSUPPORTED
    r = subprocess.run([CLI], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "usage" in r.stderr


@pytest.mark.parametrize("case", ["box_weighted_jk", "sky_unit"])
def test_cli_summary_reports_error_against_fp64(tmp_path, case):
    """two_pcf --summary FILE --check-fp64: the JSON run summary gives every
    mode's counts and, per output, the largest difference from the plain FP64
    path.  The two paths sum the same float pair weights exactly in fixed
    point, so every raw and normalised histogram and every xi agrees bit for
    bit; the report must say so, and its pair counts must add up."""
    g = _gen()
    out_dir = tmp_path / "out"
    out_dir.mkdir()
    params, _ = g.write_inputs(case, str(tmp_path), str(out_dir))
    summ = tmp_path / "summary.json"
    _run_ours(params, "--summary", str(summ), "--check-fp64")
    s = json.load(open(summ))
    assert s["status"] == 0 and s["error"] is None and s["fp64_check"] is True
    assert s["precision"] == "fp32_guard" and s["catalogues"]["data"]["kept"] > 0
    assert len(s["modes"]) >= 1
    pairs = 0
    for m in s["modes"]:
        for lab in ("DD", "DR", "RR"):
            c = m["counts"][lab]
            assert c["in_range_pairs"] > 0 and c["kernel_ms"] > 0 and c["pairs_per_s"] > 0
            pairs += c["in_range_pairs"]
            for key in (lab, lab + "_raw"):
                e = m["fp64_check"][key]
                assert e["bit_identical"] and e["max_rel_err"] == 0.0 and e["nonfinite_mismatch"] == 0
                assert e["values"] == (1 + m["n_jk_regions"]) * m["bins"]
        assert m["fp64_check"]["xi"]["max_rel_err"] == 0.0
    assert s["in_range_pairs"] == pairs
    # the same through the Python wrapper, which returns the summary
    s2 = ingest.run_param_file(params, check_fp64=True, summary=str(tmp_path / "s2.json"))
    assert [m["mode"] for m in s2["modes"]] == [m["mode"] for m in s["modes"]]
    assert [m["counts"]["RR"]["in_range_pairs"] for m in s2["modes"]] == \
        [m["counts"]["RR"]["in_range_pairs"] for m in s["modes"]]
    assert all(m["fp64_check"]["xi"]["bit_identical"] for m in s2["modes"])


def test_cli_summary_of_a_failed_run(tmp_path):
    g = _gen()
    params, _ = g.write_inputs("sky_unit", str(tmp_path), str(tmp_path))
    bad = tmp_path / "hdf5.ini"
    bad.write_text(open(params).read().replace("data_file_type = ascii", "data_file_type = hdf5"))
    summ = tmp_path / "summary.json"
    r = subprocess.run([CLI, str(bad), "--quiet", "--summary", str(summ)], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 2
    s = json.load(open(summ))
    assert s["status"] == _capi.TPCF_E_UNSUPPORTED and "HDF5" in s["error"] and s["modes"] == []
