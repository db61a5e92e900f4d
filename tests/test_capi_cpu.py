"""Host-side checks of the C-ABI library that need no GPU: it loads, exports
every symbol include/two_pcf_b200.h declares, validates arguments, and its
threshold tables reproduce the reference binning exactly."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import two_pcf_b200 as tp
from two_pcf_b200 import _capi
from oracle import port

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "two_pcf_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tpcf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if line.strip())
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    lib = _capi.lib()
    for s in syms:
        assert hasattr(lib, s)
    assert set(_capi._PROTOTYPES) >= set(syms)


def test_status_strings_and_version():
    lib = _capi.lib()
    assert lib.tpcf_abi_version() == 1
    for st in range(7):
        assert lib.tpcf_status_string(st)
    assert lib.tpcf_status_string(99) == b"unknown status"


def test_ls_estimator_matches_reference_formula():
    # src/io.cpp:643-651
    for dd, dr, rr in [(1.0, 2.0, 3.0), (0.5, 0.1, 0.0), (1e-7, 3e-7, 2e-7)]:
        exp = 0.0 if rr == 0 else dd / rr - 2.0 * dr / rr + 1.0
        assert _capi.lib().tpcf_ls_estimator(dd, dr, rr) == exp
        assert port.lib().orc_ls(dd, dr, rr) == exp


def test_argument_validation_without_device():
    lib = _capi.lib()
    h = C.c_void_p()
    # bad mode, bad bins, missing ax2
    ax = _capi.AxisSpec(0.0, 100.0, 1.3, 30)
    assert lib.tpcf_binning_create(None, 9, C.byref(ax), None, 1, C.byref(h)) == _capi.TPCF_E_INVALID_ARG
    bad = _capi.AxisSpec(0.0, 100.0, 1.3, 0)
    assert lib.tpcf_binning_create(None, 0, C.byref(bad), None, 1, C.byref(h)) == _capi.TPCF_E_INVALID_ARG
    inv = _capi.AxisSpec(10.0, 5.0, 1.0, 5)
    assert lib.tpcf_binning_create(None, 0, C.byref(inv), None, 1, C.byref(h)) == _capi.TPCF_E_INVALID_ARG
    assert lib.tpcf_binning_create(None, 2, C.byref(ax), None, 1, C.byref(h)) == _capi.TPCF_E_INVALID_ARG
    assert lib.tpcf_binning_create(None, 0, C.byref(ax), None, 0, C.byref(h)) == _capi.TPCF_E_INVALID_ARG
    assert lib.tpcf_count(None, None, None, None, 0, None, None, None) == _capi.TPCF_E_INVALID_ARG
    assert lib.tpcf_destroy(None) == _capi.TPCF_E_INVALID_ARG


@pytest.mark.parametrize("mode,ax1,ax2,space1,space2", [
    (tp.MONOPOLE, (0.0, 100.0, 1.3, 30), None, 1, None),
    (tp.MONOPOLE, (5.0, 80.0, 1.0, 15), None, 1, None),
    (tp.S_MU, (0.0, 100.0, 1.3, 40), (0.0, 1.0, 0.0, 50), 1, 0),
    (tp.SIGMA_PI, (0.0, 50.0, 1.0, 50), (0.0, 50.0, 1.0, 50), 1, 0),
    (tp.SIGMA_PI, (0.5, 40.0, 1.4, 12), (0.0, 30.0, 1.0, 10), 1, 0),
    (tp.S_MU, (0.0, 150.0, 1.3, 40), (0.0, 1.0, 0.0, 50), 1, 0),
])
def test_thresholds_reproduce_reference_bins(mode, ax1, ax2, space1, space2):
    """bin = #{T <= x} - 1 for every x: check at and just below each threshold
    and on a dense sample, with the oracle's Axis::bin_num (glibc log1pf)."""
    b = tp.Binning(None, mode, ax1, ax2)
    L = port.lib()

    def ref_bin(ax, x, sq):
        v = np.sqrt(np.float32(x)).astype(np.float32) if sq else np.float32(x)
        f = L.orc_axis_bin_num(C.byref(ax), float(v))
        return int(L.orc_to_int(C.c_float(f)))

    L.orc_to_int.argtypes = [C.c_float]
    L.orc_to_int.restype = C.c_int
    for axis, spec, sq in ((1, ax1, space1), (2, ax2, space2)):
        if spec is None:
            continue
        if mode == tp.S_MU and axis == 2:
            spec = (0.0, 1.0, 0.0, spec[3])
        oax = port.axis(spec[0], spec[1], spec[3], spec[2])
        t = b.thresholds(axis)
        assert t.size == spec[3] + 1
        assert np.all(np.diff(t[np.isfinite(t)]) >= 0)
        for k, tk in enumerate(t):
            if not np.isfinite(tk) or tk <= 0:
                continue
            assert ref_bin(oax, tk, sq) >= k
            below = np.nextafter(np.float32(tk), np.float32(-1))
            assert ref_bin(oax, below, sq) < k
        hi = float(t[np.isfinite(t)].max()) * 1.01 + 1.0
        xs = np.concatenate([np.linspace(0, hi, 4001), np.geomspace(1e-8, hi, 2001)]).astype(np.float32)
        n = spec[3]
        for x in xs:
            cnt = int(np.sum(t <= x)) - 1
            rb = ref_bin(oax, x, sq)
            # out of [0, n): dropped either way
            assert (cnt if 0 <= cnt < n else -1) == (rb if 0 <= rb < n else -1), (axis, x)


@pytest.mark.parametrize("spec,sq,hi", [
    ((0.0, 100.0, 30, 1.3), 1, 1e4),
    ((0.0, 100.0, 40, 1.3), 1, 1e4),
    ((0.0, 150.0, 40, 1.3), 1, 2.25e4),
    ((0.0, 50.0, 50, 1.0), 1, 5000.0),
    ((0.0, 50.0, 50, 1.0), 0, 80.0),
    ((0.0, 1.0, 50, 0.0), 0, 2.0),
])
def test_reference_binning_monotone_exhaustive(spec, sq, hi):
    """Every float of the domain: the binning never decreases (what the
    threshold tables assume).  Covers the shipped benchmark axes."""
    L = port.lib()
    L.orc_axis_check_monotone.argtypes = [C.POINTER(port.OrcAxis), C.c_int, C.c_float, C.c_float]
    L.orc_axis_check_monotone.restype = C.c_uint
    ax = port.axis(*spec)
    assert L.orc_axis_check_monotone(C.byref(ax), sq, 0.0, hi) == 0xFFFFFFFF


def test_release_build_has_no_device_checks():
    """The release library reports no device checks and refuses the test hook
    that would plant a bad index (nothing there would catch it)."""
    L = _capi.lib()
    assert L.tpcf_device_checks() == 0
    assert L.tpcf_debug_corrupt_work_list(1) == _capi.TPCF_E_UNSUPPORTED
    assert L.tpcf_status_string(_capi.TPCF_E_DEVICE_CHECK).decode() == "device bounds check failed"


def test_checked_build_exports_the_same_symbols():
    import ctypes
    import os
    import subprocess
    path = _capi.CHECKED_LIB_PATH
    if not os.path.exists(path):
        pytest.skip("checked build absent (TPCF_DEVICE_CHECKS=1 python two_pcf_b200/build.py)")
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert set(_capi._PROTOTYPES) <= exported
    L = ctypes.CDLL(path)
    assert L.tpcf_device_checks() == 1
