"""Shared test set-up.

Markers: ``gpu`` — needs a CUDA device (run with ``-m gpu`` on a B200).
The CPU suite (``-m "not gpu"``) checks the oracle against the reference
and the golden fixtures, the host logic, and that the C-ABI library loads
and exports every declared symbol.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


def _ensure_built():
    """Build the oracle restatement and the engine library if absent (both
    compile in seconds here; on a GPU box the prebuilt files are used)."""
    from oracle import port
    if not port.available():
        subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_oracle.sh")], check=True)
    from two_pcf_b200 import _capi
    if not os.path.exists(_capi.LIB_PATH):
        from two_pcf_b200 import build
        build.build()


_ensure_built()


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import two_pcf_b200 as tp
    c = tp.Context(0)
    yield c
    c.close()
