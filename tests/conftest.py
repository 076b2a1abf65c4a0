import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _reference_root():
    """The reference tree the oracle's recipe reads (oracle/Makefile, `print-ref`)."""
    import subprocess

    try:
        out = subprocess.run(["make", "-s", "--no-print-directory", "-C", os.path.join(ROOT, "oracle"), "print-ref"],
                             capture_output=True, text=True, timeout=30)
        return out.stdout.strip()
    except Exception:
        return ""


REFERENCE_ROOT = _reference_root()
HAVE_REFERENCE = os.path.isdir(os.path.join(REFERENCE_ROOT, "src"))
needs_reference = pytest.mark.skipif(not HAVE_REFERENCE, reason="reference source tree not present")
