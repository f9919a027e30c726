"""The C++ drop-in check: ipf::X against ipf::cuda::X on the reference's own
ipf::Image type (oracle/dropin_test.cpp, built against the reference headers
into oracle/_ref/dropin_test by oracle/Makefile)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "dropin_test")


def test_cpp_dropin_matches_reference(gpu):
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/dropin_test not built here (needs the reference headers at build time)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
    assert "dropin: all ok" in r.stdout
