"""The median selection networks of the 3x3 and 5x5 median kernels, proven
exact on the host: the packed uint8 networks (median9_2, median25_2 in
csrc/median_u8.cuh) and the forgetful selection of the other element types
(median_forgetful in csrc/median.cuh).

median_network_check.cu compiles the kernels' own headers for the host and
runs each network on every binary window (2^9 and 2^25 of them).  The
networks use only min and max, so by the 0-1 principle that covers every
window of ordered values (uint8; uint16, int16 and non-NaN floats for the
forgetful selection); a sample of random byte windows checks the two-lane
packing against std::nth_element as well.  medianBlur's reference result is the
sample of rank k*k/2 of the window (include/ipf/filter.hpp:302-332).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "imageprocessingflex_b200", "csrc")


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


def test_median_networks_exact_on_every_binary_window(tmp_path):
    exe = nvcc()
    if exe is None:
        pytest.skip("nvcc not found")
    out = str(tmp_path / "median_network_check")
    cmd = [exe, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-Xcompiler", "-fopenmp",
           os.path.join(ROOT, "tests", "median_network_check.cu"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == f"ok {2 * ((1 << 9) + (1 << 25)) + 400000}", r.stdout
