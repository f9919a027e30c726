"""The kernels' border rule (border_index in csrc/common.cuh) against the
oracle's borderIndex (include/ipf/core.hpp:187-214), on the host.

border_index_check.cu compiles the kernels' own header for the host and
compares it with the oracle's C restatement on every position of every row
length up to 256 and on sampled lengths up to the C ABI's limit of 2^30 - 1
samples per row, for all five border modes.  The device evaluation of the
same function is checked value by value on the GPU through
ipfc_probe_border_index (test_gpu_parity.py).
"""
import os
import shutil
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "imageprocessingflex_b200", "csrc")
ORACLE_BUILD = os.path.join(ROOT, "oracle", "_build")


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return None


def test_border_index_matches_oracle(tmp_path):
    exe = nvcc()
    if exe is None:
        pytest.skip("nvcc not found")
    oracle.build()
    out = str(tmp_path / "border_index_check")
    cmd = [exe, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, os.path.join(ROOT, "tests", "border_index_check.cu"),
           "-L", ORACLE_BUILD, "-loracle", "-Xlinker", "-rpath", "-Xlinker", ORACLE_BUILD, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("ok "), r.stdout
