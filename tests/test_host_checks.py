"""Device rules of csrc/common.cuh against the oracle, on the host.

Each check program compiles the kernels' own header for the host and links
the oracle's C restatement:

* border_index_check.cu: the border rule (border_index) against borderIndex
  (include/ipf/core.hpp:187-214) on every position of every row length up
  to 256 and on sampled lengths up to the C ABI's limit of 2^30 - 1 samples
  per row, for all five border modes, and its interleaved form
  (border_sample) for 1 to 4 channels;
* tcol_layout_check.cu: the shared-memory operands and descriptors of the
  tensor-core separable kernel (csrc/sep_tcol.cuh), every MMA emulated from
  the descriptor bits under the canonical layouts, and its step walk;
* saturate_check.cu: the store rounding (sat_from_f) against saturate_cast
  (include/ipf/core.hpp:69-103) on all 2^32 float bit patterns, to uint8,
  uint16 and int16.

The device evaluation of both is checked value by value on the GPU through
ipfc_probe_border_index and ipfc_probe_saturate (test_gpu_parity.py).
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


def run_check(tmp_path, name):
    """Compiles tests/<name>.cu for the host against the oracle and runs it;
    returns its output line."""
    exe = nvcc()
    if exe is None:
        pytest.skip("nvcc not found")
    oracle.build()
    out = str(tmp_path / name)
    cmd = [exe, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-Xcompiler", "-fopenmp",
           os.path.join(ROOT, "tests", name + ".cu"),
           "-L", ORACLE_BUILD, "-loracle", "-Xlinker", "-rpath", "-Xlinker", ORACLE_BUILD, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout.strip()


def test_border_index_matches_oracle(tmp_path):
    assert run_check(tmp_path, "border_index_check").startswith("ok ")


def test_saturate_matches_oracle_on_every_float(tmp_path):
    assert run_check(tmp_path, "saturate_check") == f"ok {3 * (1 << 32)}"


def test_tcol_operand_layout(tmp_path):
    assert run_check(tmp_path, "tcol_layout_check").startswith("ok ")
