import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


@pytest.fixture(scope="session")
def orc():
    import oracle

    oracle.build()
    return oracle.restatement()


@pytest.fixture(scope="session")
def refimpl():
    import oracle

    oracle.build()
    r = oracle.reference()
    if r is None:
        pytest.skip("reference headers not compiled here (oracle/_ref absent)")
    return r


@pytest.fixture(scope="session")
def gpu():
    """The CUDA library's Python mirror, on a machine with a CUDA device."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    import imageprocessingflex_b200 as ipf

    return ipf


def pytest_terminal_summary(terminalreporter):
    """Where the parity bar was wider than 1 LSB / 1e-5, and by how much."""
    try:
        import golden_cases
    except ImportError:
        return
    lines = golden_cases.widened_report()
    if lines:
        terminalreporter.write_sep("-", "parity cases on a widened bar (FP32 summation bound above 1 LSB / 1e-5)")
        for ln in lines:
            terminalreporter.write_line(ln)
