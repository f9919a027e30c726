"""Failure paths that a test can reach without faulting a GPU.

* A device-side wait that runs out: the tensor-core kernels bound every
  pipeline wait (ipfc_set_wait_limit_ns).  With the bound shortened to a
  nanosecond a wait gives up, the kernel ends early, the call reports
  IPFC_ERR_TIMEOUT, and -- since the kernel waits for every MMA it issued
  before freeing its tensor memory, on a bound of its own -- the next call
  with the normal bound runs correctly.
* An allocation that fails inside the request server (injected on the host):
  that request completes with IPFC_ERR_NOMEM and every other request in the
  mix completes with the same result it has alone.

The reference's counterpart is exception propagation out of its thread pool
(include/ipf/parallel.hpp:69-93): a failed piece of work is reported, the
rest of the program continues.
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
import oracle
from imageprocessingflex_b200 import _lib, mix
from imageprocessingflex_b200 import serve as S

pytestmark = pytest.mark.gpu

IPFC_ERR_NOMEM, IPFC_ERR_TIMEOUT = 2, 4


def _timed_out(call):
    lib = _lib.load()
    lib.ipfc_set_wait_limit_ns(1)
    try:
        with pytest.raises(ipf.Error) as e:
            call()
    finally:
        lib.ipfc_set_wait_limit_ns(0)
    return e.value


def test_filter2d_split_wait_runs_out_then_recovers(gpu):
    img = oracle.random_image(1500, 900, 1, np.uint8, 21)
    k = mix.filter2d_taps(31, seed=1031)
    want = ipf.filter2D(img, k, form="split")
    err = _timed_out(lambda: ipf.filter2D(img, k, form="split"))
    assert err.status == IPFC_ERR_TIMEOUT and "wait gave up" in str(err)
    for _ in range(2):  # later calls are correct again
        np.testing.assert_array_equal(ipf.filter2D(img, k, form="split"), want)


def test_tcol_wait_runs_out_then_recovers(gpu):
    """The same for the separable kernel with the column pass on tcgen05; run
    in a child process because that kernel is selected by IPFC_SEP_PATH."""
    import os
    import subprocess
    import sys

    code = r'''
import numpy as np, imageprocessingflex_b200 as ipf, oracle
from imageprocessingflex_b200 import _lib
img = oracle.random_image(1200, 700, 3, np.uint8, 5)
want = oracle.restatement().gaussian_blur(img, 2.0)
lib = _lib.load()
lib.ipfc_set_wait_limit_ns(1)
try:
    ipf.gaussianBlur(img, 2.0)
    raise SystemExit("no timeout reported")
except ipf.Error as e:
    assert e.status == 4, e
finally:
    lib.ipfc_set_wait_limit_ns(0)
for _ in range(2):
    d = np.abs(ipf.gaussianBlur(img, 2.0).astype(int) - want.astype(int))
    assert d.max() <= 1, d.max()
print("tcol recovered")
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, IPFC_SEP_PATH="tcol", PYTHONPATH=root)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "tcol recovered" in r.stdout, r.stdout[-2000:] + r.stderr[-3000:]


def test_server_allocation_failure_fails_one_request_only(gpu):
    import torch

    def pinned(shape, seed):
        g = torch.Generator()
        g.manual_seed(seed)
        return torch.randint(0, 256, shape, dtype=torch.int32, generator=g).to(torch.uint8).pin_memory()

    for cfg in ({}, {"max_inflight": 1, "streams": 1, "batch": False}):
        with S.Server(**cfg) as server:
            server.fail_allocation(5)  # the 5th buffer taken (in arrival order: the third request's source)
            jobs = []
            for i in range(8):
                src = pinned((97 + 13 * i, 120, 3), 50 + i)
                dst = torch.empty_like(src).pin_memory()
                t = server.submit("gaussian", src, dst, sigma_x=1.5)
                jobs.append((t, src, dst))
            server.drain(60000)
            comps = {c.ticket: c for c in server.poll(100)}
        assert len(comps) == 8
        failed = [t for t, _, _ in jobs if comps[t].status != 0]
        assert len(failed) == 1 and comps[failed[0]].status == IPFC_ERR_NOMEM, cfg
        if cfg:  # one slot, one stream: requests take their buffers in arrival order
            assert failed == [jobs[2][0]]
        for t, src, dst in jobs:
            if t != failed[0]:
                np.testing.assert_array_equal(dst.numpy(), ipf.gaussianBlur(src.numpy(), 1.5))
