"""ipfc_filter2d_noalloc: filter2D for callers that cannot allocate.

Some callers may not call cudaMalloc -- code running inside a custom
allocator, under a framework that has reserved the device's memory, or in a
pipeline that forbids allocation once started.  This entry point keeps its
tap list in a fixed device array instead of a per-call buffer.  Its results
must equal ipfc_filter2d's on the same inputs, also on a second call in a
row (the shared array then holds the previous call's taps, which the new
call must replace).  This file is collected last on purpose; it passes alone
in a fresh process as well as after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import golden_cases as G
import oracle

pytestmark = pytest.mark.gpu


def _view(t):
    from imageprocessingflex_b200 import _lib

    h, w = t.shape[0], t.shape[1]
    c = t.shape[2] if t.dim() == 3 else 1
    code = {"torch.uint8": 0, "torch.float32": 4}[str(t.dtype)]
    return _lib.IpfcImage(t.data_ptr(), w, h, c, code, t.stride(0) * t.element_size(), 1)


def _call(fn, src, dst, k, border, delta, bv):
    import torch

    from imageprocessingflex_b200 import _lib

    sv, dv = _view(src), _view(dst)
    k = np.ascontiguousarray(k, np.float32)
    rc = getattr(_lib.load(), fn)(ctypes.byref(sv), ctypes.byref(dv), k.ctypes.data, k.shape[1], k.shape[0], -1, -1,
                                  border, delta, bv, None)
    torch.cuda.synchronize()
    return rc


def test_noalloc_matches_filter2d_two_calls_in_a_row(gpu):
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(42)
    cases = [
        (oracle.random_image(301, 157, 3, np.uint8, 5), rng.normal(size=(15, 15)), 3, 0.0, 0.0),
        (oracle.random_image(256, 199, 1, np.float32, 6), rng.normal(size=(7, 9)), 0, 0.25, 7.0),
    ]
    for img, k, border, delta, bv in cases:
        k = (k / k.sum()).astype(np.float32)
        k[0, 1] = 0.0  # a zero tap, dropped from the list like the reference does
        src = torch.from_numpy(img).cuda()
        want = torch.empty_like(src)
        got = torch.empty_like(src)
        assert _call("ipfc_filter2d", src, want, k, border, delta, bv) == 0, lib.ipfc_last_error()
        assert _call("ipfc_filter2d_noalloc", src, got, k, border, delta, bv) == 0, lib.ipfc_last_error()
        x = {"src": img, "kernel": k}
        G.compare(got.cpu().numpy(), want.cpu().numpy(),
                  G.tolerance("filter2d", {"delta": delta, "border_value": bv}, x, want.cpu().numpy()))
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())


def test_noalloc_rejects_oversized_kernels_and_host_images(gpu):
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    src = torch.zeros((16, 16), dtype=torch.uint8, device="cuda")
    dst = torch.empty_like(src)
    assert _call("ipfc_filter2d_noalloc", src, dst, np.ones((65, 65), np.float32), 3, 0.0, 0.0) == 1
    assert b"capacity of 4096" in lib.ipfc_last_error()
    img = np.zeros((16, 16), np.uint8)
    out = np.zeros_like(img)
    sv = _lib.IpfcImage(img.ctypes.data, 16, 16, 1, 0, 16, 0)
    dv = _lib.IpfcImage(out.ctypes.data, 16, 16, 1, 0, 16, 0)
    k = np.ones((3, 3), np.float32)
    assert lib.ipfc_filter2d_noalloc(ctypes.byref(sv), ctypes.byref(dv), k.ctypes.data, 3, 3, -1, -1, 3, 0.0, 0.0,
                                     None) == 1
    assert b"device memory" in lib.ipfc_last_error()
