"""ipfc_filter2d_noalloc: filter2D for callers that cannot allocate.

Some callers may not call cudaMalloc -- code running inside a custom
allocator, under a framework that has reserved the device's memory, or in a
pipeline that forbids allocation once started.  This entry point keeps its
tap list in a fixed device array instead of a per-call buffer and always runs
the FP32 CUDA-core form.  Its results must equal ipfc_filter2d_fp32's on the
same inputs and stay within the filter2D bar of the oracle, on consecutive
calls whose tap lists grow and shrink (the shared array then holds the
previous call's taps, which the new call must replace).  This file is
collected last on purpose; it passes alone in a fresh process as well as
after the rest of the suite.
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


def _call(fn, src, dst, k, border, delta, bv, stream=None, sync=True):
    import torch

    from imageprocessingflex_b200 import _lib

    sv, dv = _view(src), _view(dst)
    k = np.ascontiguousarray(k, np.float32)
    rc = getattr(_lib.load(), fn)(ctypes.byref(sv), ctypes.byref(dv), k.ctypes.data, k.shape[1], k.shape[0], -1, -1,
                                  border, delta, bv, stream)
    if sync:
        torch.cuda.synchronize()
    return rc


def _kernel(rng, kh, kw):
    k = rng.normal(size=(kh, kw))
    k = (k / k.sum()).astype(np.float32)
    k[0, 1 % kw] = 0.0  # a zero tap, dropped from the list like the reference does
    return k


def test_noalloc_matches_fp32_form_and_oracle_calls_in_a_row(gpu, orc):
    """Four calls in a row: the tap list grows (15x15 -> 31x31), shrinks
    (7x9) and grows again, so every call must overwrite what the last one left
    in the shared array."""
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(42)
    cases = [
        (oracle.random_image(301, 157, 1, np.uint8, 4), _kernel(rng, 15, 15), oracle.REFLECT101, 0.0, 0.0),
        (oracle.random_image(211, 97, 3, np.uint8, 5), _kernel(rng, 31, 31), oracle.REPLICATE, 0.0, 0.0),
        (oracle.random_image(256, 199, 1, np.float32, 6), _kernel(rng, 7, 9), oracle.CONSTANT, 0.25, 7.0),
        (oracle.random_image(190, 120, 1, np.uint8, 7), _kernel(rng, 21, 17), oracle.WRAP, 0.5, 3.0),
    ]
    for img, k, border, delta, bv in cases:
        src = torch.from_numpy(img).cuda()
        want = torch.empty_like(src)
        got = torch.empty_like(src)
        assert _call("ipfc_filter2d_fp32", src, want, k, border, delta, bv) == 0, lib.ipfc_last_error()
        assert _call("ipfc_filter2d_noalloc", src, got, k, border, delta, bv) == 0, lib.ipfc_last_error()
        g = got.cpu().numpy()
        np.testing.assert_array_equal(g, want.cpu().numpy())
        ref = orc.filter2d(img, k, border, delta, (-1, -1), bv)
        x = {"src": img, "kernel": k}
        G.compare(g, ref, G.tolerance("filter2d", {"delta": delta, "border_value": bv}, x, ref))


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


def test_noalloc_refuses_a_capturing_stream(gpu):
    """A call on a stream under capture returns IPFC_ERR_UNSUPPORTED and
    enqueues nothing, so the capture itself still ends cleanly; the same call
    outside capture then works."""
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    img = oracle.random_image(64, 48, 1, np.uint8, 9)
    k = _kernel(np.random.default_rng(1), 5, 5)
    src = torch.from_numpy(img).cuda()
    dst = torch.empty_like(src)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = _call("ipfc_filter2d_noalloc", src, dst, k, 3, 0.0, 0.0, stream=ctypes.c_void_p(s.cuda_stream),
                   sync=False)
    assert rc == 5, (rc, lib.ipfc_last_error())  # IPFC_ERR_UNSUPPORTED
    assert b"capturing" in lib.ipfc_last_error()
    del g
    want = torch.empty_like(src)
    assert _call("ipfc_filter2d_noalloc", src, dst, k, 3, 0.0, 0.0) == 0, lib.ipfc_last_error()
    assert _call("ipfc_filter2d_fp32", src, want, k, 3, 0.0, 0.0) == 0, lib.ipfc_last_error()
    np.testing.assert_array_equal(dst.cpu().numpy(), want.cpu().numpy())
