"""The C-ABI library: loads, exports every symbol include/*.h declares, checks
arguments with the reference's messages, and never computes on the CPU.

No compute call here reaches a GPU; the device-independent parts (argument
checks, FP64 tap generators) run on any machine.
"""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
from imageprocessingflex_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        with open(h) as f:
            text = f.read()
        names.update(re.findall(r"IPFC_API\s+[\w\s\*]*?\b(ipfc_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.library_path() if os.path.exists(_lib.library_path()) else _lib.load()._name)
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding describes each of them
    bound = set(_lib.exported_names())
    assert set(names) <= bound, sorted(set(names) - bound)


def test_version():
    assert _lib.load().ipfc_version() >> 16 == 1


def test_tap_generators_match_restatement(orc):
    for s in (0.5, 1.0, 2.0, 2.3, 4.0):
        np.testing.assert_array_equal(ipf.gaussianKernel1D(s), orc.gaussian_kernel_1d(s))
    np.testing.assert_array_equal(ipf.gaussianKernel1D(0, 7), orc.gaussian_kernel_1d(0, 7))
    for order, k in ((1, 3), (1, 5), (2, 5), (0, 7), (1, 1), (2, 1), (3, 31)):
        np.testing.assert_array_equal(ipf.derivKernel(order, k), orc.deriv_kernel(order, k))
    for shape in (0, 1, 2):
        for w, h in ((3, 3), (5, 7), (9, 5), (1, 1), (4, 2)):
            np.testing.assert_array_equal(ipf.getStructuringElement(shape, w, h), orc.structuring_element(shape, w, h))


@pytest.mark.parametrize("call, msg", [
    (lambda x: ipf.medianBlur(x, 4), "ipf: medianBlur: ksize must be odd and positive"),
    (lambda x: ipf.medianBlur(x, 3, ipf.BorderMode.Constant), "ipf: medianBlur: Constant border is not supported"),
    (lambda x: ipf.sepFilter2D(x, [], [1.0]), "ipf: separable filter: empty kernel"),
    (lambda x: ipf.boxFilter(x, 0, 3), "ipf: boxFilter: kernel size must be positive"),
    (lambda x: ipf.gaussianBlur(x, 0.0), "ipf: gaussianKernel1D: need sigma > 0 or ksize > 0"),
    (lambda x: ipf.gaussianBlur(x, 1.0, 0.0, 4), "ipf: gaussianKernel1D: ksize must be odd"),
    (lambda x: ipf.sobel(x, 0, 0), "ipf: sobel: need dx + dy > 0"),
    (lambda x: ipf.sobel(x, 1, 0, 4), "ipf: derivKernel: ksize must be odd in [3, 31]"),
    (lambda x: ipf.filter2D(x, np.ones((3, 3)), anchor=(3, 0)), "ipf: filter2D: anchor outside kernel"),
    (lambda x: ipf.filter2D(x, np.ones((0, 3))), "ipf: filter2D: kernel must be a non-empty single-channel image"),
    (lambda x: ipf.erode(x, np.ones((0, 0))),
     "ipf: morphology: structuring element must be a non-empty single-channel mask"),
])
def test_argument_errors_carry_reference_messages(call, msg):
    x = np.zeros((8, 8), np.uint8)
    with pytest.raises(ipf.Error) as e:
        call(x)
    assert str(e.value) == msg
    assert e.value.status == 1


def test_structuring_element_error():
    with pytest.raises(ipf.Error, match="ipf: getStructuringElement: size must be positive"):
        ipf.getStructuringElement(ipf.MorphShape.Rect, 0)


def test_unknown_dtype_code_is_rejected():
    """Element codes outside the reference's six image types are refused
    before any device work (IPFC_ERR_UNSUPPORTED)."""
    import ctypes

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    x = np.zeros((4, 4), np.uint8)
    sv = _lib.IpfcImage(x.ctypes.data, 4, 4, 1, 9, 4, 0)
    dv = _lib.IpfcImage(x.ctypes.data, 4, 4, 1, 0, 4, 0)
    assert lib.ipfc_gaussian_blur(ctypes.byref(sv), ctypes.byref(dv), 1.0, 0.0, 0, 3, None) == 5
    assert b"element type" in lib.ipfc_last_error()


def test_empty_image_returns_empty():
    out = ipf.gaussianBlur(np.zeros((0, 5, 3), np.uint8), 2.0)
    assert out.shape == (0, 5, 3)


def test_no_cpu_fallback_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(ipf.Error) as e:
        ipf.gaussianBlur(np.zeros((4, 4), np.uint8), 1.0)
    assert e.value.status == 3
    assert "no CUDA device" in str(e.value)


# ---- batch API: argument checks and the autotune table (no GPU needed) -------

def test_batch_rejects_host_images_and_null_batch():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.ipfc_batch_create(ctypes.byref(h)) == 0
    x = np.zeros((4, 4), np.uint8)
    y = np.zeros((4, 4), np.uint8)
    sv = _lib.IpfcImage(x.ctypes.data, 4, 4, 1, 0, 4, 0)
    dv = _lib.IpfcImage(y.ctypes.data, 4, 4, 1, 0, 4, 0)
    assert lib.ipfc_batch_add_gaussian_blur(h, ctypes.byref(sv), ctypes.byref(dv), 1.0, 0.0, 0, 3) == 1
    assert "batched images must be in device memory" in lib.ipfc_last_error().decode()
    sv.mem = dv.mem = 1
    sv.dtype = dv.dtype = 4
    assert lib.ipfc_batch_add_median_blur(h, ctypes.byref(sv), ctypes.byref(dv), 3, 1) == 5
    assert "uint8" in lib.ipfc_last_error().decode()
    assert lib.ipfc_batch_add_median_blur(None, ctypes.byref(sv), ctypes.byref(dv), 3, 1) == 1
    v = ctypes.c_longlong(-1)
    assert lib.ipfc_batch_info(h, 0, ctypes.byref(v)) == 0 and v.value == 0
    assert lib.ipfc_batch_run(h, None) == 0  # nothing to do
    assert lib.ipfc_batch_set_option(h, 99, 1) == 1
    assert lib.ipfc_batch_destroy(h) == 0


def test_autotune_table_round_trip(tmp_path):
    from imageprocessingflex_b200 import batch as B

    B.tune_clear()
    assert B.tune_get(B.OP_SEP, 13, 3, 2) is None
    B.tune_set(B.OP_SEP, 13, 3, 2, 104)
    B.tune_set(B.OP_MEDIAN, 5, 1, 0, 256, 16)
    with pytest.raises(ipf.Error):
        B.tune_set(B.OP_MEDIAN, 5, 1, 9, 256, 16)
    p = str(tmp_path / "tune.txt")
    B.tune_save(p)
    B.tune_clear()
    assert B.tune_get(B.OP_SEP, 13, 3, 2) is None
    assert B.tune_load(p) == 2
    assert B.tune_get(B.OP_SEP, 13, 3, 2) == (104, 0)
    assert B.tune_get(B.OP_MEDIAN, 5, 1, 0) == (256, 16)
    B.tune_clear()


def test_uneven_mix_is_seeded():
    from imageprocessingflex_b200 import mix

    a = mix.uneven_mix(512, seed=2024)
    b = mix.uneven_mix(512, seed=2024)
    assert a == b
    ops = [it.op for it in a]
    assert 0.4 < ops.count("gaussian") / 512 < 0.6
    assert all(64 <= it.width <= 2048 and 64 <= it.height <= 2048 and it.channels in (1, 3, 4) for it in a)
    assert all(0.5 <= it.sigma <= 4.0 for it in a if it.op == "gaussian")


def test_server_argument_checks():
    lib = _lib.load()
    r = _lib.IpfcRequest()
    r.op = 99
    assert lib.ipfc_server_submit(None, ctypes.byref(r), None) == 1
    cfg = _lib.IpfcServerConfig(0, 1, 1, 1)
    h = ctypes.c_void_p()
    assert lib.ipfc_server_create(ctypes.byref(h), ctypes.byref(cfg)) == 1
    assert "invalid configuration" in lib.ipfc_last_error().decode()
    assert lib.ipfc_server_destroy(None) == 0


def test_served_stream_is_seeded():
    from imageprocessingflex_b200 import mix

    a = mix.served_stream(4000, rate=3000.0, seed=77)
    assert a == mix.served_stream(4000, rate=3000.0, seed=77)
    px = np.array([r.pixels for r in a])
    assert 1e4 * 0.99 <= px.min() and px.max() <= 33e6 * 1.01
    assert 0.8e6 < np.median(px) < 1.25e6
    gaps = np.diff([r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 3000.0) < 0.1 / 3000.0
    ops = [r.op for r in a]
    assert abs(ops.count("gaussian") / len(a) - 0.45) < 0.03
    t = mix.filter2d_taps()
    assert t.shape == (15, 15) and abs(float(t.sum()) - 1.0) < 1e-5
