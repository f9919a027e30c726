"""Python mirror of ipf's neighbourhood-filter functions over the CUDA C ABI.

Names, argument order, defaults and error texts follow the reference's free
functions (include/ipf/filter.hpp, include/ipf/morphology.hpp).  The output
type template parameter ``TOut`` of the reference is the ``dtype`` keyword.

Images are ``numpy`` arrays shaped (H, W) or (H, W, C) -- host memory, the
call copies in and out and returns a new array -- or CUDA ``torch`` tensors of
the same shapes -- device memory, the call is asynchronous on ``stream``
(default: torch's current stream) and returns a new tensor.  Every call runs
on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes
from enum import IntEnum

import numpy as np

from . import _lib


class BorderMode(IntEnum):
    """ipf::BorderMode (core.hpp:183)."""

    Constant = 0
    Replicate = 1
    Reflect = 2
    Reflect101 = 3
    Wrap = 4


class MorphShape(IntEnum):
    """ipf::MorphShape (morphology.hpp:21)."""

    Rect = 0
    Cross = 1
    Ellipse = 2


class MorphOp(IntEnum):
    """ipf::MorphOp (morphology.hpp:129-138)."""

    Erode = 0
    Dilate = 1
    Open = 2
    Close = 3
    Gradient = 4
    TopHat = 5
    BlackHat = 6


class AdaptiveMethod(IntEnum):
    """ipf::AdaptiveMethod (filter.hpp:545)."""

    Mean = 0
    Gaussian = 1


class ThresholdType(IntEnum):
    """ipf::ThresholdType (pixel_ops.hpp:253-259); adaptiveThreshold takes the first two."""

    Binary = 0
    BinaryInv = 1
    Trunc = 2
    ToZero = 3
    ToZeroInv = 4


class Error(RuntimeError):
    """ipf::Error (core.hpp:35-38): every failure is reported with this type."""

    def __init__(self, message: str, status: int = 1):
        super().__init__(message)
        self.status = status


U8, U16, I16, I32, F32, F64 = range(6)
_NP_CODE = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.int16): I16,
            np.dtype(np.int32): I32, np.dtype(np.float32): F32, np.dtype(np.float64): F64}
_CODE_NP = {v: k for k, v in _NP_CODE.items()}
MEM_HOST, MEM_DEVICE = 0, 1


def _torch():
    import torch  # imported lazily: host-array use needs no torch

    return torch


def _is_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and hasattr(x, "is_cuda")


def _torch_code(t) -> int:
    torch = _torch()
    table = {torch.uint8: U8, torch.uint16: U16, torch.int16: I16, torch.int32: I32,
             torch.float32: F32, torch.float64: F64}
    if t.dtype not in table:
        raise Error(f"ipf: unsupported tensor dtype {t.dtype}", 5)
    return table[t.dtype]


def _code_of(dtype, like) -> int:
    """Element code of an output dtype request (numpy or torch dtype), or of `like`."""
    if dtype is None:
        return _torch_code(like) if _is_tensor(like) else _NP_CODE[like.dtype]
    if _is_tensor(like) or type(dtype).__module__.startswith("torch"):
        torch = _torch()
        table = {torch.uint8: U8, torch.uint16: U16, torch.int16: I16, torch.int32: I32,
                 torch.float32: F32, torch.float64: F64}
        if dtype in table:
            return table[dtype]
    return _NP_CODE[np.dtype(dtype)]


def _dims(x):
    if x.ndim == 2:
        return x.shape[1], x.shape[0], 1
    if x.ndim == 3:
        return x.shape[1], x.shape[0], x.shape[2]
    raise Error("ipf: image must be shaped (H, W) or (H, W, C)")


def _view(x) -> _lib.IpfcImage:
    """ipfc_image describing array/tensor x (rows may be pitched, samples dense)."""
    w, h, c = _dims(x)
    if _is_tensor(x):
        if not x.is_cuda:
            raise Error("ipf: torch tensors must live on a CUDA device (use numpy arrays for host images)")
        es = x.element_size()
        st = [s * es for s in x.stride()]
        dense_row = (x.ndim == 2 and st[1] == es) or (x.ndim == 3 and st[2] == es and st[1] == c * es)
        if not dense_row:
            raise Error("ipf: image rows must be contiguous (interleaved channels)")
        return _lib.IpfcImage(x.data_ptr(), w, h, c, _torch_code(x), st[0], MEM_DEVICE)
    if not isinstance(x, np.ndarray):
        raise Error("ipf: images are numpy arrays or CUDA torch tensors")
    es = x.itemsize
    st = x.strides
    dense_row = (x.ndim == 2 and st[1] == es) or (x.ndim == 3 and st[2] == es and st[1] == c * es)
    if not dense_row or st[0] < w * c * es:
        x = np.ascontiguousarray(x)
        st = x.strides
    return _lib.IpfcImage(x.ctypes.data, w, h, c, _NP_CODE[x.dtype], st[0], MEM_HOST), x


def _new_like(src, code: int):
    if _is_tensor(src):
        torch = _torch()
        tmap = {U8: torch.uint8, U16: torch.uint16, I16: torch.int16, I32: torch.int32,
                F32: torch.float32, F64: torch.float64}
        return torch.empty(tuple(src.shape), dtype=tmap[code], device=src.device)
    return np.empty(src.shape, _CODE_NP[code])


def _stream_of(src, stream):
    if stream is not None:
        return ctypes.c_void_p(stream if isinstance(stream, int) else stream.cuda_stream)
    if _is_tensor(src):
        return ctypes.c_void_p(_torch().cuda.current_stream(src.device).cuda_stream)
    return ctypes.c_void_p(0)


def _check(rc: int) -> None:
    if rc != 0:
        msg = _lib.load().ipfc_last_error().decode() or f"ipf: error {rc}"
        raise Error(msg, rc)


def _pair(src, dtype):
    """Returns (src view, keep-alive source, dst object, dst view)."""
    lib = _lib.load()
    del lib
    if _is_tensor(src):
        sv = _view(src)
        keep = src
    else:
        sv, keep = _view(src)
    dst = _new_like(src, _code_of(dtype, src))
    if _is_tensor(dst):
        dv = _view(dst)
    else:
        dv, dst = _view(dst)
    return sv, keep, dst, dv


def _f64(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())


# ---------------------------------------------------------------------------
# Tap and element generators
# ---------------------------------------------------------------------------

def gaussianKernel1D(sigma: float, ksize: int = 0) -> np.ndarray:
    """gaussianKernel1D (filter.hpp:129-145): normalised FP64 taps."""
    lib = _lib.load()
    buf = np.zeros(1024, np.float64)
    n = lib.ipfc_gaussian_kernel_1d(sigma, ksize, buf.ctypes.data, buf.size)
    if n < 0:
        raise Error(lib.ipfc_last_error().decode())
    if n > buf.size:
        buf = np.zeros(n, np.float64)
        lib.ipfc_gaussian_kernel_1d(sigma, ksize, buf.ctypes.data, buf.size)
    return buf[:n].copy()


def derivKernel(order: int, ksize: int) -> np.ndarray:
    """detail::derivKernel (filter.hpp:93-114)."""
    lib = _lib.load()
    buf = np.zeros(64, np.float64)
    n = lib.ipfc_deriv_kernel(order, ksize, buf.ctypes.data, buf.size)
    if n < 0:
        raise Error(lib.ipfc_last_error().decode())
    return buf[:n].copy()


def getStructuringElement(shape: int, width: int, height: int = 0) -> np.ndarray:
    """getStructuringElement (morphology.hpp:24-49): uint8 mask shaped (h, w)."""
    lib = _lib.load()
    h = height if height > 0 else width
    out = np.zeros((max(h, 0), max(width, 0)), np.uint8)
    _check(lib.ipfc_structuring_element(int(shape), width, height, out.ctypes.data if out.size else None))
    return out


# ---------------------------------------------------------------------------
# Filters
# ---------------------------------------------------------------------------

def sepFilter2D(src, kx, ky, border=BorderMode.Reflect101, delta=0.0, borderValue=0.0, dtype=None, stream=None,
                anchor=(-1, -1)):
    """sepFilter2D (filter.hpp:197-203) over detail::sepFilterImpl (37-90)."""
    lib = _lib.load()
    kx, ky = _f64(kx), _f64(ky)
    sv, keep, dst, dv = _pair(src, dtype)
    _check(lib.ipfc_sep_filter2d(ctypes.byref(sv), ctypes.byref(dv), kx.ctypes.data if kx.size else None, kx.size,
                                 ky.ctypes.data if ky.size else None, ky.size, anchor[0], anchor[1], int(border),
                                 float(delta), float(borderValue), _stream_of(src, stream)))
    del keep
    return dst


def gaussianBlur(src, sigmaX, sigmaY=0.0, ksize=0, border=BorderMode.Reflect101, dtype=None, stream=None):
    """gaussianBlur (filter.hpp:262-267)."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, dtype)
    _check(lib.ipfc_gaussian_blur(ctypes.byref(sv), ctypes.byref(dv), float(sigmaX), float(sigmaY), int(ksize),
                                  int(border), _stream_of(src, stream)))
    del keep
    return dst


def boxFilter(src, kw, kh, normalize=True, border=BorderMode.Reflect101, borderValue=0.0, dtype=None, stream=None):
    """boxFilter (filter.hpp:206-253)."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, dtype)
    _check(lib.ipfc_box_filter(ctypes.byref(sv), ctypes.byref(dv), int(kw), int(kh), int(bool(normalize)),
                               int(border), float(borderValue), _stream_of(src, stream)))
    del keep
    return dst


def blur(src, ksize, border=BorderMode.Reflect101, dtype=None, stream=None):
    """blur (filter.hpp:256-259): normalised ksize x ksize box."""
    return boxFilter(src, ksize, ksize, True, border, 0.0, dtype, stream)


def sobel(src, dx, dy, ksize=3, scale=1.0, border=BorderMode.Reflect101, dtype=np.float32, stream=None):
    """sobel (filter.hpp:395-407).  The reference returns float32; other
    dtypes give sepFilter2D<dtype> with the same taps (e.g. int16)."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, dtype)
    _check(lib.ipfc_sobel(ctypes.byref(sv), ctypes.byref(dv), int(dx), int(dy), int(ksize), float(scale),
                          int(border), _stream_of(src, stream)))
    del keep
    return dst


_F2D_ENTRY = {"auto": "ipfc_filter2d", "fp32": "ipfc_filter2d_fp32", "split": "ipfc_filter2d_split"}


def filter2D(src, kernel, border=BorderMode.Reflect101, delta=0.0, anchor=(-1, -1), borderValue=0.0, dtype=None,
             stream=None, form="auto"):
    """filter2D (filter.hpp:159-194): correlation with float32 taps (kh, kw).

    ``form``: "auto" (the library's choice), "fp32" (CUDA cores, FP32) or
    "split" (tcgen05 tensor cores, FP16 hi + lo operands, FP32 accumulation)."""
    lib = _lib.load()
    entry = getattr(lib, _F2D_ENTRY[form])
    k = np.ascontiguousarray(np.asarray(kernel, dtype=np.float32))
    if k.ndim != 2 or k.size == 0:
        raise Error("ipf: filter2D: kernel must be a non-empty single-channel image")
    sv, keep, dst, dv = _pair(src, dtype)
    _check(entry(ctypes.byref(sv), ctypes.byref(dv), k.ctypes.data, k.shape[1], k.shape[0], int(anchor[0]),
                 int(anchor[1]), int(border), float(delta), float(borderValue), _stream_of(src, stream)))
    del keep
    return dst


def medianBlur(src, ksize, border=BorderMode.Replicate, stream=None):
    """medianBlur (filter.hpp:302-332)."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, None)
    _check(lib.ipfc_median_blur(ctypes.byref(sv), ctypes.byref(dv), int(ksize), int(border),
                                _stream_of(src, stream)))
    del keep
    return dst


def _morph(fn, src, se, iterations, stream):
    lib = _lib.load()
    if se is None:
        se = getStructuringElement(MorphShape.Rect, 3)
    se = np.ascontiguousarray(np.asarray(se, dtype=np.uint8))
    if se.ndim != 2 or se.size == 0:
        raise Error("ipf: morphology: structuring element must be a non-empty single-channel mask")
    sv, keep, dst, dv = _pair(src, None)
    _check(getattr(lib, fn)(ctypes.byref(sv), ctypes.byref(dv), se.ctypes.data, se.shape[1], se.shape[0],
                            int(iterations), _stream_of(src, stream)))
    del keep
    return dst


def erode(src, se=None, iterations=1, stream=None):
    """erode (morphology.hpp:112-118); default element: 3x3 rect."""
    return _morph("ipfc_erode", src, se, iterations, stream)


def dilate(src, se=None, iterations=1, stream=None):
    """dilate (morphology.hpp:121-127); default element: 3x3 rect."""
    return _morph("ipfc_dilate", src, se, iterations, stream)


def morphologyEx(src, op, se=None, iterations=1, stream=None):
    """morphologyEx (morphology.hpp:140-158); default element: 3x3 rect."""
    lib = _lib.load()
    if se is None:
        se = getStructuringElement(MorphShape.Rect, 3)
    se = np.ascontiguousarray(np.asarray(se, dtype=np.uint8))
    if se.ndim != 2 or se.size == 0:
        raise Error("ipf: morphology: structuring element must be a non-empty single-channel mask")
    sv, keep, dst, dv = _pair(src, None)
    _check(lib.ipfc_morphology_ex(ctypes.byref(sv), ctypes.byref(dv), int(op), se.ctypes.data, se.shape[1],
                                  se.shape[0], int(iterations), _stream_of(src, stream)))
    del keep
    return dst


def bilateralFilter(src, d, sigmaColor, sigmaSpace, border=BorderMode.Reflect101, stream=None):
    """bilateralFilter (filter.hpp:337-387)."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, None)
    _check(lib.ipfc_bilateral_filter(ctypes.byref(sv), ctypes.byref(dv), int(d), float(sigmaColor),
                                     float(sigmaSpace), int(border), _stream_of(src, stream)))
    del keep
    return dst


def _alloc(src, shape, code):
    """A destination of `shape` and element code in src's memory space: (obj, view)."""
    if _is_tensor(src):
        torch = _torch()
        tmap = {U8: torch.uint8, U16: torch.uint16, I16: torch.int16, I32: torch.int32,
                F32: torch.float32, F64: torch.float64}
        dst = torch.empty(shape, dtype=tmap[code], device=src.device)
        return dst, _view(dst)
    dst = np.empty(shape, _CODE_NP[code])
    dv, dst = _view(dst)
    return dst, dv


def _source(src):
    if _is_tensor(src):
        return _view(src), src
    return _view(src)


def integralImage(src, squared=False, stream=None):
    """integralImage (filter.hpp:527-541): float64, (H+1) x (W+1) [x C]."""
    lib = _lib.load()
    sv, keep = _source(src)
    w, h, c = _dims(src)
    dst, dv = _alloc(src, (h + 1, w + 1) + ((c,) if src.ndim == 3 else ()), F64)
    _check(lib.ipfc_integral_image(ctypes.byref(sv), ctypes.byref(dv), int(bool(squared)), _stream_of(src, stream)))
    del keep
    return dst


def adaptiveThreshold(src, maxval, method, type, blockSize, C, stream=None):
    """adaptiveThreshold (filter.hpp:554-567), single channel."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, None)
    _check(lib.ipfc_adaptive_threshold(ctypes.byref(sv), ctypes.byref(dv), float(maxval), int(method), int(type),
                                       int(blockSize), float(C), _stream_of(src, stream)))
    del keep
    return dst


def pyrDown(src, stream=None):
    """pyrDown (geometry.hpp:504-513): ((W+1)/2) x ((H+1)/2)."""
    lib = _lib.load()
    sv, keep = _source(src)
    w, h, c = _dims(src)
    dst, dv = _alloc(src, ((h + 1) // 2, (w + 1) // 2) + tuple(src.shape[2:]), sv.dtype)
    _check(lib.ipfc_pyr_down(ctypes.byref(sv), ctypes.byref(dv), _stream_of(src, stream)))
    del keep
    return dst


def _float_result(fn, src, stream, *args):
    lib = _lib.load()
    sv, keep = _source(src)
    dst, dv = _alloc(src, tuple(src.shape), F32)  # ImageF
    _check(getattr(lib, fn)(ctypes.byref(sv), ctypes.byref(dv), *args, _stream_of(src, stream)))
    del keep
    return dst


def scharr(src, dx, dy, scale=1.0, border=BorderMode.Reflect101, stream=None):
    """scharr (filter.hpp:411-414): float32, {-scale, 0, scale} x {3, 10, 3}."""
    if not ((dx, dy) in ((1, 0), (0, 1))):
        raise Error("ipf: scharr: (dx, dy) must be (1,0) or (0,1)")
    d, s = [-scale, 0.0, scale], [3.0, 10.0, 3.0]
    kx, ky = (d, s) if dx else (s, d)
    return sepFilter2D(src, kx, ky, border, dtype=np.float32, stream=stream)


def prewitt(src, dx, dy, border=BorderMode.Reflect101, stream=None):
    """prewitt (filter.hpp:419-422): float32, {-1, 0, 1} x {1, 1, 1}."""
    if not ((dx, dy) in ((1, 0), (0, 1))):
        raise Error("ipf: prewitt: (dx, dy) must be (1,0) or (0,1)")
    d, s = [-1.0, 0.0, 1.0], [1.0, 1.0, 1.0]
    kx, ky = (d, s) if dx else (s, d)
    return sepFilter2D(src, kx, ky, border, dtype=np.float32, stream=stream)


def sharpen(src, strength=1.0, stream=None):
    """sharpen (filter.hpp:487-490): filter2D with {0,-s,0, -s,1+4s,-s, 0,-s,0}, s = float(strength)."""
    s = np.float32(strength)
    k = np.array([[0, -s, 0], [-s, np.float32(1) + np.float32(4) * s, -s], [0, -s, 0]], np.float32)
    return filter2D(src, k, stream=stream)


def emboss(src, stream=None):
    """emboss (filter.hpp:494-496): filter2D with {-2,-1,0, -1,1,1, 0,1,2}."""
    return filter2D(src, np.array([[-2, -1, 0], [-1, 1, 1], [0, 1, 2]], np.float32), stream=stream)


def laplacian(src, ksize=1, scale=1.0, border=BorderMode.Reflect101, stream=None):
    """laplacian (filter.hpp:426-438): float32 result."""
    return _float_result("ipfc_laplacian", src, stream, int(ksize), float(scale), int(border))


def gradientMagnitude(src, ksize=3, stream=None):
    """gradientMagnitude (filter.hpp:462-467): float32 result."""
    return _float_result("ipfc_gradient_magnitude", src, stream, int(ksize))


def unsharpMask(src, sigma=1.0, amount=1.0, threshold=0.0, stream=None):
    """unsharpMask (filter.hpp:473-483): the source's type."""
    lib = _lib.load()
    sv, keep, dst, dv = _pair(src, None)
    _check(lib.ipfc_unsharp_mask(ctypes.byref(sv), ctypes.byref(dv), float(sigma), float(amount), float(threshold),
                                 _stream_of(src, stream)))
    del keep
    return dst


def pyrUp(src, stream=None):
    """pyrUp (geometry.hpp:516-525): 2W x 2H."""
    lib = _lib.load()
    sv, keep = _source(src)
    w, h, c = _dims(src)
    dst, dv = _alloc(src, (2 * h, 2 * w) + tuple(src.shape[2:]), sv.dtype)
    _check(lib.ipfc_pyr_up(ctypes.byref(sv), ctypes.byref(dv), _stream_of(src, stream)))
    del keep
    return dst


def ssim(a, b, ssimMap=False, stream=None):
    """ssim (metrics.hpp:51-78): the mean SSIM, and with ssimMap=True also the
    float32 per-pixel map (the reference's ImageF* out-parameter)."""
    lib = _lib.load()
    av, keep_a = _source(a)
    bv, keep_b = _source(b)
    res = ctypes.c_double(0.0)
    m = mv = None
    if ssimMap:
        m, mv = _alloc(a, tuple(a.shape), F32)
    _check(lib.ipfc_ssim(ctypes.byref(av), ctypes.byref(bv), ctypes.byref(res),
                         ctypes.byref(mv) if ssimMap else None, _stream_of(a, stream)))
    del keep_a, keep_b
    return (res.value, m) if ssimMap else res.value


def _corners(fn, src, args, stream):
    lib = _lib.load()
    sv, keep = _source(src)
    w, h, c = _dims(src)
    dst, dv = _alloc(src, (h, w), F32)
    _check(getattr(lib, fn)(ctypes.byref(sv), ctypes.byref(dv), *args, _stream_of(src, stream)))
    del keep
    return dst


def cornerHarris(src, blockSize=3, ksize=3, k=0.04, stream=None):
    """cornerHarris (features.hpp:128-136): float32 response."""
    return _corners("ipfc_corner_harris", src, (int(blockSize), int(ksize), float(k)), stream)


def cornerMinEigenVal(src, blockSize=3, ksize=3, stream=None):
    """cornerMinEigenVal (features.hpp:138-146): float32 response."""
    return _corners("ipfc_corner_min_eigen_val", src, (int(blockSize), int(ksize)), stream)


def canny(src, lowThreshold, highThreshold, ksize=3, l2Gradient=False, stream=None):
    """canny (features.hpp:27-88): uint8 0/255 edge map, single channel."""
    lib = _lib.load()
    sv, keep = _source(src)
    w, h, c = _dims(src)
    dst, dv = _alloc(src, (h, w), U8)
    _check(lib.ipfc_canny(ctypes.byref(sv), ctypes.byref(dv), float(lowThreshold), float(highThreshold), int(ksize),
                          int(bool(l2Gradient)), _stream_of(src, stream)))
    del keep
    return dst
