"""CPU checkers for the neighbourhood-filter path (TEST INFRASTRUCTURE ONLY).

Two libraries with one interface:

* ``restatement()`` -- ``oracle/_build/liboracle.so``, the C restatement of the
  reference algorithms (``oracle/oracle.c``).  Always buildable from this
  repository.
* ``reference()`` -- ``oracle/_ref/libipfref.so``, the reference's own headers
  (``include/ipf/filter.hpp``, ``include/ipf/morphology.hpp``) behind a C shim.
  Built only where the reference checkout is present; ``None`` elsewhere.

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The product library never does.

Images are numpy arrays shaped (H, W) or (H, W, C), interleaved like
``ipf::Image<T>``.  Border codes follow ``ipf::BorderMode`` order:
0 Constant, 1 Replicate, 2 Reflect, 3 Reflect101, 4 Wrap.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
_REF_SO = os.path.join(HERE, "_ref", "libipfref.so")

DTYPE_CODE = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.int16): 2,
              np.dtype(np.int32): 3, np.dtype(np.float32): 4, np.dtype(np.float64): 5}

CONSTANT, REPLICATE, REFLECT, REFLECT101, WRAP = range(5)
BORDERS = (CONSTANT, REPLICATE, REFLECT, REFLECT101, WRAP)

_c_void_p, _c_int, _c_double = ctypes.c_void_p, ctypes.c_int, ctypes.c_double


def build(force: bool = False) -> None:
    """Builds both checker libraries with oracle/Makefile (the _ref one only
    where the reference checkout exists)."""
    if force or not os.path.exists(_ORACLE_SO) or not os.path.exists(_REF_SO):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True, stdout=subprocess.DEVNULL)


def _shape(a: np.ndarray):
    if a.ndim == 2:
        return a.shape[1], a.shape[0], 1
    if a.ndim == 3:
        return a.shape[1], a.shape[0], a.shape[2]
    raise ValueError("image must be (H, W) or (H, W, C)")


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_c_void_p)


class CpuFilters:
    """ctypes view of one checker library; ``prefix`` is ``orc`` or ``ref``."""

    def __init__(self, path: str, prefix: str):
        self.path = path
        self.prefix = prefix
        self.lib = ctypes.CDLL(path)
        self._f = lambda name: getattr(self.lib, f"{prefix}_{name}")

    # -- tap generators -----------------------------------------------------
    def gaussian_kernel_1d(self, sigma: float, ksize: int = 0) -> np.ndarray:
        buf = np.zeros(4096, np.float64)
        f = self._f("gaussian_kernel_1d")
        f.restype = _c_int
        n = f(_c_double(sigma), _c_int(ksize), _ptr(buf), _c_int(buf.size))
        if n < 0:
            raise ValueError("ipf: gaussianKernel1D: invalid arguments")
        return buf[:n].copy()

    def deriv_kernel(self, order: int, ksize: int) -> np.ndarray:
        buf = np.zeros(64, np.float64)
        f = self._f("deriv_kernel")
        f.restype = _c_int
        n = f(_c_int(order), _c_int(ksize), _ptr(buf), _c_int(buf.size))
        if n < 0:
            raise ValueError("ipf: derivKernel: invalid arguments")
        return buf[:n].copy()

    def structuring_element(self, shape: int, w: int, h: int = 0) -> np.ndarray:
        hh = h if h > 0 else w
        out = np.zeros((hh, w), np.uint8)
        rc = self._f("structuring_element")(_c_int(shape), _c_int(w), _c_int(h), _ptr(out))
        if rc:
            raise ValueError("ipf: getStructuringElement: size must be positive")
        return out

    # -- filters ------------------------------------------------------------
    def _out(self, src, out_dtype):
        return np.zeros(src.shape, np.dtype(out_dtype) if out_dtype is not None else src.dtype)

    def sep_filter(self, src, kx, ky, ax=-1, ay=-1, border=REFLECT101, delta=0.0, border_value=0.0, out_dtype=None):
        src = np.ascontiguousarray(src)
        kx = np.ascontiguousarray(kx, np.float64)
        ky = np.ascontiguousarray(ky, np.float64)
        ax = len(kx) // 2 if ax < 0 else ax
        ay = len(ky) // 2 if ay < 0 else ay
        out = self._out(src, out_dtype)
        W, H, C = _shape(src)
        rc = self._f("sep_filter")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), DTYPE_CODE[out.dtype],
                                   _ptr(kx), len(kx), _ptr(ky), len(ky), ax, ay, border, _c_double(delta),
                                   _c_double(border_value))
        if rc:
            raise ValueError(f"ipf: separable filter failed ({rc})")
        return out

    def gaussian_blur(self, src, sigma_x, sigma_y=0.0, ksize=0, border=REFLECT101, out_dtype=None):
        if sigma_y <= 0:
            sigma_y = sigma_x
        kx = self.gaussian_kernel_1d(sigma_x, ksize)
        ky = self.gaussian_kernel_1d(sigma_y, ksize)
        return self.sep_filter(src, kx, ky, border=border, out_dtype=out_dtype)

    def sobel_taps(self, dx, dy, ksize=3, scale=1.0):
        kx = self.deriv_kernel(dx, ksize)
        ky = self.deriv_kernel(dy, ksize)
        if ksize == 1:
            if kx.size == 1:
                kx = np.array([0.0, 1.0, 0.0])
            if ky.size == 1:
                ky = np.array([0.0, 1.0, 0.0])
        return kx * scale, ky

    def sobel(self, src, dx, dy, ksize=3, scale=1.0, border=REFLECT101, out_dtype=np.float32):
        kx, ky = self.sobel_taps(dx, dy, ksize, scale)
        return self.sep_filter(src, kx, ky, border=border, out_dtype=out_dtype)

    def filter2d(self, src, kernel, border=REFLECT101, delta=0.0, anchor=(-1, -1), border_value=0.0, out_dtype=None):
        src = np.ascontiguousarray(src)
        k = np.ascontiguousarray(kernel, np.float32)
        kh, kw = k.shape
        out = self._out(src, out_dtype)
        W, H, C = _shape(src)
        rc = self._f("filter2d")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), DTYPE_CODE[out.dtype],
                                 _ptr(k), kw, kh, anchor[0], anchor[1], border, _c_double(delta),
                                 _c_double(border_value))
        if rc:
            raise ValueError(f"ipf: filter2D failed ({rc})")
        return out

    def filter2d_rows(self, src, kernel, y0, y1, border=REFLECT101, delta=0.0, anchor=(-1, -1), border_value=0.0,
                      out_dtype=None, threads=0):
        """Output rows [y0, y1) of filter2D over the whole image (restatement
        only), computed by ``threads`` host threads (0: all cores) on
        sub-bands; the C routine runs without the GIL."""
        import concurrent.futures as cf

        src = np.ascontiguousarray(src)
        k = np.ascontiguousarray(kernel, np.float32)
        kh, kw = k.shape
        W, H, C = _shape(src)
        y0, y1 = max(0, y0), min(H, y1)
        shape = (y1 - y0,) + src.shape[1:]
        out = np.zeros(shape, np.dtype(out_dtype) if out_dtype is not None else src.dtype)
        f = self._f("filter2d_rows")
        nt = threads or os.cpu_count() or 1
        step = max(1, -(-(y1 - y0) // nt))
        row_bytes = out[0].nbytes if out.shape[0] else 0

        def band(a):
            b = min(y1, a + step)
            dst = ctypes.c_void_p(out.ctypes.data + (a - y0) * row_bytes)
            return f(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, dst, DTYPE_CODE[out.dtype], _ptr(k), kw, kh,
                     anchor[0], anchor[1], border, _c_double(delta), _c_double(border_value), a, b)

        with cf.ThreadPoolExecutor(nt) as ex:
            rcs = list(ex.map(band, range(y0, y1, step)))
        if any(rcs):
            raise ValueError(f"ipf: filter2D failed ({rcs})")
        return out

    # -- the reference's other filters and callers of the filters -------------
    def morphology_ex(self, src, op, se, iterations=1):
        src = np.ascontiguousarray(src)
        se = np.ascontiguousarray(se, np.uint8)
        out = np.zeros_like(src)
        W, H, C = _shape(src)
        rc = self._f("morphology_ex")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), op, _ptr(se),
                                      se.shape[1], se.shape[0], iterations)
        if rc:
            raise ValueError(f"ipf: morphologyEx failed ({rc})")
        return out

    def bilateral(self, src, d, sigma_color, sigma_space, border=REFLECT101):
        src = np.ascontiguousarray(src)
        out = np.zeros_like(src)
        W, H, C = _shape(src)
        rc = self._f("bilateral")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), d, _c_double(sigma_color),
                                  _c_double(sigma_space), border)
        if rc:
            raise ValueError(f"ipf: bilateralFilter failed ({rc})")
        return out

    def integral(self, src, squared=False):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros((H + 1, W + 1) + ((C,) if src.ndim == 3 else ()), np.float64)
        rc = self._f("integral")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), int(bool(squared)))
        if rc:
            raise ValueError(f"ipf: integralImage failed ({rc})")
        return out

    def adaptive_threshold(self, src, maxval, method, ttype, block_size, c):
        src = np.ascontiguousarray(src)
        out = np.zeros_like(src)
        W, H, _ = _shape(src)
        rc = self._f("adaptive_threshold")(_ptr(src), DTYPE_CODE[src.dtype], W, H, _ptr(out), _c_double(maxval),
                                           method, ttype, block_size, _c_double(c))
        if rc:
            raise ValueError(f"ipf: adaptiveThreshold failed ({rc})")
        return out

    def pyr_down(self, src):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros(((H + 1) // 2, (W + 1) // 2) + src.shape[2:], src.dtype)
        if self._f("pyr_down")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out)):
            raise ValueError("ipf: pyrDown failed")
        return out

    def pyr_up(self, src):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros((2 * H, 2 * W) + src.shape[2:], src.dtype)
        if self._f("pyr_up")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out)):
            raise ValueError("ipf: pyrUp failed")
        return out

    def ssim(self, a, b, want_map=False):
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        W, H, C = _shape(a)
        res = np.zeros(1, np.float64)
        m = np.zeros(a.shape, np.float32) if want_map else None
        rc = self._f("ssim")(_ptr(a), _ptr(b), DTYPE_CODE[a.dtype], W, H, C, _ptr(res),
                             _ptr(m) if want_map else None)
        if rc:
            raise ValueError(f"ipf: ssim failed ({rc})")
        return (float(res[0]), m) if want_map else float(res[0])

    def corner(self, src, block_size=3, ksize=3, k=0.04, min_eig=False):
        src = np.ascontiguousarray(src)
        W, H, _ = _shape(src)
        out = np.zeros((H, W), np.float32)
        rc = self._f("corner")(_ptr(src), DTYPE_CODE[src.dtype], W, H, _ptr(out), block_size, ksize, _c_double(k),
                               int(bool(min_eig)))
        if rc:
            raise ValueError(f"ipf: corner response failed ({rc})")
        return out

    def canny(self, src, low, high, ksize=3, l2=False):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros((H, W), np.uint8)
        rc = self._f("canny")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), _c_double(low),
                              _c_double(high), ksize, int(bool(l2)))
        if rc:
            raise ValueError(f"ipf: canny failed ({rc})")
        return out

    def laplacian(self, src, ksize=1, scale=1.0, border=REFLECT101):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros(src.shape, np.float32)
        if self._f("laplacian")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), ksize, _c_double(scale), border):
            raise ValueError("ipf: laplacian failed")
        return out

    def gradient_magnitude(self, src, ksize=3):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros(src.shape, np.float32)
        if self._f("gradient_magnitude")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), ksize):
            raise ValueError("ipf: gradientMagnitude failed")
        return out

    def unsharp_mask(self, src, sigma=1.0, amount=1.0, threshold=0.0):
        src = np.ascontiguousarray(src)
        W, H, C = _shape(src)
        out = np.zeros_like(src)
        if self._f("unsharp_mask")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), _c_double(sigma),
                                   _c_double(amount), _c_double(threshold)):
            raise ValueError("ipf: unsharpMask failed")
        return out

    def box_filter(self, src, kw, kh, normalize=True, border=REFLECT101, border_value=0.0, out_dtype=None):
        src = np.ascontiguousarray(src)
        out = self._out(src, out_dtype)
        W, H, C = _shape(src)
        rc = self._f("box_filter")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), DTYPE_CODE[out.dtype],
                                   kw, kh, int(bool(normalize)), border, _c_double(border_value))
        if rc:
            raise ValueError(f"ipf: boxFilter failed ({rc})")
        return out

    def median_blur(self, src, ksize, border=REPLICATE):
        src = np.ascontiguousarray(src)
        out = np.zeros_like(src)
        W, H, C = _shape(src)
        rc = self._f("median_blur")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), ksize, border)
        if rc:
            raise ValueError(f"ipf: medianBlur failed ({rc})")
        return out

    def morph(self, src, se, erode=True, iterations=1):
        src = np.ascontiguousarray(src)
        se = np.ascontiguousarray(se, np.uint8)
        out = np.zeros_like(src)
        W, H, C = _shape(src)
        rc = self._f("morph")(_ptr(src), DTYPE_CODE[src.dtype], W, H, C, _ptr(out), _ptr(se), se.shape[1],
                              se.shape[0], int(bool(erode)), iterations)
        if rc:
            raise ValueError(f"ipf: morphology failed ({rc})")
        return out

    def erode(self, src, se, iterations=1):
        return self.morph(src, se, True, iterations)

    def dilate(self, src, se, iterations=1):
        return self.morph(src, se, False, iterations)


_cache: dict = {}


def restatement() -> CpuFilters:
    """The C restatement (builds it on first use if needed)."""
    if "orc" not in _cache:
        if not os.path.exists(_ORACLE_SO):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)
        _cache["orc"] = CpuFilters(_ORACLE_SO, "orc")
    return _cache["orc"]


def reference():
    """The reference's compiled headers, or None where they were not built."""
    if "ref" not in _cache:
        _cache["ref"] = CpuFilters(_REF_SO, "ref") if os.path.exists(_REF_SO) else None
    return _cache["ref"]


def random_image(w: int, h: int, c: int, dtype, seed: int = 1) -> np.ndarray:
    """Seeded image with the sample stream of the reference's randomImage()
    (std::mt19937, one draw per sample in memory order)."""
    dt = np.dtype(dtype)
    out = np.zeros((h, w, c), dt)
    f = restatement().lib.orc_random_image
    f.argtypes = [_c_void_p, _c_int, ctypes.c_size_t, ctypes.c_uint]
    if f(_ptr(out), DTYPE_CODE[dt], out.size, seed):
        raise ValueError("unsupported dtype")
    return out


def set_reference_threads(n: int) -> None:
    lib = reference()
    if lib is not None:
        lib.lib.ref_set_threads(_c_int(n))


def reference_threads() -> int:
    lib = reference()
    return int(lib.lib.ref_get_threads()) if lib is not None else 0
