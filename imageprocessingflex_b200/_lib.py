"""ctypes binding of ``libipfcuda.so`` (the C ABI declared in include/ipfc.h).

The library is built in-tree by ``imageprocessingflex_b200.build``.  Loading
fails loudly (``ImportError``) when it is missing and cannot be built: there is
no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

c_int, c_double, c_void_p, c_longlong = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong


class IpfcImage(ctypes.Structure):
    """Mirror of ``struct ipfc_image``."""

    _fields_ = [
        ("data", c_void_p),
        ("width", c_int),
        ("height", c_int),
        ("channels", c_int),
        ("dtype", c_int),
        ("pitch", c_longlong),
        ("mem", c_int),
    ]


class IpfcRequest(ctypes.Structure):
    """Mirror of ``struct ipfc_request``."""

    _fields_ = [
        ("op", c_int), ("src", IpfcImage), ("dst", IpfcImage), ("sigma_x", c_double), ("sigma_y", c_double),
        ("ksize", c_int), ("dx", c_int), ("dy", c_int), ("scale", c_double), ("kernel", c_void_p), ("kw", c_int),
        ("kh", c_int), ("border", c_int), ("delta", c_double), ("border_value", c_double), ("arrival", c_double),
    ]


class IpfcCompletion(ctypes.Structure):
    """Mirror of ``struct ipfc_completion``."""

    _fields_ = [("ticket", ctypes.c_ulonglong), ("status", c_int), ("arrival", c_double), ("admitted", c_double),
                ("done", c_double)]


class IpfcServerConfig(ctypes.Structure):
    """Mirror of ``struct ipfc_server_config``."""

    _fields_ = [("device_budget_bytes", ctypes.c_size_t), ("max_inflight", c_int), ("streams", c_int),
                ("batch", c_int)]


IMG_P = ctypes.POINTER(IpfcImage)
DBL_P = ctypes.POINTER(c_double)

# name -> (restype, argtypes)
_SIGNATURES = {
    "ipfc_last_error": (ctypes.c_char_p, []),
    "ipfc_version": (c_int, []),
    "ipfc_check_device": (c_int, [c_void_p]),
    "ipfc_set_wait_limit_ns": (ctypes.c_ulonglong, [ctypes.c_ulonglong]),
    "ipfc_gaussian_kernel_1d": (c_int, [c_double, c_int, c_void_p, c_int]),
    "ipfc_deriv_kernel": (c_int, [c_int, c_int, c_void_p, c_int]),
    "ipfc_structuring_element": (c_int, [c_int, c_int, c_int, c_void_p]),
    "ipfc_sep_filter2d": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_int, c_double,
                                  c_double, c_void_p]),
    "ipfc_gaussian_blur": (c_int, [IMG_P, IMG_P, c_double, c_double, c_int, c_int, c_void_p]),
    "ipfc_box_filter": (c_int, [IMG_P, IMG_P, c_int, c_int, c_int, c_int, c_double, c_void_p]),
    "ipfc_sobel": (c_int, [IMG_P, IMG_P, c_int, c_int, c_int, c_double, c_int, c_void_p]),
    "ipfc_filter2d": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_double,
                              c_void_p]),
    "ipfc_filter2d_fp32": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_double,
                                   c_void_p]),
    "ipfc_filter2d_split": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_int, c_int, c_double, c_double,
                                    c_void_p]),
    "ipfc_filter2d_noalloc": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_int, c_int, c_double,
                                      c_double, c_void_p]),
    "ipfc_median_blur": (c_int, [IMG_P, IMG_P, c_int, c_int, c_void_p]),
    "ipfc_morphology_ex": (c_int, [IMG_P, IMG_P, c_int, c_void_p, c_int, c_int, c_int, c_void_p]),
    "ipfc_bilateral_filter": (c_int, [IMG_P, IMG_P, c_int, c_double, c_double, c_int, c_void_p]),
    "ipfc_integral_image": (c_int, [IMG_P, IMG_P, c_int, c_void_p]),
    "ipfc_adaptive_threshold": (c_int, [IMG_P, IMG_P, c_double, c_int, c_int, c_int, c_double, c_void_p]),
    "ipfc_pyr_down": (c_int, [IMG_P, IMG_P, c_void_p]),
    "ipfc_pyr_up": (c_int, [IMG_P, IMG_P, c_void_p]),
    "ipfc_ssim": (c_int, [IMG_P, IMG_P, DBL_P, IMG_P, c_void_p]),
    "ipfc_corner_harris": (c_int, [IMG_P, IMG_P, c_int, c_int, c_double, c_void_p]),
    "ipfc_corner_min_eigen_val": (c_int, [IMG_P, IMG_P, c_int, c_int, c_void_p]),
    "ipfc_canny": (c_int, [IMG_P, IMG_P, c_double, c_double, c_int, c_int, c_void_p]),
    "ipfc_laplacian": (c_int, [IMG_P, IMG_P, c_int, c_double, c_int, c_void_p]),
    "ipfc_gradient_magnitude": (c_int, [IMG_P, IMG_P, c_int, c_void_p]),
    "ipfc_unsharp_mask": (c_int, [IMG_P, IMG_P, c_double, c_double, c_double, c_void_p]),
    "ipfc_erode": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_void_p]),
    "ipfc_dilate": (c_int, [IMG_P, IMG_P, c_void_p, c_int, c_int, c_int, c_void_p]),
    "ipfc_batch_create": (c_int, [c_void_p]),
    "ipfc_batch_destroy": (c_int, [c_void_p]),
    "ipfc_batch_set_option": (c_int, [c_void_p, c_int, c_int]),
    "ipfc_batch_add_sep_filter": (c_int, [c_void_p, IMG_P, IMG_P, c_void_p, c_int, c_void_p, c_int, c_int, c_double,
                                          c_double]),
    "ipfc_batch_add_gaussian_blur": (c_int, [c_void_p, IMG_P, IMG_P, c_double, c_double, c_int, c_int]),
    "ipfc_batch_add_median_blur": (c_int, [c_void_p, IMG_P, IMG_P, c_int, c_int]),
    "ipfc_batch_add_erode": (c_int, [c_void_p, IMG_P, IMG_P, c_void_p, c_int, c_int, c_int]),
    "ipfc_batch_add_dilate": (c_int, [c_void_p, IMG_P, IMG_P, c_void_p, c_int, c_int, c_int]),
    "ipfc_batch_run": (c_int, [c_void_p, c_void_p]),
    "ipfc_batch_info": (c_int, [c_void_p, c_int, c_void_p]),
    "ipfc_tune_get": (c_int, [c_int, c_int, c_int, c_int, c_void_p, c_void_p]),
    "ipfc_tune_set": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int]),
    "ipfc_tune_save": (c_int, [ctypes.c_char_p]),
    "ipfc_tune_load": (c_int, [ctypes.c_char_p, c_void_p]),
    "ipfc_tune_clear": (c_int, []),
    "ipfc_server_create": (c_int, [c_void_p, ctypes.POINTER(IpfcServerConfig)]),
    "ipfc_server_destroy": (c_int, [c_void_p]),
    "ipfc_server_now": (c_double, [c_void_p]),
    "ipfc_server_submit": (c_int, [c_void_p, ctypes.POINTER(IpfcRequest), c_void_p]),
    "ipfc_server_poll": (c_int, [c_void_p, ctypes.POINTER(IpfcCompletion), c_int, c_void_p, c_int]),
    "ipfc_server_drain": (c_int, [c_void_p, c_int]),
    "ipfc_server_stats": (c_int, [c_void_p, c_int, c_void_p]),
    "ipfc_server_fail_allocation": (c_int, [c_void_p, c_longlong]),
    "ipfc_probe_border_index": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p]),
    "ipfc_probe_saturate": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p]),
}

_lib = None


def library_path() -> str:
    return _build.LIBPATH


def load() -> ctypes.CDLL:
    """Loads (building first if needed) and returns the CUDA library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIBPATH
    if not os.path.exists(path) or os.environ.get("IPFC_REBUILD") == "1":
        try:
            _build.build()
        except Exception as exc:  # toolchain missing or compile error
            raise ImportError(f"libipfcuda.so is missing and could not be built: {exc}") from exc
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_names():
    return list(_SIGNATURES)
