"""Batches: many device images through a few launches (ipfc_batch_*).

A ``Batch`` collects per-image calls -- ``add_gaussianBlur``,
``add_sepFilter2D``, ``add_medianBlur``, ``add_erode``, ``add_dilate``, with
the arguments of the functions of the same name -- on CUDA uint8 tensors and
runs them together.  The first ``run`` plans the batch (autotuned tile shapes,
longest tiles first) and captures it as a CUDA graph; later runs replay the
graph.  Every image's result is bit-identical to its per-image call.

The batch keeps references to its tensors: their storage must not move
while the batch exists.  New pixels are processed by writing them into the
same tensors and calling ``run`` again.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .filters import BorderMode, Error, _check, _f64, _is_tensor, _stream_of, _view, getStructuringElement

AUTOTUNE, GRAPH = 1, 2
INFO = {"items": 0, "planned": 1, "tiles_light": 2, "tiles_heavy": 3, "grid_light": 4, "grid_heavy": 5,
        "kernels": 6, "graph": 7, "tiles_mem": 8, "grid_mem": 9}
OP_SEP, OP_MEDIAN, OP_MORPH = 0, 1, 2


class Batch:
    """An ``ipfc_batch``: add images and ops, then ``run``."""

    def __init__(self, autotune: bool = True, graph: bool = True):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _check(self._lib.ipfc_batch_create(ctypes.byref(h)))
        self._h = h
        self._keep = []
        _check(self._lib.ipfc_batch_set_option(self._h, AUTOTUNE, int(bool(autotune))))
        _check(self._lib.ipfc_batch_set_option(self._h, GRAPH, int(bool(graph))))

    def close(self) -> None:
        if self._h:
            self._lib.ipfc_batch_destroy(self._h)
            self._h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _views(self, src, dst):
        if not (_is_tensor(src) and _is_tensor(dst)):
            raise Error("ipf: batch: images must be CUDA torch tensors")
        sv, dv = _view(src), _view(dst)
        self._keep += [src, dst]
        return sv, dv

    def add_sepFilter2D(self, src, dst, kx, ky, border=BorderMode.Reflect101, delta=0.0, borderValue=0.0):
        kx, ky = _f64(kx), _f64(ky)
        sv, dv = self._views(src, dst)
        _check(self._lib.ipfc_batch_add_sep_filter(self._h, ctypes.byref(sv), ctypes.byref(dv), kx.ctypes.data,
                                                   kx.size, ky.ctypes.data, ky.size, int(border), float(delta),
                                                   float(borderValue)))

    def add_gaussianBlur(self, src, dst, sigmaX, sigmaY=0.0, ksize=0, border=BorderMode.Reflect101):
        sv, dv = self._views(src, dst)
        _check(self._lib.ipfc_batch_add_gaussian_blur(self._h, ctypes.byref(sv), ctypes.byref(dv), float(sigmaX),
                                                      float(sigmaY), int(ksize), int(border)))

    def add_medianBlur(self, src, dst, ksize, border=BorderMode.Replicate):
        sv, dv = self._views(src, dst)
        _check(self._lib.ipfc_batch_add_median_blur(self._h, ctypes.byref(sv), ctypes.byref(dv), int(ksize),
                                                    int(border)))

    def _morph(self, fn, src, dst, se, iterations):
        se = getStructuringElement(0, 3) if se is None else np.ascontiguousarray(np.asarray(se, np.uint8))
        sv, dv = self._views(src, dst)
        _check(getattr(self._lib, fn)(self._h, ctypes.byref(sv), ctypes.byref(dv), se.ctypes.data, se.shape[1],
                                      se.shape[0], int(iterations)))

    def add_erode(self, src, dst, se=None, iterations=1):
        self._morph("ipfc_batch_add_erode", src, dst, se, iterations)

    def add_dilate(self, src, dst, se=None, iterations=1):
        self._morph("ipfc_batch_add_dilate", src, dst, se, iterations)

    def run(self, stream=None) -> None:
        """Runs every item (asynchronous on `stream`, default torch's current stream)."""
        like = self._keep[0] if self._keep else None
        _check(self._lib.ipfc_batch_run(self._h, _stream_of(like, stream) if like is not None else None))

    def info(self, what: str) -> int:
        v = ctypes.c_longlong()
        _check(self._lib.ipfc_batch_info(self._h, INFO[what], ctypes.byref(v)))
        return v.value


def tune_get(op: int, k: int, channels: int, size_class: int):
    """The autotuner's (a, b) for a key, or None."""
    lib = _lib.load()
    a, b = ctypes.c_int(), ctypes.c_int()
    if lib.ipfc_tune_get(op, k, channels, size_class, ctypes.byref(a), ctypes.byref(b)) != 0:
        return None
    return a.value, b.value


def tune_set(op: int, k: int, channels: int, size_class: int, a: int, b: int = 0) -> None:
    _check(_lib.load().ipfc_tune_set(op, k, channels, size_class, a, b))


def tune_save(path: str) -> None:
    _check(_lib.load().ipfc_tune_save(path.encode()))


def tune_load(path: str) -> int:
    n = ctypes.c_int()
    _check(_lib.load().ipfc_tune_load(path.encode(), ctypes.byref(n)))
    return n.value


def tune_clear() -> None:
    _check(_lib.load().ipfc_tune_clear())
