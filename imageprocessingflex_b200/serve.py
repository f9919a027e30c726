"""The request server (ipfc_server_*): continuous batching of filter requests.

``Server`` wraps one ``ipfc_server``.  ``submit`` queues a request -- an op
name, a source and destination image (numpy arrays or pinned CPU torch
tensors for host images, CUDA tensors for device images) and the op's
parameters -- with an arrival time on the server's clock; the server's
scheduler thread admits requests against its slot and device-memory budget,
overlaps them over several streams and merges those the batch kernels cover
into one batch plan for each group of requests admitted together.  ``poll``
returns completions with their arrival, admission and completion times.  The
caller keeps every image alive and unchanged until its request completes.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .filters import BorderMode, Error, _check, _dims, _is_tensor, _torch_code, _NP_CODE

OPS = {"gaussian": 0, "sobel": 1, "median": 2, "filter2d": 3, "box": 4, "erode": 5, "dilate": 6}
STATS = {"groups": 0, "batched": 1, "batch_launches": 2, "max_inflight": 3, "max_bytes": 4, "failed": 5}


@dataclass
class Completion:
    ticket: int
    status: int
    arrival: float
    admitted: float
    done: float

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def image_view(x) -> _lib.IpfcImage:
    """ipfc_image of a numpy array or a torch tensor (CPU tensors: host memory)."""
    w, h, c = _dims(x)
    if _is_tensor(x):
        es = x.element_size()
        if not x.is_contiguous():
            raise Error("ipf: server: images must be contiguous")
        return _lib.IpfcImage(x.data_ptr(), w, h, c, _torch_code(x), w * c * es, 1 if x.is_cuda else 0)
    if not (isinstance(x, np.ndarray) and x.flags.c_contiguous):
        raise Error("ipf: server: images must be contiguous numpy arrays or torch tensors")
    return _lib.IpfcImage(x.ctypes.data, w, h, c, _NP_CODE[x.dtype], w * c * x.itemsize, 0)


class Server:
    def __init__(self, budget_bytes: int = 40 << 30, max_inflight: int = 64, streams: int = 4, batch: bool = True):
        self._lib = _lib.load()
        cfg = _lib.IpfcServerConfig(budget_bytes, max_inflight, streams, int(bool(batch)))
        h = ctypes.c_void_p()
        _check(self._lib.ipfc_server_create(ctypes.byref(h), ctypes.byref(cfg)))
        self._h = h
        self._keep = {}

    def close(self) -> None:
        if self._h:
            self._lib.ipfc_server_destroy(self._h)
            self._h = None
            self._keep = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def now(self) -> float:
        return self._lib.ipfc_server_now(self._h)

    def submit(self, op: str, src, dst, arrival: float = -1.0, *, sigma_x=0.0, sigma_y=0.0, ksize=0, dx=0, dy=0,
               scale=1.0, kernel=None, border=None, delta=0.0, border_value=0.0, keep=True) -> int:
        r = _lib.IpfcRequest()
        r.op = OPS[op]
        r.src = image_view(src)
        r.dst = image_view(dst)
        r.sigma_x, r.sigma_y, r.ksize, r.dx, r.dy, r.scale = float(sigma_x), float(sigma_y), int(ksize), int(dx), int(
            dy), float(scale)
        if border is None:
            border = BorderMode.Replicate if op == "median" else BorderMode.Reflect101
        r.border = int(border)
        r.delta, r.border_value, r.arrival = float(delta), float(border_value), float(arrival)
        k = None
        if kernel is not None:
            k = np.ascontiguousarray(np.asarray(kernel, np.float32))
            r.kernel, r.kw, r.kh = k.ctypes.data, k.shape[1], k.shape[0]
        t = ctypes.c_ulonglong()
        _check(self._lib.ipfc_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        if keep:
            self._keep[t.value] = (src, dst)
        return t.value

    def poll(self, max_n: int = 4096, wait_ms: int = 0):
        buf = (_lib.IpfcCompletion * max_n)()
        n = ctypes.c_int()
        _check(self._lib.ipfc_server_poll(self._h, buf, max_n, ctypes.byref(n), int(wait_ms)))
        out = []
        for i in range(n.value):
            c = buf[i]
            self._keep.pop(c.ticket, None)
            out.append(Completion(c.ticket, c.status, c.arrival, c.admitted, c.done))
        return out

    def drain(self, timeout_ms: int = -1) -> None:
        _check(self._lib.ipfc_server_drain(self._h, int(timeout_ms)))

    def fail_allocation(self, nth: int) -> None:
        """Failure injection: the nth device-buffer allocation the server makes
        for a request fails as out of memory (0 disables)."""
        _check(self._lib.ipfc_server_fail_allocation(self._h, int(nth)))

    def stats(self) -> dict:
        out = {}
        for name, code in STATS.items():
            v = ctypes.c_double()
            _check(self._lib.ipfc_server_stats(self._h, code, ctypes.byref(v)))
            out[name] = v.value
        return out
