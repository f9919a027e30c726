"""Seeded synthetic workloads of the batched and served forms.

``served_stream`` is the served configuration: requests with Poisson
arrivals at `rate` per second; image area lognormal with median 1 MP and
log-sd `area_sigma` (1.0 unless stated), clipped to [0.01, 33] MP; aspect
ratio uniform in [0.5, 2]; 1 or 3 channels; uint8 pixels.  Op mix:
gaussianBlur 45 % (sigma uniform in [0.5, 4]), sobel 20 % (ksize 3, dx=1 or
dy=1, float output), medianBlur 5x5 15 %, filter2D 15x15 20 % (one seeded
N(0,1) kernel normalised to sum 1, uint8 output).

``uneven_mix`` is the batched configuration: images with width and height
uniform in [lo, hi], channels from {1, 3, 4}, uint8 pixels uniform 0-255, and
one op each -- gaussianBlur with sigma uniform in [0.5, 4] (50 %), medianBlur
3x3 or 5x5 (25 %), erode or dilate with a 3x3 rect (25 %).  The generator is
numpy's PCG64 seeded by the caller, so a seed names one fixed mix.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class MixItem:
    width: int
    height: int
    channels: int
    op: str        # "gaussian", "median", "erode", "dilate"
    sigma: float = 0.0
    ksize: int = 0
    seed: int = 0  # pixel seed

    @property
    def pixels(self) -> int:
        return self.width * self.height


def uneven_mix(n: int = 512, seed: int = 2024, lo: int = 64, hi: int = 2048):
    rng = np.random.default_rng(seed)
    items = []
    for i in range(n):
        w, h = (int(v) for v in rng.integers(lo, hi + 1, size=2))
        c = int(rng.choice([1, 3, 4]))
        u = rng.random()
        if u < 0.5:
            items.append(MixItem(w, h, c, "gaussian", sigma=float(rng.uniform(0.5, 4.0)), seed=i))
        elif u < 0.75:
            items.append(MixItem(w, h, c, "median", ksize=int(rng.choice([3, 5])), seed=i))
        else:
            items.append(MixItem(w, h, c, "erode" if rng.random() < 0.5 else "dilate", ksize=3, seed=i))
    return items


@dataclass
class Request:
    arrival: float
    width: int
    height: int
    channels: int
    op: str  # "gaussian", "sobel", "median", "filter2d"
    sigma: float = 0.0
    dx: int = 0
    dy: int = 0

    @property
    def pixels(self) -> int:
        return self.width * self.height


def served_stream(n: int = 20000, rate: float = 3000.0, seed: int = 77, area_sigma: float = 1.0):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    area = np.clip(np.exp(np.log(1e6) + area_sigma * rng.standard_normal(n)), 1e4, 33e6)
    aspect = rng.uniform(0.5, 2.0, size=n)
    out = []
    for i in range(n):
        w = max(1, int(round(np.sqrt(area[i] * aspect[i]))))
        h = max(1, int(round(area[i] / w)))
        c = int(rng.choice([1, 3]))
        u = rng.random()
        if u < 0.45:
            out.append(Request(float(t[i]), w, h, c, "gaussian", sigma=float(rng.uniform(0.5, 4.0))))
        elif u < 0.65:
            dx = int(rng.random() < 0.5)
            out.append(Request(float(t[i]), w, h, c, "sobel", dx=dx, dy=1 - dx))
        elif u < 0.80:
            out.append(Request(float(t[i]), w, h, c, "median"))
        else:
            out.append(Request(float(t[i]), w, h, c, "filter2d"))
    return out


def filter2d_taps(k: int = 15, seed: int = 15) -> np.ndarray:
    """Seeded dense k x k taps drawn N(0,1) and normalised to sum 1 (float32)."""
    rng = np.random.default_rng(seed)
    while True:
        w = rng.standard_normal((k, k))
        if abs(w.sum()) > 0.25 * k:  # keep the normalisation away from a near-zero sum
            return (w / w.sum()).astype(np.float32)


def fill_uniform_u8(t, seed: int) -> None:
    """Fills a CUDA uint8 tensor with seeded uniform 0-255 pixels on the device."""
    import torch

    g = torch.Generator(device=t.device)
    g.manual_seed(seed)
    t.copy_(torch.randint(0, 256, t.shape, generator=g, device=t.device, dtype=torch.int32).to(torch.uint8))
