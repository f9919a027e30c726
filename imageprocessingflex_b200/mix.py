"""Seeded synthetic workloads of the batched and served forms.

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


def fill_uniform_u8(t, seed: int) -> None:
    """Fills a CUDA uint8 tensor with seeded uniform 0-255 pixels on the device."""
    import torch

    g = torch.Generator(device=t.device)
    g.manual_seed(seed)
    t.copy_(torch.randint(0, 256, t.shape, generator=g, device=t.device, dtype=torch.int32).to(torch.uint8))
