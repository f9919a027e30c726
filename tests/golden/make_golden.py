"""Generates the golden fixtures tests/golden/cases.json + arrays.npz.

Runs the REFERENCE's own code -- its headers compiled into
oracle/_ref/libipfref.so by oracle/Makefile -- on seeded inputs (the sample
stream of the reference test helper randomImage(), std::mt19937) and records
inputs, parameters and outputs.  The fixtures travel with the repository so
the parity tests can check the C restatement and the CUDA path against the
reference where the reference itself is absent.

Usage (needs the reference checkout for oracle/_ref):
    make -C oracle all && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

B = oracle.BORDERS
NAMES = {0: "constant", 1: "replicate", 2: "reflect", 3: "reflect101", 4: "wrap"}


def main() -> None:
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libipfref.so not built: run `make -C oracle all` with the reference present")
    cases = []
    arrays = {}

    def add(op, params, inputs, out):
        i = len(cases)
        entry = {"op": op, "params": params, "inputs": {}}
        for k, v in inputs.items():
            key = f"c{i}_{k}"
            arrays[key] = v
            entry["inputs"][k] = key
        arrays[f"c{i}_out"] = out
        entry["out"] = f"c{i}_out"
        cases.append(entry)

    rng = np.random.default_rng(20261203)
    img_u8 = {}

    def image(w, h, c, dt, seed):
        key = (w, h, c, np.dtype(dt).str, seed)
        if key not in img_u8:
            img_u8[key] = oracle.random_image(w, h, c, dt, seed)
        return img_u8[key]

    # gaussianBlur, uint8 (tests/test_filter.cpp style inputs), all borders
    for (w, h, c) in [(37, 23, 3), (16, 9, 1), (5, 4, 4), (1, 1, 1), (1, 13, 3), (19, 1, 1)]:
        src = image(w, h, c, np.uint8, 100 + w + h + c)
        for b in B:
            for sx, sy in [(1.0, 0.0), (2.0, 0.0), (2.3, 0.8)]:
                out = ref.gaussian_blur(src, sx, sy, 0, b)
                add("gaussian", {"sigma_x": sx, "sigma_y": sy, "ksize": 0, "border": b}, {"src": src}, out)
    # gaussianBlur<float> of uint8 and float32 sources
    src = image(33, 21, 3, np.uint8, 7)
    srcf = image(33, 21, 1, np.float32, 8)
    for b in B:
        add("gaussian", {"sigma_x": 1.5, "sigma_y": 0.0, "ksize": 0, "border": b, "dtype": "float32"}, {"src": src},
            ref.gaussian_blur(src, 1.5, 0.0, 0, b, np.float32))
        add("gaussian", {"sigma_x": 2.0, "sigma_y": 0.0, "ksize": 0, "border": b}, {"src": srcf},
            ref.gaussian_blur(srcf, 2.0, 0.0, 0, b))
    # sepFilter2D, float32 sources, random normalised taps of 3/7/15/31, delta and border value
    srcf = image(45, 38, 1, np.float32, 9)
    for L in (3, 7, 15, 31):
        kx = rng.normal(size=L)
        ky = rng.normal(size=L)
        kx /= kx.sum()
        ky /= ky.sum()
        for b in B:
            add("sep", {"border": b, "delta": 0.25, "border_value": 0.5}, {"src": srcf, "kx": kx, "ky": ky},
                ref.sep_filter(srcf, kx, ky, border=b, delta=0.25, border_value=0.5))
    # sepFilter2D with uneven taps (impulse-style) on uint8 -> uint8 / int16
    src = image(29, 17, 2, np.uint8, 10)
    for b in B:
        kx, ky = rng.normal(size=7), rng.normal(size=3)
        add("sep", {"border": b, "delta": 0.0, "border_value": 3.0, "dtype": "int16"},
            {"src": src, "kx": kx, "ky": ky}, ref.sep_filter(src, kx, ky, border=b, border_value=3.0,
                                                            out_dtype=np.int16))
    # Sobel: uint8 -> int16 (sepFilter2D<int16_t> with derivKernel taps) and float32 (sobel())
    src = image(40, 30, 1, np.uint8, 11)
    for ksize in (1, 3, 5):
        for dx, dy in ((1, 0), (0, 1), (1, 1), (2, 0)):
            for b in B:
                kx, ky = ref.sobel_taps(dx, dy, ksize)
                add("sep", {"border": b, "delta": 0.0, "border_value": 0.0, "dtype": "int16"},
                    {"src": src, "kx": kx, "ky": ky},
                    ref.sep_filter(src, kx, ky, border=b, out_dtype=np.int16))
            out = np.zeros(src.shape, np.float32)
            f = ref.lib.ref_sobel
            W, H, C = 40, 30, 1
            rc = f(src.ctypes.data, 0, W, H, C, out.ctypes.data, dx, dy, ksize, oracle.ctypes.c_double(1.0), 3)
            assert rc == 0
            add("sobel", {"dx": dx, "dy": dy, "ksize": ksize, "scale": 1.0, "border": 3}, {"src": src}, out)
    # boxFilter: odd/even sizes, normalised or not, uint8 -> uint8 / float32, all borders, borderValue 3
    for (w, h, c) in [(31, 17, 2), (12, 11, 3)]:
        src = image(w, h, c, np.uint8, 12 + c)
        for kw, kh in ((5, 3), (4, 4), (7, 7), (2, 6)):
            for norm in (True, False):
                for b in B:
                    add("box", {"kw": kw, "kh": kh, "normalize": norm, "border": b, "border_value": 3.0},
                        {"src": src}, ref.box_filter(src, kw, kh, norm, b, 3.0))
                    add("box", {"kw": kw, "kh": kh, "normalize": norm, "border": b, "border_value": 3.0,
                                "dtype": "float32"},
                        {"src": src}, ref.box_filter(src, kw, kh, norm, b, 3.0, np.float32))
    # filter2D: 3x5 N(0,1) kernel (crossval style) on float32 and uint8, all borders, borderValue 7
    k35 = rng.normal(size=(3, 5)).astype(np.float32)
    k15 = rng.normal(size=(15, 15))
    k15 = (k15 / k15.sum()).astype(np.float32)
    k15[3, 4] = 0.0  # a zero tap, skipped by the reference
    for src in (image(27, 33, 1, np.float32, 13), image(27, 33, 3, np.uint8, 14)):
        for b in B:
            add("filter2d", {"border": b, "delta": 0.5, "border_value": 7.0, "anchor": [-1, -1]},
                {"src": src, "kernel": k35}, ref.filter2d(src, k35, b, 0.5, (-1, -1), 7.0))
        add("filter2d", {"border": 3, "delta": 0.0, "border_value": 0.0, "anchor": [-1, -1]},
            {"src": src, "kernel": k15}, ref.filter2d(src, k15, 3))
        add("filter2d", {"border": 0, "delta": 0.0, "border_value": 2.0, "anchor": [3, 1]},
            {"src": src, "kernel": k35}, ref.filter2d(src, k35, 0, 0.0, (3, 1), 2.0))
    # medianBlur: exact; uint8 k = 3, 5, 7, 11 x 4 borders; float32 k = 3, 5; tiny images
    for (w, h, c) in [(31, 37, 1), (13, 9, 3), (2, 3, 1)]:
        src = image(w, h, c, np.uint8, 15 + w)
        for k in (3, 5, 7, 11):
            for b in (1, 2, 3, 4):
                add("median", {"ksize": k, "border": b}, {"src": src}, ref.median_blur(src, k, b))
    srcf = image(21, 19, 1, np.float32, 16)
    for k in (3, 5):
        add("median", {"ksize": k, "border": 1}, {"src": srcf}, ref.median_blur(srcf, k, 1))
    # erode / dilate: rect, cross, ellipse at 3x3, 5x7, 9x5, iterations 1 and 2
    for (w, h, c) in [(31, 37, 1), (14, 10, 3)]:
        src = image(w, h, c, np.uint8, 17 + c)
        for shape in (0, 1, 2):
            for sw, sh in ((3, 3), (5, 7), (9, 5)):
                se = ref.structuring_element(shape, sw, sh)
                for it in (1, 2):
                    add("erode", {"iterations": it}, {"src": src, "se": se}, ref.erode(src, se, it))
                    add("dilate", {"iterations": it}, {"src": src, "se": se}, ref.dilate(src, se, it))
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(cases, f, indent=0)
    np.savez_compressed(os.path.join(HERE, "arrays.npz"), **arrays)
    print(f"{len(cases)} cases")


if __name__ == "__main__":
    main()
