"""The tensor-core (tcgen05) split-precision form of filter2D against the
oracle, and against the FP32 CUDA-core form's own error.

Bars: uint8 outputs within 1 LSB of the reference (mismatch rate printed);
float outputs within the filter2D tolerance of the rest of the suite
(max(1e-5 max(1, |ref|), FP32 summation bound)); and on the dense N(0,1)
kernels of the measured configuration the split form's error against the
FP64 oracle is no larger than the FP32 form's.
"""
import numpy as np
import pytest

import golden_cases as G
import imageprocessingflex_b200 as ipf
import oracle

pytestmark = pytest.mark.gpu


def _taps(kh, kw, seed):
    rng = np.random.default_rng(seed)
    while True:
        w = rng.standard_normal((kh, kw))
        if abs(w.sum()) > 0.25 * np.sqrt(kw * kh):
            return (w / w.sum()).astype(np.float32)


SHAPES = [(1, 1), (3, 7), (130, 65), (333, 257), (129, 200), (600, 70)]


@pytest.mark.parametrize("wh", SHAPES, ids=lambda s: f"{s[0]}x{s[1]}")
def test_split_u8_all_borders_vs_oracle(gpu, orc, wh):
    w, h = wh
    img = oracle.random_image(w, h, 1, np.uint8, w + h)
    for kw, kh, anchor in ((15, 15, (-1, -1)), (31, 31, (-1, -1)), (16, 9, (3, 8)), (32, 33, (31, 0))):
        k = _taps(kh, kw, kw * 100 + kh)
        for b in oracle.BORDERS:
            got = ipf.filter2D(img, k, ipf.BorderMode(b), 0.5, anchor, 7.0, form="split")
            want = orc.filter2d(img, k, b, 0.5, anchor, 7.0)
            d = np.abs(got.astype(int) - want.astype(int))
            assert d.max(initial=0) <= 1, (kw, kh, b, d.max())
            for od in ((np.float32, np.int16) if b == oracle.REFLECT101 else ()):
                got = ipf.filter2D(img, k, ipf.BorderMode(b), 0.5, anchor, 7.0, dtype=od, form="split")
                want = orc.filter2d(img, k, b, 0.5, anchor, 7.0, od)
                pp = {"border_value": 7.0, "delta": 0.5}
                G.compare(got, want, G.tolerance("filter2d", pp, {"src": img, "kernel": k}, want))


@pytest.mark.parametrize("wh", [(333, 257), (5, 3), (128, 64)], ids=lambda s: f"{s[0]}x{s[1]}")
def test_split_f32_vs_oracle(gpu, orc, wh):
    w, h = wh
    img = oracle.random_image(w, h, 1, np.float32, 3 * w + h)
    img = img * np.float32(50.0) - np.float32(10.0)  # values beyond [0,1]: the per-tile scale matters
    for kw, kh in ((15, 15), (31, 31), (7, 20)):
        k = _taps(kh, kw, kw + kh)
        for b in oracle.BORDERS:
            got = ipf.filter2D(img, k, ipf.BorderMode(b), 0.25, (-1, -1), 3.0, form="split")
            want = orc.filter2d(img, k, b, 0.25, (-1, -1), 3.0)
            pp = {"border_value": 3.0, "delta": 0.25}
            G.compare(got, want, G.tolerance("filter2d", pp, {"src": img, "kernel": k}, want))


def test_split_error_vs_fp64_no_worse_than_fp32_form(gpu, orc):
    """The measured configuration's kernels (dense N(0,1), normalised) on a
    1024 x 512 crop: error of each form against the FP64 oracle."""
    for dt in (np.uint8, np.float32):
        img = oracle.random_image(1024, 512, 1, dt, 11)
        for kk in (15, 31):
            k = _taps(kk, kk, 1000 + kk)
            ref = orc.filter2d(img, k, oracle.REFLECT101, 0.0, (-1, -1), 0.0, np.float64)
            e_split = np.abs(ipf.filter2D(img, k, form="split", dtype=np.float32).astype(np.float64) - ref)
            e_fp32 = np.abs(ipf.filter2D(img, k, form="fp32", dtype=np.float32).astype(np.float64) - ref)
            print(f"\n{np.dtype(dt).name} {kk}x{kk}: max |err| split {e_split.max():.3e} fp32 {e_fp32.max():.3e}; "
                  f"mean split {e_split.mean():.3e} fp32 {e_fp32.mean():.3e}")
            # no worse than the FP32 form, max and mean
            assert e_split.max() <= e_fp32.max() + 1e-12
            assert e_split.mean() <= e_fp32.mean() + 1e-12
            if dt == np.uint8:
                want = orc.filter2d(img, k, oracle.REFLECT101)
                got = ipf.filter2D(img, k, form="split")
                d = np.abs(got.astype(int) - want.astype(int))
                assert d.max() <= 1
                print(f"u8 out {kk}x{kk}: mismatch rate {(d > 0).mean():.3e}, saturated {(want == 0).mean() + (want == 255).mean():.3f}")


def test_split_device_tensors_match_host(gpu):
    import torch

    img = oracle.random_image(700, 300, 1, np.uint8, 5)
    k = _taps(31, 31, 9)
    want = ipf.filter2D(img, k, form="split")
    got = ipf.filter2D(torch.from_numpy(img).cuda(), k, form="split").cpu().numpy()
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("c", [3, 4])
def test_split_u8_interleaved_channels_vs_oracle(gpu, orc, c):
    """3- and 4-channel uint8 images: the row of W*C samples with the taps C
    samples apart; the same 1-LSB bar, every border."""
    for w, h in ((1, 1), (7, 3), (130, 65), (333, 129)):
        img = oracle.random_image(w, h, c, np.uint8, 7 * w + h + c)
        for kw, kh, anchor in ((15, 15, (-1, -1)), (31, 31, (-1, -1)), (16, 9, (3, 8)), (5, 33, (4, 0))):
            k = _taps(kh, kw, kw * 100 + kh + c)
            for b in oracle.BORDERS:
                got = ipf.filter2D(img, k, ipf.BorderMode(b), 0.5, anchor, 7.0, form="split")
                want = orc.filter2d(img, k, b, 0.5, anchor, 7.0)
                d = np.abs(got.astype(int) - want.astype(int))
                assert d.max(initial=0) <= 1, (w, h, kw, kh, b, d.max())
        got = ipf.filter2D(img, k, ipf.BorderMode.Reflect101, 0.0, (-1, -1), 0.0, dtype=np.float32, form="split")
        want = orc.filter2d(img, k, oracle.REFLECT101, 0.0, (-1, -1), 0.0, np.float32)
        G.compare(got, want, G.tolerance("filter2d", {"border_value": 0.0, "delta": 0.0}, {"src": img, "kernel": k},
                                         want))


def test_split_rejects_what_it_does_not_cover(gpu):
    img3 = oracle.random_image(40, 30, 3, np.float32, 1)
    with pytest.raises(ipf.Error, match="tensor-core form"):
        ipf.filter2D(img3, _taps(15, 15, 1), form="split")
    img = oracle.random_image(40, 30, 1, np.uint8, 1)
    with pytest.raises(ipf.Error, match="tensor-core form"):
        ipf.filter2D(img, _taps(15, 40, 1), form="split")


def test_register_tiled_fp32_form_equals_the_general_one(gpu, tmp_path):
    """The register-tiled FP32 kernel (1 and 3 channels, 9..32 taps per row)
    repeats the general FP32 kernel's accumulation sequence, so their
    outputs are bit-identical; the general one is forced in a child process
    with IPFC_F2D_TILED=0."""
    import os
    import subprocess
    import sys

    code = r'''
import sys, numpy as np, imageprocessingflex_b200 as ipf, oracle
out = {}
for c in (1, 3):
    for dt in (np.uint8, np.float32):
        img = oracle.random_image(517, 203, c, dt, 7 + c)
        for kw, kh in ((9, 9), (15, 15), (16, 3), (31, 31), (32, 33), (13, 21)):
            if c == 3 and kw > 16:
                continue
            rng = np.random.default_rng(kw * 100 + kh)
            k = rng.normal(size=(kh, kw)).astype(np.float32)
            k /= k.sum()
            for b in range(5):
                for od in (None, np.float32):
                    key = f"{c}_{np.dtype(dt).name}_{kw}x{kh}_{b}_{od is None}"
                    out[key] = ipf.filter2D(img, k, ipf.BorderMode(b), 0.5, (-1, -1), 7.0, dtype=od, form="fp32")
np.savez(sys.argv[1], **out)
'''
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = {}
    for tiled in ("1", "0"):
        f = str(tmp_path / f"out_{tiled}.npz")
        env = dict(os.environ, IPFC_F2D_TILED=tiled, PYTHONPATH=root)
        r = subprocess.run([sys.executable, "-c", code, f], env=env, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        res[tiled] = np.load(f)
    assert set(res["1"].files) == set(res["0"].files) and len(res["1"].files) > 50
    for key in res["1"].files:
        np.testing.assert_array_equal(res["1"][key], res["0"][key], err_msg=key)
