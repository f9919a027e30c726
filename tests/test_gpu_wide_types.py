"""int32 and double images (ImageI32, ImageD) and double / int32 outputs of
uint8 sources (TOut), through the C ABI, against the oracle.

These calls accumulate in FP64 in the reference's own operation order
(separable: the row pass from 0 then the column pass from delta, tap by tap;
filter2D: delta then each non-zero tap in row-major order; products and
sums rounded separately, as the reference is built without FMA contraction)
and round with its saturate_cast, so the bar is bit-exact -- except the box
filter of a double image, whose reference running sums round in an order
that depends on the position (filter.hpp:220-251): within 1e-12 relative
there.  Median and morphology are exact order statistics.
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
import oracle

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (37, 5, 3), (130, 67, 1), (301, 97, 4)]


def _image(w, h, c, dt, seed):
    img = oracle.random_image(w, h, c, dt, seed)
    if dt == np.int32:  # values beyond FP32's exact range
        img = (img.astype(np.int64) * 40000 - 5_000_000).astype(np.int32)
    return img


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("dt", [np.int32, np.float64, np.uint8], ids=["i32", "f64", "u8"])
def test_fp64_accumulated_calls_match_the_oracle(gpu, orc, dt, shape):
    w, h, c = shape
    img = _image(w, h, c, dt, 7 * w + h + c)
    rng = np.random.default_rng(w + 3 * h + c)
    outs = (None, np.float64, np.int32) if dt != np.uint8 else (np.float64, np.int32)
    B = ipf.BorderMode
    for b in oracle.BORDERS:
        for kw, kh in ((3, 3), (7, 5), (1, 9), (33, 3)):
            kx, ky = rng.normal(size=kw), rng.normal(size=kh)
            for od in outs:
                got = ipf.sepFilter2D(img, kx, ky, B(b), 0.3, 2.0, dtype=od)
                want = orc.sep_filter(img, kx, ky, border=b, delta=0.3, border_value=2.0, out_dtype=od)
                np.testing.assert_array_equal(got, want, err_msg=f"sep {kw}x{kh} border {b} out {od}")
            k2 = rng.normal(size=(kh, kw)).astype(np.float32)
            k2[0, 0] = 0.0
            for od in outs:
                got = ipf.filter2D(img, k2, B(b), 0.5, (-1, -1), 7.0, dtype=od)
                want = orc.filter2d(img, k2, b, 0.5, (-1, -1), 7.0, od)
                np.testing.assert_array_equal(got, want, err_msg=f"filter2D {kw}x{kh} border {b} out {od}")
                for norm in (True, False):
                    got = ipf.boxFilter(img, kw, kh, norm, B(b), 3.0, dtype=od)
                    want = orc.box_filter(img, kw, kh, norm, b, 3.0, od)
                    if dt == np.float64 or (od is None and dt == np.float64):
                        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-9)
                    else:
                        np.testing.assert_array_equal(got, want, err_msg=f"box {kw}x{kh} {norm} {b} {od}")
    if dt == np.uint8:
        return
    for b in (oracle.REPLICATE, oracle.REFLECT, oracle.REFLECT101, oracle.WRAP):
        for k in (3, 5, 7, 9):
            np.testing.assert_array_equal(ipf.medianBlur(img, k, B(b)), orc.median_blur(img, k, b))
    for shp in (ipf.MorphShape.Rect, ipf.MorphShape.Cross, ipf.MorphShape.Ellipse):
        for sw, sh in ((3, 3), (9, 7), (15, 15)):
            se = ipf.getStructuringElement(shp, sw, sh)
            for it in (1, 2):
                np.testing.assert_array_equal(ipf.erode(img, se, it), orc.erode(img, se, it))
                np.testing.assert_array_equal(ipf.dilate(img, se, it), orc.dilate(img, se, it))


def test_gaussian_and_sobel_to_double_match_the_oracle(gpu, orc):
    """TOut = double from uint8, the form ssim and the pyramids use."""
    img = oracle.random_image(211, 143, 3, np.uint8, 5)
    for s in (0.8, 1.5, 2.0):
        got = ipf.gaussianBlur(img, s, dtype=np.float64)
        want = orc.gaussian_blur(img, s, 0.0, 0, oracle.REFLECT101, np.float64)
        np.testing.assert_array_equal(got, want)
    for dx, dy in ((1, 0), (0, 1), (1, 1)):
        got = ipf.sobel(img, dx, dy, 5, 0.5, ipf.BorderMode.Replicate, dtype=np.float64)
        want = orc.sobel(img, dx, dy, 5, 0.5, oracle.REPLICATE, out_dtype=np.float64)
        np.testing.assert_array_equal(got, want)


def test_device_tensors_of_wide_types(gpu, orc):
    import torch

    img = _image(129, 65, 1, np.int32, 3)
    got = ipf.gaussianBlur(torch.from_numpy(img).cuda(), 1.2).cpu().numpy()
    np.testing.assert_array_equal(got, orc.gaussian_blur(img, 1.2))
    d = np.random.default_rng(2).random((65, 129, 3))
    got = ipf.medianBlur(torch.from_numpy(d).cuda(), 5).cpu().numpy()
    np.testing.assert_array_equal(got, orc.median_blur(d, 5, oracle.REPLICATE))
