"""The reference's other filters and its callers of the filters, on the GPU,
against the oracle (whose restatements test_oracle.py pins bit for bit to
the compiled reference):

  morphologyEx, integralImage, adaptiveThreshold, pyrDown / pyrUp,
  canny, ssim (its map)             -- bit-exact;
  bilateralFilter                   -- bit-exact for integer images (the
                                       reference's range table), within
                                       1e-12 relative for float images
                                       (exp evaluated per tap on the GPU);
  ssim (the mean)                   -- within 1e-12 relative (parallel sum);
  cornerHarris / cornerMinEigenVal  -- within 1e-6 of the response scale
                                       (FP64 window sums where the reference
                                       keeps FP64 running sums).
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
import oracle

pytestmark = pytest.mark.gpu

DTYPES = [np.uint8, np.uint16, np.int16, np.int32, np.float32, np.float64]
SHAPES = [(1, 1, 1), (37, 23, 3), (130, 67, 1), (301, 97, 4)]


def _ids(d):
    return np.dtype(d).name


@pytest.mark.parametrize("dt", DTYPES, ids=_ids)
def test_morphology_ex_integral_pyramids(gpu, orc, dt):
    for w, h, c in SHAPES:
        img = oracle.random_image(w, h, c, dt, 3 * w + h + c)
        for op in ipf.MorphOp:
            for shape, sw, sh in ((ipf.MorphShape.Rect, 3, 3), (ipf.MorphShape.Ellipse, 7, 5),
                                  (ipf.MorphShape.Rect, 15, 11)):
                se = ipf.getStructuringElement(shape, sw, sh)
                for it in (1, 2):
                    np.testing.assert_array_equal(ipf.morphologyEx(img, op, se, it), orc.morphology_ex(img, op, se, it),
                                                  err_msg=f"{op.name} {sw}x{sh} it {it} {w}x{h}x{c}")
        for sq in (False, True):
            np.testing.assert_array_equal(ipf.integralImage(img, sq), orc.integral(img, sq))
        np.testing.assert_array_equal(ipf.pyrDown(img), orc.pyr_down(img))
        np.testing.assert_array_equal(ipf.pyrUp(img), orc.pyr_up(img))


@pytest.mark.parametrize("dt", DTYPES, ids=_ids)
def test_bilateral(gpu, orc, dt):
    for w, h, c in SHAPES:
        img = oracle.random_image(w, h, c, dt, w + 5 * h + c)
        for b in oracle.BORDERS:
            for d, sc, ss in ((5, 30.0, 2.0), (0, 0.3, 1.4), (9, 75.0, 75.0)):
                got = ipf.bilateralFilter(img, d, sc, ss, ipf.BorderMode(b))
                want = orc.bilateral(img, d, sc, ss, b)
                if dt in (np.float32, np.float64):
                    np.testing.assert_allclose(got, want, rtol=1e-12 if dt == np.float64 else 1e-6, atol=1e-12)
                else:
                    np.testing.assert_array_equal(got, want, err_msg=f"d {d} border {b} {w}x{h}x{c}")


@pytest.mark.parametrize("dt", DTYPES, ids=_ids)
def test_adaptive_threshold_and_corners(gpu, orc, dt):
    for w, h in ((1, 1), (45, 31), (257, 130)):
        img = oracle.random_image(w, h, 1, dt, w * 3 + h)
        for method in ipf.AdaptiveMethod:
            for tt in (ipf.ThresholdType.Binary, ipf.ThresholdType.BinaryInv):
                for bs, cc in ((3, 2.0), (7, -1.5), (11, 0.0)):
                    got = ipf.adaptiveThreshold(img, 200.0, method, tt, bs, cc)
                    want = orc.adaptive_threshold(img, 200.0, int(method), int(tt), bs, cc)
                    if dt in (np.float32, np.float64) and method == ipf.AdaptiveMethod.Mean:
                        # float boxFilter: FP64 window sums vs the reference's running sums
                        assert (got != want).mean() < 1e-3
                    else:
                        np.testing.assert_array_equal(got, want, err_msg=f"{method.name} {tt.name} {bs}")
        for bs, ks in ((3, 3), (5, 5), (2, 1)):
            for me in (False, True):
                got = ipf.cornerMinEigenVal(img, bs, ks) if me else ipf.cornerHarris(img, bs, ks, 0.04)
                want = orc.corner(img, bs, ks, 0.04, me)
                scale = max(float(np.abs(want).max(initial=0.0)), 1e-30)
                np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * scale)


@pytest.mark.parametrize("dt", DTYPES, ids=_ids)
def test_canny_and_ssim(gpu, orc, dt):
    integer = dt in (np.uint8, np.uint16, np.int16, np.int32)
    for w, h, c in SHAPES:
        img = oracle.random_image(w, h, c, dt, 11 * w + h + c)
        for ks in (3, 5, 7):
            for l2 in (False, True):
                lo, hi = (20.0, 60.0) if integer else (0.05, 0.3)
                np.testing.assert_array_equal(ipf.canny(img, lo, hi, ks, l2), orc.canny(img, lo, hi, ks, l2),
                                              err_msg=f"ksize {ks} l2 {l2} {w}x{h}x{c}")
        other = oracle.random_image(w, h, c, dt, 7 * w + h)
        g, gm = ipf.ssim(img, other, ssimMap=True)
        r, rm = orc.ssim(img, other, True)
        np.testing.assert_array_equal(gm, rm)
        assert abs(g - r) <= 1e-12 * max(1.0, abs(r)), (g, r)
        assert ipf.ssim(img, img) == pytest.approx(1.0, abs=1e-12)


def test_canny_on_an_image_with_long_edges(gpu, orc):
    """Hysteresis over long weak chains that cross many GPU tiles."""
    h, w = 300, 400
    y, x = np.mgrid[0:h, 0:w]
    img = (128 + 100 * np.sin(x / 17.0) * np.cos(y / 23.0)).astype(np.uint8)
    img = np.ascontiguousarray(np.dstack([img, img[::-1], img[:, ::-1]]))
    for lo, hi in ((5.0, 200.0), (1.0, 400.0), (30.0, 31.0)):
        np.testing.assert_array_equal(ipf.canny(img, lo, hi), orc.canny(img, lo, hi))


def test_callers_on_device_tensors(gpu, orc):
    import torch

    img = oracle.random_image(211, 130, 3, np.uint8, 9)
    dev = torch.from_numpy(img).cuda()
    se = ipf.getStructuringElement(ipf.MorphShape.Cross, 5)
    np.testing.assert_array_equal(ipf.morphologyEx(dev, ipf.MorphOp.Gradient, se).cpu().numpy(),
                                  orc.morphology_ex(img, 4, se, 1))
    np.testing.assert_array_equal(ipf.pyrDown(dev).cpu().numpy(), orc.pyr_down(img))
    np.testing.assert_array_equal(ipf.canny(dev, 20.0, 60.0).cpu().numpy(), orc.canny(img, 20.0, 60.0))
    np.testing.assert_array_equal(ipf.integralImage(dev).cpu().numpy(), orc.integral(img))


@pytest.mark.parametrize("dt", DTYPES, ids=_ids)
def test_laplacian_gradient_magnitude_unsharp_mask(gpu, orc, dt):
    """laplacian, gradientMagnitude and unsharpMask against the oracle (pinned
    to the compiled reference in test_oracle.py).  Exact where the GPU's sums
    are exact or FP64 (integer sources with integer taps; int32 and double
    sources; unsharpMask always, whose blur is FP64); otherwise FP32 against
    the reference's FP64 sums, within 1e-5 of the result's scale plus 1e-6 of
    the summed terms' scale (a flat window cancels terms of |scale| x the
    kernel's L1 norm x the largest sample down to 0, and FP32 keeps the
    rounding of those terms)."""
    integer = dt in (np.uint8, np.uint16, np.int16, np.int32)
    fp64 = dt in (np.int32, np.float64)
    l1 = {1: 8.0, 3: 32.0, 5: 128.0}  # L1 norms of the ksize 1 / 3 / 5 Laplacian kernels

    def check(got, want, exact, what, terms=0.0):
        if exact:
            np.testing.assert_array_equal(got, want, err_msg=what)
        else:
            scale = max(1.0, float(np.abs(want).max(initial=0.0)))
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5 * scale + 1e-6 * terms, err_msg=what)

    for w, h, c in SHAPES:
        img = oracle.random_image(w, h, c, dt, 5 * w + 3 * h + c)
        peak = float(np.abs(img.astype(np.float64)).max(initial=0.0))
        for ks in (1, 3, 5):
            for sc in (1.0, 0.37):
                for b in oracle.BORDERS:
                    check(ipf.laplacian(img, ks, sc, ipf.BorderMode(b)), orc.laplacian(img, ks, sc, b),
                          fp64 or (integer and sc == 1.0), f"laplacian ksize {ks} scale {sc} border {b} {w}x{h}x{c}",
                          sc * l1[ks] * peak)
            check(ipf.gradientMagnitude(img, ks), orc.gradient_magnitude(img, ks), fp64 or integer,
                  f"gradientMagnitude ksize {ks} {w}x{h}x{c}")
        for sigma, amount, thr in ((1.0, 1.0, 0.0), (2.3, 0.6, 4.0), (0.5, 2.5, 0.01)):
            np.testing.assert_array_equal(ipf.unsharpMask(img, sigma, amount, thr), orc.unsharp_mask(img, sigma, amount, thr),
                                          err_msg=f"unsharpMask {sigma} {amount} {thr} {w}x{h}x{c}")


def test_scharr_prewitt_sharpen_emboss(gpu, orc):
    """The thin wrappers over sepFilter2D<float> / filter2D against the
    oracle with the reference's taps (filter.hpp:411-422, 487-496): exact with
    integer taps on uint8, within 1 LSB for sharpen's fractional ones."""
    for w, h, c in SHAPES:
        img = oracle.random_image(w, h, c, np.uint8, 17 * w + h + c)
        d, s = [-1.0, 0.0, 1.0], [3.0, 10.0, 3.0]
        np.testing.assert_array_equal(ipf.scharr(img, 1, 0), orc.sep_filter(img, d, s, out_dtype=np.float32))
        np.testing.assert_array_equal(ipf.scharr(img, 0, 1), orc.sep_filter(img, s, d, out_dtype=np.float32))
        p = [1.0, 1.0, 1.0]
        np.testing.assert_array_equal(ipf.prewitt(img, 1, 0), orc.sep_filter(img, d, p, out_dtype=np.float32))
        np.testing.assert_array_equal(ipf.prewitt(img, 0, 1), orc.sep_filter(img, p, d, out_dtype=np.float32))
        em = np.array([[-2, -1, 0], [-1, 1, 1], [0, 1, 2]], np.float32)
        np.testing.assert_array_equal(ipf.emboss(img), orc.filter2d(img, em))
        st = np.float32(0.7)
        sk = np.array([[0, -st, 0], [-st, np.float32(1) + np.float32(4) * st, -st], [0, -st, 0]], np.float32)
        diff = np.abs(ipf.sharpen(img, 0.7).astype(np.int32) - orc.filter2d(img, sk).astype(np.int32))
        assert diff.max(initial=0) <= 1
    with pytest.raises(ipf.Error, match="scharr"):
        ipf.scharr(oracle.random_image(4, 4, 1, np.uint8, 1), 1, 1)
