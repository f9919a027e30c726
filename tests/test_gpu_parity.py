"""Parity of the CUDA path (through the C ABI) with the reference.

Every golden fixture -- outputs of the reference's own compiled headers -- is
replayed through the CUDA library from host arrays, and a subset from device
tensors; seeded random cases, edge shapes and full-size configurations are
compared with the C restatement.  Bars (see golden_cases.tolerance): exact
for median, morphology, integer box sums and integer-tap separable filters;
within 1 LSB for integer outputs of FP32-accumulated sums, with the mismatch
rate reported; float outputs within 1e-5 x max(1, |ref|).
"""
import numpy as np
import pytest

import golden_cases as G
import oracle

pytestmark = pytest.mark.gpu

CASES = G.case_ids()


@pytest.mark.parametrize("idx", range(len(CASES)), ids=CASES)
def test_golden_host_arrays(gpu, idx):
    op, p, x, want = G.case(idx)
    got = G.run_gpu(gpu, op, p, x)
    G.compare(got, want, G.tolerance(op, p, x, want))


@pytest.mark.parametrize("idx", range(0, len(CASES), 5), ids=CASES[::5])
def test_golden_device_tensors(gpu, idx):
    op, p, x, want = G.case(idx)
    got = G.run_gpu(gpu, op, p, x, device_images=True)
    G.compare(got, want, G.tolerance(op, p, x, want))


def test_probe_border_index(gpu, orc):
    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    p = torch.arange(-70, 71, dtype=torch.int32, device="cuda")
    out = torch.empty_like(p)
    for n in (1, 2, 3, 5, 8, 13):
        for mode in oracle.BORDERS:
            assert lib.ipfc_probe_border_index(p.data_ptr(), out.data_ptr(), p.numel(), n, mode, None) == 0
            torch.cuda.synchronize()
            want = [oracle.restatement().lib.orc_border_index(int(v), n, mode) for v in range(-70, 71)]
            assert out.cpu().tolist() == want, (n, mode)


def test_probe_saturate(gpu):
    import ctypes

    import torch

    from imageprocessingflex_b200 import _lib

    lib = _lib.load()
    orc = oracle.restatement().lib
    orc.orc_saturate.restype = ctypes.c_double
    orc.orc_saturate.argtypes = [ctypes.c_double, ctypes.c_int]
    vals = np.array([0.0, 0.5, -0.5, 0.49999997, 1.5, 2.5, -1.5, -2.5, 254.5, 255.49, 255.5, 256.0, -0.49999997,
                     32766.5, 32767.5, -32768.5, -32769.0, 65534.5, 65535.5, 1e9, -1e9, np.inf, -np.inf, np.nan,
                     0.49999997, 100.50001, 7.4999995], np.float32)
    v = torch.from_numpy(vals).cuda()
    for code, tdt in ((0, torch.uint8), (1, torch.uint16), (2, torch.int16), (4, torch.float32)):
        out = torch.empty(vals.size, dtype=tdt, device="cuda")
        assert lib.ipfc_probe_saturate(v.data_ptr(), out.data_ptr(), vals.size, code, None) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        want = np.array([orc.orc_saturate(float(x), code) for x in vals])
        np.testing.assert_array_equal(got, want, err_msg=f"dtype code {code}")


# ---- known answers of the reference's unit tests, on the GPU ----------------

def test_kat_impulse_and_constant(gpu):
    B = gpu.BorderMode
    impulse = np.zeros((7, 7), np.float32)
    impulse[3, 3] = 1
    r = gpu.filter2D(impulse, np.arange(1, 10, dtype=np.float32).reshape(3, 3), B.Constant)
    assert r[2, 2] == 9 and r[4, 4] == 1 and r[2, 3] == 8
    sep = gpu.sepFilter2D(impulse, [1, 2, 3], [4, 5, 6], B.Constant)
    assert sep[2, 2] == 18 and sep[2, 4] == 6 and sep[4, 2] == 12
    c = np.full((15, 20, 3), 77, np.uint8)
    np.testing.assert_array_equal(gpu.gaussianBlur(c, 2.0), c)
    np.testing.assert_array_equal(gpu.blur(c, 5), c)
    np.testing.assert_array_equal(gpu.medianBlur(c, 5), c)
    np.testing.assert_array_equal(gpu.medianBlur(c, 9), c)
    for m in (B.Replicate, B.Reflect, B.Reflect101, B.Wrap):
        np.testing.assert_array_equal(gpu.boxFilter(c, 4, 6, True, m), c)


def test_kat_gradients(gpu):
    y, x = np.mgrid[0:16, 0:16]
    ramp = (3 * x + 2 * y).astype(np.float32)
    assert abs(gpu.sobel(ramp, 1, 0)[8, 8] - 24) < 1e-4
    assert abs(gpu.sobel(ramp, 0, 1)[8, 8] - 16) < 1e-4
    assert abs(gpu.sobel(ramp, 1, 0, 1)[8, 8] - 6) < 1e-4
    assert abs(gpu.sobel(ramp, 1, 0, 5)[8, 8] - 384) < 1e-3


def test_kat_morphology(gpu):
    img = np.zeros((9, 9), np.uint8)
    img[3:6, 3:6] = 255
    er = gpu.erode(img)
    assert np.count_nonzero(er) == 1 and er[4, 4] == 255
    di = gpu.dilate(img)
    assert np.count_nonzero(di) == 25
    np.testing.assert_array_equal(gpu.erode(di), img)
    cross = gpu.dilate(er, gpu.getStructuringElement(gpu.MorphShape.Cross, 3))
    assert np.count_nonzero(cross) == 5
    np.testing.assert_array_equal(gpu.dilate(er, None, 2), gpu.dilate(er, gpu.getStructuringElement(0, 5)))
    white = np.full((4, 6, 2), 255, np.uint8)
    np.testing.assert_array_equal(gpu.erode(white, gpu.getStructuringElement(gpu.MorphShape.Ellipse, 5)), white)


# ---- seeded random cases and edge shapes vs the restatement -----------------

EDGE_SHAPES = [(1, 1, 1), (1, 7, 3), (9, 1, 1), (2, 3, 4), (3, 2, 2), (17, 5, 3), (130, 33, 1), (257, 70, 3),
               (64, 64, 4)]


@pytest.mark.parametrize("shape", EDGE_SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_random_cases_vs_restatement(gpu, orc, shape):
    w, h, c = shape
    rng = np.random.default_rng(w * 1000 + h * 10 + c)
    B = gpu.BorderMode
    for dt in (np.uint8, np.float32, np.uint16, np.int16):
        img = oracle.random_image(w, h, c, dt, w + 3 * h + c)
        for b in oracle.BORDERS:
            for kw, kh in ((3, 3), (13, 13), (4, 2), (1, 5), (31, 7)):
                kx, ky = rng.normal(size=kw), rng.normal(size=kh)
                for od in (None, np.float32, np.int16):
                    got = gpu.sepFilter2D(img, kx, ky, B(b), 0.3, 2.0, dtype=od)
                    want = orc.sep_filter(img, kx, ky, border=b, delta=0.3, border_value=2.0, out_dtype=od)
                    x = {"src": img, "kx": kx, "ky": ky}
                    pp = {"border_value": 2.0, "delta": 0.3}
                    G.compare(got, want, G.tolerance("sep", pp, x, want))
                k2 = rng.normal(size=(kh, kw)).astype(np.float32)
                got = gpu.filter2D(img, k2, B(b), 0.5, (-1, -1), 7.0)
                want = orc.filter2d(img, k2, b, 0.5, (-1, -1), 7.0)
                pp = {"border_value": 7.0, "delta": 0.5}
                G.compare(got, want, G.tolerance("filter2d", pp, {"src": img, "kernel": k2}, want))
                for norm in (True, False):
                    for od in (None, np.float32):
                        got = gpu.boxFilter(img, kw, kh, norm, B(b), 3.0, dtype=od)
                        want = orc.box_filter(img, kw, kh, norm, b, 3.0, od)
                        pp = {"kw": kw, "kh": kh, "normalize": norm, "border_value": 3.0}
                        G.compare(got, want, G.tolerance("box", pp, {"src": img}, want))
            if b != 0:
                for k in (1, 3, 5, 7, 9):
                    np.testing.assert_array_equal(gpu.medianBlur(img, k, B(b)), orc.median_blur(img, k, b))
        for shp in (0, 1, 2):
            for sw, sh in ((3, 3), (5, 7), (4, 2), (1, 1)):
                se = orc.structuring_element(shp, sw, sh)
                for it in (0, 1, 3):
                    np.testing.assert_array_equal(gpu.erode(img, se, it), orc.erode(img, se, it))
                    np.testing.assert_array_equal(gpu.dilate(img, se, it), orc.dilate(img, se, it))


def test_box_exact_ties_u8(gpu, orc):
    """Even windows give exact x.5 means; the rounding must follow the
    reference's FP64 expression tie by tie."""
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, size=(64, 96, 1), dtype=np.uint8)
    for kw, kh in ((2, 1), (2, 2), (4, 4), (6, 2), (8, 8), (10, 6), (2, 50)):
        for b in oracle.BORDERS:
            np.testing.assert_array_equal(gpu.boxFilter(img, kw, kh, True, gpu.BorderMode(b), 3.0),
                                          orc.box_filter(img, kw, kh, True, b, 3.0))


def test_long_taps_two_pass_form(gpu, orc):
    """Kernels longer than the fused form takes (two-pass with scratch)."""
    img = oracle.random_image(300, 120, 2, np.float32, 4)
    rng = np.random.default_rng(9)
    kx, ky = rng.normal(size=101), rng.normal(size=67)
    kx /= kx.sum()
    ky /= ky.sum()
    for b in oracle.BORDERS:
        got = gpu.sepFilter2D(img, kx, ky, gpu.BorderMode(b), 0.1, 0.5)
        want = orc.sep_filter(img, kx, ky, border=b, delta=0.1, border_value=0.5)
        x = {"src": img, "kx": kx, "ky": ky}
        G.compare(got, want, G.tolerance("sep", {"delta": 0.1, "border_value": 0.5}, x, want))


# ---- full-size configurations ------------------------------------------------

def _lsb_report(got, want, label):
    d = np.abs(got.astype(np.int32) - want.astype(np.int32))
    assert d.max() <= 1, f"{label}: max |diff| {d.max()}"
    rate = float((d > 0).mean())
    print(f"\n{label}: mismatch rate {rate:.3e} ({int((d > 0).sum())} of {d.size} samples), max 1 LSB")
    return rate


def test_fullsize_gaussian_u8_rgb(gpu, orc):
    """gaussianBlur sigma=2 (13 taps), 1920x1080x3 and 3840x2160x3 uint8, Reflect101."""
    for w, h in ((1920, 1080), (3840, 2160)):
        img = oracle.random_image(w, h, 3, np.uint8, 1)
        got = gpu.gaussianBlur(img, 2.0)
        want = orc.gaussian_blur(img, 2.0)
        rate = _lsb_report(got, want, f"gaussian {w}x{h}x3")
        assert rate < 1e-4


@pytest.mark.parametrize("c", [1, 3, 4])
def test_fullsize_gaussian_u8_every_tap_count(gpu, orc, c):
    """gaussianBlur on 3840x2160 uint8 at sigmas giving 3, 7, 9, 11 and 15
    taps, 1, 3 and 4 channels: the default path (tensor-core kernel from 9 taps
    on 3 or 4 channels and 15 on one, the CUDA-core kernel below) within 1 LSB,
    mismatch rate below 1e-4."""
    img = oracle.random_image(3840, 2160, c, np.uint8, 20 + c)
    for sigma in (0.4, 1.0, 1.4, 1.7, 2.4):
        got = gpu.gaussianBlur(img, sigma)
        want = orc.gaussian_blur(img, sigma)
        rate = _lsb_report(got, want, f"gaussian sigma {sigma} 3840x2160x{c}")
        assert rate < 1e-4


def test_fullsize_sobel_int16_exact(gpu, orc):
    img = oracle.random_image(3840, 2160, 1, np.uint8, 2)
    for ksize in (3, 5):
        for dx, dy in ((1, 0), (0, 1)):
            got = gpu.sobel(img, dx, dy, ksize, dtype=np.int16)
            kx, ky = orc.sobel_taps(dx, dy, ksize)
            want = orc.sep_filter(img, kx, ky, out_dtype=np.int16)
            np.testing.assert_array_equal(got, want)


def d2_taps(L, seed=0):
    """Seeded N(0,1) taps of length L normalised to sum 1 (the separable sweep
    configuration), drawing until the raw sum is not small (|sum| >= L/4),
    so normalisation does not blow the taps up."""
    rng = np.random.default_rng(seed * 1000 + L)
    while True:
        k = rng.normal(size=L)
        if abs(k.sum()) >= L / 4:
            return k / k.sum()


def test_fullsize_sep_f32(gpu, orc):
    """3840x2160 float32 in [0, 1), normalised random taps 3/7/15/31 under
    every border: within 1e-5 absolute of the reference."""
    img = oracle.random_image(3840, 2160, 1, np.float32, 3)
    for L in (3, 7, 15, 31):
        kx, ky = d2_taps(L, 1), d2_taps(L, 2)
        for b in oracle.BORDERS:
            got = gpu.sepFilter2D(img, kx, ky, gpu.BorderMode(b))
            want = orc.sep_filter(img, kx, ky, border=b, out_dtype=np.float64)
            d = np.abs(got.astype(np.float64) - want)
            print(f"\nsep f32 L={L} border={b}: max |err| vs FP64 {d.max():.3e}, mean {d.mean():.3e}")
            assert d.max() <= 1e-5, d.max()


def test_generic_separable_path(gpu):
    """The generic separable kernels (taken for shapes the fast kernel does not
    cover) against every separable golden case, forced for all cases."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, IPFC_SEP_PATH="generic")
    r = subprocess.run([sys.executable, os.path.join(here, "sep_generic_check.py")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "separable cases ok (generic path)" in r.stdout


def test_tcol_separable_path(gpu):
    """The kernel with the column pass on tcgen05 and the row pass out of
    tensor memory (sep_tcol.cu), forced for every uint8 separable call it
    covers: every separable golden case, the full-size uint8 Gaussians and a
    sweep of awkward shapes, channels, tap signs and borders."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, IPFC_SEP_PATH="tcol")
    r = subprocess.run([sys.executable, os.path.join(here, "sep_generic_check.py"), "--fullsize", "--sweep"],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "separable cases ok (tcol path)" in r.stdout and "3840x2160x3 ok" in r.stdout
    assert "sweep cases ok" in r.stdout
    print(r.stdout)


def test_cuda_core_separable_path_at_full_size(gpu):
    """The CUDA-core fast kernel, which large uint8 images leave for the
    tensor-core kernel by default, kept on for every call (IPFC_SEP_PATH=fast):
    the golden cases and the full-size uint8 Gaussians."""
    import os
    import subprocess
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, IPFC_SEP_PATH="fast")
    r = subprocess.run([sys.executable, os.path.join(here, "sep_generic_check.py"), "--fullsize"], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "separable cases ok (fast path)" in r.stdout and "3840x2160x3 ok" in r.stdout


@pytest.mark.parametrize("c", [1, 3, 4])
@pytest.mark.parametrize("w", [1200, 1201])
def test_medium_all_borders_u8(gpu, orc, c, w):
    """Images wide enough for interior strips: aligned rows (w*c a multiple
    of 4, one word load per lane) and unaligned rows (border-lane word
    copies), every border, host arrays and device tensors, against the
    restatement within 1 LSB."""
    import torch

    img = oracle.random_image(w, 157, c, np.uint8, 7 * c + w)
    dev = torch.from_numpy(img).cuda()
    for b in oracle.BORDERS:
        for sigma in (0.8, 2.0, 3.7):
            want = orc.gaussian_blur(img, sigma, 0.0, 0, b)
            got = gpu.gaussianBlur(img, sigma, border=gpu.BorderMode(b))
            G.compare(got, want, ("lsb", 1, 0.0))
            got_d = gpu.gaussianBlur(dev, sigma, border=gpu.BorderMode(b)).cpu().numpy()
            G.compare(got_d, want, ("lsb", 1, 0.0))
    from imageprocessingflex_b200 import _lib

    assert _lib.load().ipfc_check_device(None) == 0


@pytest.mark.parametrize("c,dt", [(1, np.uint8), (3, np.uint8), (4, np.uint8), (1, np.float32)],
                         ids=["u8c1", "u8c3", "u8c4", "f32c1"])
def test_sep_border_lanes_every_row_residue(gpu, orc, c, dt):
    """The fast separable kernel's load plan: lanes whose samples are border
    mapped or straddle the row end assemble them from up to three aligned
    words; unaligned sources load sample by sample.  Widths with every row
    length mod 4, one strip and several, every border, host arrays (pitch
    padded to 128 B), contiguous device tensors (pitch = row length) and a
    view one pixel in (unaligned base).  Integer taps make the u8 bar exact."""
    import torch

    B = gpu.BorderMode
    rng = np.random.default_rng(11 * c + (dt == np.float32))
    widths = [1, 2, 3, 5, 6, 7, 8, 9, 30, 31, 33, 34, 313, 314, 315, 316, 629, 630, 631, 633, 1001, 1002]
    ks = (5, 13, 17) if dt == np.float32 else (5, 13, 25)
    for w in widths:
        img = oracle.random_image(w + 1, 23, c, dt, 1000 * c + w)
        host = np.ascontiguousarray(img[:, 1:])
        dev = torch.from_numpy(host).cuda()
        view = torch.from_numpy(img).cuda()[:, 1:]
        for k in ks:
            kx = rng.integers(-3, 4, size=k).astype(np.float64)
            ky = rng.integers(-3, 4, size=k).astype(np.float64)
            for b in oracle.BORDERS:
                want = orc.sep_filter(host, kx, ky, border=b, delta=0.0, border_value=2.0)
                tol = G.tolerance("sep", {"border_value": 2.0, "delta": 0.0}, {"src": host, "kx": kx, "ky": ky}, want)
                G.compare(gpu.sepFilter2D(host, kx, ky, B(b), 0.0, 2.0), want, tol)
                G.compare(gpu.sepFilter2D(dev, kx, ky, B(b), 0.0, 2.0).cpu().numpy(), want, tol)
                G.compare(gpu.sepFilter2D(view, kx, ky, B(b), 0.0, 2.0).cpu().numpy(), want, tol)


def test_threaded_host_calls_match_single_thread(gpu):
    """Host-image calls from several threads, each on its own stream (the
    overlapped form a streaming caller uses), give the single-thread results
    for every op; each call returns with its result in host memory."""
    import threading

    import torch

    imgs = [oracle.random_image(300 + 37 * i, 200 + 11 * i, (1, 3, 4)[i % 3], np.uint8, 4242 + i) for i in range(8)]
    se = gpu.getStructuringElement(gpu.MorphShape.Rect, 3)
    ops = [lambda im, s: gpu.gaussianBlur(im, 2.0, stream=s),
           lambda im, s: gpu.gaussianBlur(im, 3.7, border=gpu.BorderMode.Wrap, stream=s),
           lambda im, s: gpu.medianBlur(im, 5, stream=s),
           lambda im, s: gpu.erode(im, se, stream=s),
           lambda im, s: gpu.boxFilter(im, 5, 5, stream=s)]
    want = [[op(im, None) for op in ops] for im in imgs]
    got = [[None] * len(ops) for _ in imgs]
    errors = []

    def worker(k):
        try:
            st = torch.cuda.Stream()
            for rep in range(3):
                for i in range(k, len(imgs), 4):
                    for j, op in enumerate(ops):
                        got[i][j] = op(imgs[i], st)
        except Exception as e:  # reported below, on the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i in range(len(imgs)):
        for j in range(len(ops)):
            np.testing.assert_array_equal(got[i][j], want[i][j], err_msg=f"image {i} op {j}")
