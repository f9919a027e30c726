"""The batched form (ipfc_batch_*): separable group launches and persistent
tile-queue kernels over many uneven uint8 images, replayed as a CUDA graph.

The tile bodies are the per-image kernels' own code, so every batched image
must equal its per-image call bit for bit; the per-image calls are held to
the oracle by test_gpu_parity.py, and a sample of batched results is checked
against the oracle here as well (uint8 Gaussian within 1 LSB, median and
morphology exact).
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
import oracle
from imageprocessingflex_b200 import batch as B
from imageprocessingflex_b200 import mix

pytestmark = pytest.mark.gpu


def _tensor(w, h, c, seed):
    import torch

    shape = (h, w, c) if c > 1 else (h, w)
    t = torch.empty(shape, dtype=torch.uint8, device="cuda")
    if t.numel():
        mix.fill_uniform_u8(t, seed)
    return t


def _add(b, it, s, d):
    if it.op == "gaussian":
        b.add_gaussianBlur(s, d, it.sigma)
    elif it.op == "median":
        b.add_medianBlur(s, d, it.ksize)
    elif it.op == "erode":
        b.add_erode(s, d)
    else:
        b.add_dilate(s, d)


def _single(it, s):
    if it.op == "gaussian":
        return ipf.gaussianBlur(s, it.sigma)
    if it.op == "median":
        return ipf.medianBlur(s, it.ksize)
    if it.op == "erode":
        return ipf.erode(s)
    return ipf.dilate(s)


def _build(items, **kw):
    import torch

    b = B.Batch(**kw)
    srcs, dsts = [], []
    for it in items:
        s = _tensor(it.width, it.height, it.channels, it.seed)
        d = torch.zeros_like(s)
        _add(b, it, s, d)
        srcs.append(s)
        dsts.append(d)
    return b, srcs, dsts


def _assert_same(items, srcs, dsts):
    import torch

    torch.cuda.synchronize()
    for i, (it, s, d) in enumerate(zip(items, srcs, dsts)):
        want = _single(it, s)
        assert torch.equal(d, want), (i, it)


def test_uneven_mix_matches_per_image(gpu):
    import torch

    items = mix.uneven_mix(n=96, seed=7, lo=1, hi=420)
    b, srcs, dsts = _build(items)
    b.run()
    _assert_same(items, srcs, dsts)
    assert b.info("graph") == 1 and b.info("planned") == 1
    classes = [b.info(k) for k in ("tiles_light", "tiles_heavy", "tiles_mem")]
    assert b.info("kernels") >= sum(n > 0 for n in classes)  # separable items: one launch per (taps, channels)
    assert classes[2] > 0  # the mix holds 3x3 / 5x5 medians and morphology
    assert b.info("grid_mem") > 0
    # replay on new pixels written into the same buffers
    for it, s in zip(items, srcs):
        if s.numel():
            mix.fill_uniform_u8(s, it.seed + 1000)
    for d in dsts:
        d.zero_()
    b.run()
    _assert_same(items, srcs, dsts)
    torch.cuda.synchronize()
    b.close()


def test_direct_launch_and_default_tiles_agree(gpu):
    import torch

    items = mix.uneven_mix(n=24, seed=11, lo=30, hi=700)
    b1, srcs, d1 = _build(items, autotune=False, graph=False)
    b1.run()
    assert b1.info("graph") == 0
    b2 = B.Batch()
    d2 = []
    for it, s in zip(items, srcs):
        d = torch.zeros_like(s)
        _add(b2, it, s, d)
        d2.append(d)
    b2.run()
    torch.cuda.synchronize()
    for x, y in zip(d1, d2):
        assert torch.equal(x, y)
    _assert_same(items, srcs, d1)


EDGE = [(1, 1, 1), (1, 7, 3), (9, 1, 1), (2, 3, 4), (3, 2, 3), (17, 5, 3), (130, 33, 1), (257, 70, 3), (5, 600, 4),
        (0, 5, 1), (4, 0, 3)]


def test_edge_shapes_every_op_and_border(gpu):
    import torch

    rng = np.random.default_rng(3)
    b = B.Batch()
    jobs = []
    seed = 100
    for (w, h, c) in EDGE:
        for border in range(5):
            for k in (3, 5, 9, 13, 15, 21, 25):
                seed += 1
                s = _tensor(w, h, c, seed)
                d = torch.zeros_like(s)
                if border == 0 or k in (9, 21):
                    kx = rng.normal(size=k)
                    ky = rng.normal(size=k)
                    delta, bv = float(rng.normal() * 3), float(rng.uniform(-20, 300))
                    b.add_sepFilter2D(s, d, kx, ky, ipf.BorderMode(border), delta, bv)
                    jobs.append((d, lambda s=s, kx=kx, ky=ky, bo=border, de=delta, bv=bv:
                                 ipf.sepFilter2D(s, kx, ky, ipf.BorderMode(bo), de, bv)))
                else:
                    sigma = float(rng.uniform(0.3, 4.5))
                    b.add_gaussianBlur(s, d, sigma, 0.0, k, ipf.BorderMode(border))
                    jobs.append((d, lambda s=s, sg=sigma, k=k, bo=border:
                                 ipf.gaussianBlur(s, sg, 0.0, k, ipf.BorderMode(bo))))
            if border != 0:
                for k in (3, 5, 7):
                    seed += 1
                    s = _tensor(w, h, c, seed)
                    d = torch.zeros_like(s)
                    b.add_medianBlur(s, d, k, ipf.BorderMode(border))
                    jobs.append((d, lambda s=s, k=k, bo=border: ipf.medianBlur(s, k, ipf.BorderMode(bo))))
        for sw, sh in ((3, 3), (1, 5), (7, 2)):
            se = np.ones((sh, sw), np.uint8)
            for erode in (True, False):
                seed += 1
                s = _tensor(w, h, c, seed)
                d = torch.zeros_like(s)
                (b.add_erode if erode else b.add_dilate)(s, d, se)
                jobs.append((d, lambda s=s, se=se, e=erode: (ipf.erode if e else ipf.dilate)(s, se)))
    b.run()
    torch.cuda.synchronize()
    for i, (d, single) in enumerate(jobs):
        assert torch.equal(d, single()), i


def test_batched_results_vs_oracle(gpu, orc):
    items = mix.uneven_mix(n=16, seed=5, lo=40, hi=300)
    b, srcs, dsts = _build(items)
    b.run()
    import torch

    torch.cuda.synchronize()
    for it, s, d in zip(items, srcs, dsts):
        x = s.cpu().numpy()
        got = d.cpu().numpy()
        if it.op == "gaussian":
            want = orc.gaussian_blur(x, it.sigma)
            assert np.abs(got.astype(int) - want.astype(int)).max(initial=0) <= 1
        elif it.op == "median":
            np.testing.assert_array_equal(got, orc.median_blur(x, it.ksize, oracle.REPLICATE))
        else:
            se = orc.structuring_element(0, 3, 3)
            want = orc.erode(x, se) if it.op == "erode" else orc.dilate(x, se)
            np.testing.assert_array_equal(got, want)


def test_autotuner_records_its_keys(gpu):
    B.tune_clear()
    items = [mix.MixItem(700, 500, 3, "gaussian", sigma=2.0, seed=1), mix.MixItem(300, 200, 1, "median", ksize=5, seed=2)]
    b, srcs, dsts = _build(items)
    b.run()
    a = B.tune_get(B.OP_SEP, 13, 3, 1)
    assert a is not None and a[0] in (26, 52, 104, 208)
    m = B.tune_get(B.OP_MEDIAN, 5, 1, 0)
    assert m in ((128, 16), (128, 32), (256, 16), (256, 32), (256, 64))
    _assert_same(items, srcs, dsts)


def test_unsupported_items_are_rejected(gpu):
    import torch

    b = B.Batch()
    f = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    u = torch.zeros((8, 8), dtype=torch.uint8, device="cuda")
    u2 = torch.zeros((8, 8, 2), dtype=torch.uint8, device="cuda")
    with pytest.raises(ipf.Error, match="uint8"):
        b.add_gaussianBlur(f, torch.zeros_like(f), 1.0)
    with pytest.raises(ipf.Error, match="1, 3 or 4 channels"):
        b.add_gaussianBlur(u2, torch.zeros_like(u2), 1.0)
    with pytest.raises(ipf.Error, match="tap counts"):
        b.add_gaussianBlur(u, torch.zeros_like(u), 5.0)  # 31 taps
    with pytest.raises(ipf.Error, match="all-ones"):
        b.add_erode(u, torch.zeros_like(u), ipf.getStructuringElement(ipf.MorphShape.Cross, 3))
    with pytest.raises(ipf.Error, match="one iteration"):
        b.add_dilate(u, torch.zeros_like(u), None, 2)
    with pytest.raises(ipf.Error, match="ksize must be odd"):
        b.add_medianBlur(u, torch.zeros_like(u), 4)
    assert b.info("items") == 0
