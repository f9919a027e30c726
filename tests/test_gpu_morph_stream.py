"""erode / dilate of uint8 images by the 3 x 3 element through the
register-streaming kernel (csrc/morph3_stream.cu), which per-image calls take
when the source and destination rows start 16-byte aligned, against the
oracle: exact.

Cases: host images (staged with aligned pitches), device images with padded
aligned pitches, every channel count 1..4, row lengths on both sides of the
kernel's 16-sample chunks and 512-sample slices, heights on both sides of its
32-row bands, 1 x 1 to 4K RGB, and iterations > 1 (ping-pong through the
scratch image).  Unaligned device images take the tile kernel; both must
agree.
"""
import numpy as np
import pytest

import imageprocessingflex_b200 as ipf
import oracle

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (2, 3), (5, 31), (16, 32), (17, 33), (171, 64), (172, 65), (512, 7), (513, 40), (1000, 97)]


def _padded(img):
    """A device copy of img whose rows start 16-byte aligned with padding."""
    import torch

    h, w = img.shape[0], img.shape[1]
    c = img.shape[2] if img.ndim == 3 else 1
    pitch = (w * c + 15) // 16 * 16 + 16
    buf = torch.zeros((h, pitch), dtype=torch.uint8, device="cuda")
    buf[:, :w * c] = torch.from_numpy(np.ascontiguousarray(img).reshape(h, w * c)).cuda()
    view = buf[:, :w * c].view(h, w, c) if img.ndim == 3 else buf[:, :w]
    return view


@pytest.mark.parametrize("c", [1, 2, 3, 4])
def test_stream_erode_dilate_vs_oracle(gpu, orc, c):
    se = orc.structuring_element(0, 3)
    for w, h in SHAPES:
        img = oracle.random_image(w, h, c, np.uint8, 7 * w + h + c)
        if c == 1:
            img = img.reshape(h, w)
        for it in (1, 2):
            want_e = orc.erode(img, se, iterations=it) if it > 1 else orc.erode(img, se)
            want_d = orc.dilate(img, se, iterations=it) if it > 1 else orc.dilate(img, se)
            np.testing.assert_array_equal(ipf.erode(img, iterations=it), want_e, err_msg=f"{w}x{h}x{c} it {it}")
            np.testing.assert_array_equal(ipf.dilate(img, iterations=it), want_d, err_msg=f"{w}x{h}x{c} it {it}")
        dev = _padded(img)
        np.testing.assert_array_equal(ipf.erode(dev).cpu().numpy(), orc.erode(img, se), err_msg=f"{w}x{h}x{c} dev")
        np.testing.assert_array_equal(ipf.dilate(dev).cpu().numpy(), orc.dilate(img, se), err_msg=f"{w}x{h}x{c} dev")


def test_stream_full_size_and_unaligned_agree(gpu, orc):
    import torch

    img = oracle.random_image(3840, 2160, 3, np.uint8, 5)
    se = orc.structuring_element(0, 3)
    got = ipf.erode(img)
    np.testing.assert_array_equal(got, orc.erode(img, se))
    # a device image with an odd pitch takes the tile kernel: the same result
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    base = torch.randint(0, 256, (301, 3 * 211 + 1), generator=g, device="cuda", dtype=torch.int32).to(torch.uint8)
    odd = base[:, 1:1 + 3 * 211].view(301, 211, 3)
    want = orc.dilate(odd.cpu().numpy(), se)
    np.testing.assert_array_equal(ipf.dilate(odd).cpu().numpy(), want)
    np.testing.assert_array_equal(ipf.dilate(_padded(odd.cpu().numpy())).cpu().numpy(), want)
