"""Dense filter2D at the measured 4096 x 4096 x 1 configuration, both forms
(FP32 CUDA cores and split-precision tcgen05), against the oracle.

Configuration: 4096 x 4096 x 1 images, uint8 (seeded uniform 0-255) and
float (seeded uniform [0, 1)), Reflect101, dense taps drawn N(0, 1) and
normalised to sum 1 -- ``mix.filter2d_taps(k, seed=1000 + k)``, which redraws
until |sum| > 0.25 k so the normalisation cannot blow the taps up -- at 15 x 15
and 31 x 31 (include/ipf/filter.hpp:159-194).

The whole image is filtered on the GPU; the oracle (filter2D restated in
FP64, row-band form) checks three full-width bands of 256 rows: the top and
bottom ones, which hold every vertical border case, and one in the middle.
Bars:
  * uint8 output: within 1 LSB of filter2D<uint8_t>, with the mismatch rate
    and the saturated fraction printed;
  * float output: within the suite's filter2D bar of filter2D<float>;
  * error against filter2D<double> (FP64): the split form's maximum and mean
    no larger than the FP32 form's, both printed.
"""
import numpy as np
import pytest

import golden_cases as G
import imageprocessingflex_b200 as ipf
import oracle
from imageprocessingflex_b200 import mix

pytestmark = pytest.mark.gpu

N = 4096
BANDS = ((0, 256), (N // 2 - 128, N // 2 + 128), (N - 256, N))


def _image(dt):
    return oracle.random_image(N, N, 1, dt, 4096 if dt == np.uint8 else 4097)


@pytest.mark.parametrize("kk", [15, 31])
@pytest.mark.parametrize("dt", [np.uint8, np.float32], ids=["u8", "f32"])
def test_filter2d_4096_both_forms_vs_oracle(gpu, orc, dt, kk):
    import torch

    img = _image(dt)
    k = mix.filter2d_taps(kk, seed=1000 + kk)
    dev = torch.from_numpy(img).cuda()
    out = {}
    for form in ("split", "fp32"):
        out[form] = ipf.filter2D(dev, k, form=form).cpu().numpy()
        out[form + "_f"] = ipf.filter2D(dev, k, form=form, dtype=torch.float32).cpu().numpy().astype(np.float64)
    err = {"split": [], "fp32": []}
    mism = {"split": 0, "fp32": 0}
    total = 0
    sat = 0
    for y0, y1 in BANDS:
        want = orc.filter2d_rows(img, k, y0, y1)
        ref64 = orc.filter2d_rows(img, k, y0, y1, out_dtype=np.float64)
        total += want.size
        for form in ("split", "fp32"):
            got = out[form][y0:y1]
            if dt == np.uint8:
                d = np.abs(got.astype(np.int64) - want.astype(np.int64))
                assert d.max() <= 1, (form, kk, y0, d.max())
                mism[form] += int((d > 0).sum())
            else:
                G.compare(got, want, G.tolerance("filter2d", {"delta": 0.0, "border_value": 0.0},
                                                 {"src": img, "kernel": k}, want))
            err[form].append(np.abs(out[form + "_f"][y0:y1] - ref64))
        if dt == np.uint8:
            sat += int(((want == 0) | (want == 255)).sum())
    e = {f: np.concatenate([x.ravel() for x in v]) for f, v in err.items()}
    name = f"{np.dtype(dt).name} {kk}x{kk} 4096^2"
    print(f"\n{name}: |err| vs FP64  split max {e['split'].max():.3e} mean {e['split'].mean():.3e}; "
          f"fp32 max {e['fp32'].max():.3e} mean {e['fp32'].mean():.3e}")
    if dt == np.uint8:
        print(f"{name}: mismatch rate vs filter2D<uint8_t> split {mism['split'] / total:.3e} fp32 "
              f"{mism['fp32'] / total:.3e}; saturated fraction {sat / total:.4f}")
    assert e["split"].max() <= e["fp32"].max() + 1e-12
    assert e["split"].mean() <= e["fp32"].mean() + 1e-12
