"""Replays the separable golden cases (gaussian, sep, sobel) through the CUDA
library and exits non-zero on any parity failure.  Run by
test_gpu_parity.test_generic_separable_path with IPFC_SEP_PATH=generic (the
generic fused / two-pass kernels), by test_tcol_separable_path with
IPFC_SEP_PATH=tcol (the tensor-core column-pass kernel) and by
test_cuda_core_separable_path_at_full_size with IPFC_SEP_PATH=fast (the
CUDA-core kernel), so each kernel is checked whichever the default picks.  With --fullsize it also checks
gaussianBlur sigma=2 on 1920x1080x3 and 3840x2160x3 uint8 within 1 LSB.
With --sweep it also runs uint8 sepFilter2D over awkward shapes (1x1,
widths and heights that are no multiple of the kernels' tiles), 1, 3 and 4
channels, every odd tap count from 3 to 15 (non-negative and signed), every border (Constant
with an integer border value) against the oracle within 1 LSB."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import golden_cases as G  # noqa: E402
import imageprocessingflex_b200 as ipf  # noqa: E402


def main():
    n = 0
    for i in range(len(G.case_ids())):
        op, p, x, want = G.case(i)
        if op not in ("gaussian", "sep", "sobel"):
            continue
        got = G.run_gpu(ipf, op, p, x)
        G.compare(got, want, G.tolerance(op, p, x, want))
        n += 1
    print(f"{n} separable cases ok ({os.environ.get('IPFC_SEP_PATH', 'auto')} path)")
    if "--fullsize" in sys.argv:
        import numpy as np

        import oracle

        orc = oracle.restatement()
        for w, h in ((1920, 1080), (3840, 2160)):
            img = oracle.random_image(w, h, 3, np.uint8, 1)
            d = np.abs(ipf.gaussianBlur(img, 2.0).astype(np.int32) - orc.gaussian_blur(img, 2.0).astype(np.int32))
            rate = float((d > 0).mean())
            if d.max() > 1 or rate >= 1e-4:
                raise SystemExit(f"gaussian {w}x{h}x3: max {d.max()}, mismatch rate {rate:.3e}")
            print(f"gaussian {w}x{h}x3 ok: mismatch rate {rate:.3e}")


def sweep():
    import numpy as np

    import oracle

    orc = oracle.restatement()
    rng = np.random.default_rng(2027)
    shapes = [(1, 1), (7, 3), (129, 130), (300, 257), (1000, 131), (43, 600)]
    n = 0
    for c in (1, 3, 4):
        for w, h in shapes:
            img = oracle.random_image(w, h, c, np.uint8, 31 * w + h + c)
            for k in (3, 5, 7, 9, 11, 13, 15):
                if c * (k // 2) > 32:
                    continue
                for signed in (False, True):
                    kx = rng.random(k) + (-0.3 if signed else 0.0)
                    ky = rng.random(k) + (-0.3 if signed else 0.0)
                    if signed:  # keep the sums well away from 0 before normalising
                        kx[k // 2] += 2.0
                        ky[k // 2] += 2.0
                    kx /= kx.sum()
                    ky /= ky.sum()
                    for b in oracle.BORDERS:
                        bv = 37.0 if b == oracle.CONSTANT else 0.0
                        want = orc.sep_filter(img, kx, ky, border=b, delta=0.25, border_value=bv)
                        got = ipf.sepFilter2D(img, kx, ky, ipf.BorderMode(b), 0.25, bv)
                        d = np.abs(got.astype(np.int32) - want.astype(np.int32))
                        if d.max(initial=0) > 1:
                            raise SystemExit(f"sweep {w}x{h}x{c} k{k} signed={signed} border {b}: max {d.max()}")
                        n += 1
    print(f"{n} sweep cases ok")


if __name__ == "__main__":
    main()
    if "--sweep" in sys.argv:
        sweep()
