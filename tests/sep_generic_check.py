"""Replays the separable golden cases (gaussian, sep, sobel) through the CUDA
library and exits non-zero on any parity failure.  Run by
test_gpu_parity.test_generic_separable_path with IPFC_SEP_PATH=generic (the
generic fused / two-pass kernels) and by test_tc_separable_path with
IPFC_SEP_PATH=tc (the tensor-core column-pass kernel), so those kernels are
checked as well as the default one.  With --fullsize it also checks
gaussianBlur sigma=2 on 1920x1080x3 and 3840x2160x3 uint8 within 1 LSB."""
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


if __name__ == "__main__":
    main()
