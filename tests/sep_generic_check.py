"""Replays the separable golden cases (gaussian, sep, sobel) through the CUDA
library and exits non-zero on any parity failure.  Run by
test_gpu_parity.test_generic_separable_path with IPFC_SEP_PATH=generic so the
generic fused / two-pass kernels are checked as well as the fast one."""
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


if __name__ == "__main__":
    main()
