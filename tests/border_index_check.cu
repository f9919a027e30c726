// Host check of the kernels' border rule (border_index in common.cuh,
// compiled here for the host from the same source) against the oracle's
// restatement of ipf's borderIndex (orc_border_index, after
// include/ipf/core.hpp:187-214), for all five modes:
//
//  * every row length 1..256 and every position from -4n - 40 to 5n + 40;
//  * sampled lengths up to the C ABI's limit (2^30 - 1 samples per row),
//    with positions around both row ends and a full kernel halo away;
//  * the interleaved form the tile loaders use (border_sample: sample
//    index x*C + c to its source sample, channel kept) for C = 1..4, every
//    row length 1..128 and every sample from a few rows left to a few rows
//    right of the row.
//
// Prints "ok <cases checked>" and exits 0, or prints the first failures and
// exits 1.
#include <cstdio>
#include <random>

#include "common.cuh"

extern "C" int orc_border_index(int p, int len, int mode);

int main() {
    long long bad = 0, checked = 0;
    auto check = [&](int p, int n, int mode) {
        const int got = ipfc::border_index(p, n, mode), want = orc_border_index(p, n, mode);
        ++checked;
        if (got != want && bad++ < 5) std::printf("mode %d n %d p %d: %d, oracle %d\n", mode, n, p, got, want);
    };
    for (int mode = 0; mode < 5; ++mode) {
        for (int n = 1; n <= 256; ++n)
            for (int p = -4 * n - 40; p <= 5 * n + 40; ++p) check(p, n, mode);
        std::mt19937 rng(7 + mode);
        for (int t = 0; t < 20000; ++t) {
            const int n = (int)(rng() % ((1u << 30) - 1)) + 1;
            for (int d = -70; d <= 70; ++d) {
                check(d, n, mode);
                check(n - 1 + d, n, mode);
            }
        }
        for (int n : {(1 << 30) - 1, (1 << 30) - 2, 1 << 29}) {
            for (int d = -300; d <= 300; ++d) {
                check(d, n, mode);
                check(n - 1 + d, n, mode);
                check(-n + d, n, mode);
            }
        }
    }
    for (int mode = 0; mode < 5; ++mode)
        for (int C = 1; C <= 4; ++C)
            for (int w = 1; w <= 128; ++w)
                for (int s = -(4 * w + 10) * C; s < (5 * w + 10) * C; ++s) {
                    const int x = s >= 0 ? s / C : -((-s + C - 1) / C), c = s - x * C;
                    const int sx = orc_border_index(x, w, mode);
                    const int want = sx < 0 ? -1 : sx * C + c, got = ipfc::border_sample(s, w, C, mode);
                    ++checked;
                    if (got != want && bad++ < 5)
                        std::printf("sample: mode %d C %d w %d s %d: %d, oracle %d\n", mode, C, w, s, got, want);
                }
    if (bad) {
        std::printf("FAILED %lld of %lld\n", bad, checked);
        return 1;
    }
    std::printf("ok %lld\n", checked);
    return 0;
}
