// Exhaustive host check of the median selection networks that the 3x3 and
// 5x5 median kernels run, compiled here for the host from the same source:
// the packed uint8 networks (median9_2 and median25_2 in median_u8.cuh) and
// the forgetful selection of the other element types (median_forgetful in
// median.cuh, on floats).
//
// All of them are compositions of min and max only, so they commute with
// every non-decreasing map of the samples.  By the 0-1 principle a network
// that returns the sample of rank k*k/2 for every window of zeros and ones
// returns it for every window: for any threshold t, [f(x) >= t] equals
// f([x >= t]), which is [at least k*k/2 + 1 samples are >= t], which is
// [x_(k*k/2) >= t].  So the check below, over all 2^9 and 2^25 binary
// windows, proves the networks exact for every window of ordered values:
// uint8 for the packed networks; uint16, int16 and non-NaN floats (all exact
// in float) for the forgetful selection.  A sample of random byte windows
// compared with std::nth_element checks the lane packing on top.
//
// Prints "ok <windows checked>" and exits 0, or prints the first failures
// and exits 1.
#include <algorithm>
#include <cstdio>
#include <random>

#include "median.cuh"
#include "median_u8.cuh"

using ipfc::median25_2;
using ipfc::median9_2;
using ipfc::median_detail::median_forgetful;

static unsigned lanes(unsigned lo, unsigned hi) { return lo | (hi << 16); }

int main() {
    long long bad = 0, checked = 0;

    // 3x3: lane 0 holds window m, lane 1 its complement.
    for (unsigned m = 0; m < 512u; ++m) {
        unsigned v[9];
        const unsigned c = ~m & 511u;
        for (int i = 0; i < 9; ++i) v[i] = lanes((m >> i) & 1u, (c >> i) & 1u);
        const unsigned want = lanes(__builtin_popcount(m) >= 5, __builtin_popcount(c) >= 5);
        if (median9_2(v) != want && bad++ < 5) std::printf("3x3 window %03x: wrong median\n", m);
    }
    checked += 512;

    // 5x5: lane 0 holds window m (bit 24 clear), lane 1 window m | 2^24,
    // so 2^24 evaluations cover all 2^25 windows.
    long long bad5 = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad5)
    for (int m = 0; m < (1 << 24); ++m) {
        const unsigned a = (unsigned)m, b = (unsigned)m | (1u << 24);
        unsigned v[25];
        for (int i = 0; i < 25; ++i) v[i] = lanes((a >> i) & 1u, (b >> i) & 1u);
        const unsigned want = lanes(__builtin_popcount(a) >= 13, __builtin_popcount(b) >= 13);
        if (median25_2(v) != want) ++bad5;
    }
    if (bad5) std::printf("5x5: %lld binary windows with a wrong median\n", bad5);
    bad += bad5;
    checked += 1ll << 25;

    // Forgetful selection on float windows of zeros and ones.
    for (unsigned m = 0; m < 512u; ++m) {
        float v[9];
        for (int i = 0; i < 9; ++i) v[i] = (float)((m >> i) & 1u);
        if (median_forgetful<9>(v) != (float)(__builtin_popcount(m) >= 5) && bad++ < 5)
            std::printf("forgetful 3x3 window %03x: wrong median\n", m);
    }
    long long badf = 0;
#pragma omp parallel for schedule(static) reduction(+ : badf)
    for (int m = 0; m < (1 << 25); ++m) {
        float v[25];
        for (int i = 0; i < 25; ++i) v[i] = (float)(((unsigned)m >> i) & 1u);
        if (median_forgetful<25>(v) != (float)(__builtin_popcount((unsigned)m) >= 13)) ++badf;
    }
    if (badf) std::printf("forgetful 5x5: %lld binary windows with a wrong median\n", badf);
    bad += badf;
    checked += 512 + (1ll << 25);

    // Random byte windows, two per evaluation, against nth_element.
    std::mt19937 rng(12345);
    for (int t = 0; t < 200000; ++t) {
        const int k = (t & 1) ? 5 : 3, n = k * k;
        unsigned lo[25], hi[25], v[25];
        for (int i = 0; i < n; ++i) {
            lo[i] = rng() & 255u;
            hi[i] = (t & 2) ? (rng() & 3u) * 85u : rng() & 255u;  // ties in every other pair
            v[i] = lanes(lo[i], hi[i]);
        }
        unsigned got;
        if (k == 3) {
            unsigned w[9];
            std::copy(v, v + 9, w);
            got = median9_2(w);
        } else {
            got = median25_2(v);
        }
        std::nth_element(lo, lo + n / 2, lo + n);
        std::nth_element(hi, hi + n / 2, hi + n);
        if (got != lanes(lo[n / 2], hi[n / 2]) && bad++ < 5) std::printf("random %dx%d window %d: wrong median\n", k, k, t);
    }
    checked += 400000;

    if (bad) {
        std::printf("FAILED %lld\n", bad);
        return 1;
    }
    std::printf("ok %lld\n", checked);
    return 0;
}
