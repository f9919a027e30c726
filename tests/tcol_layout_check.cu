// Host check of the tensor-core separable kernel's shared-memory operands
// (csrc/sep_tcol.cuh, compiled here for the host from the same source).
//
// The kernel writes A (banded vertical taps, K-major) and B (converted
// source rows, MN-major) with tcol_a_off / tcol_b_off and hands the tensor
// cores descriptors built by tcol_desc_a / tcol_desc_b / tcol_idesc.  This
// program fills a shared-memory image with the kernel's own writers, then
// emulates every MMA of a slab step from the descriptor and instruction
// descriptor bits alone, reading operands through the canonical no-swizzle
// layouts as the PTX ISA and CUTLASS define them:
//   K-major:  (row r, k) at start + (r/8) SBO + (k/8) LBO + (r%8) 16 + (k%8) 2
//   MN-major: (col n, k) at start + (n/8) SBO + (k/8) LBO + (k%8) 16 + (n%8) 2
// It checks that every read stays inside its operand, that the instruction
// descriptor says M = 128, the step's N, FP16 in, FP32 out, A K-major and B
// MN-major, and that the emulated D equals the direct column correlation
// sum_j (hi_j + lo_j) B[n][m + j] for every (m, n), for slab and halo steps
// and every K the kernel is built for.  It also walks TcolWalk for many
// (units, CTAs, slabs per band) and checks that every unit is a slab step
// exactly once, bracketed by halo steps of its own band, and that the
// host's cost-balanced split of the units (tcol_split_units) is contiguous,
// never empty and within two edge units of the average cost.
//
// Prints "ok <cases>" and exits 0, or the first failures and exits 1.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#include "sep_tcol.cuh"

using namespace ipfc;

static long long bad = 0, cases = 0;

static void fail(const char* what, int a, int b, int c) {
    if (bad++ < 10) std::printf("FAIL %s (%d, %d, %d)\n", what, a, b, c);
}

static void check_k(int K, std::mt19937& rng) {
    const int KR = tcol_kr(K), KG = KR / 8;
    const int ob = tcol_operand_bytes(K);
    std::vector<uint16_t> sm((size_t)tcol_smem(K) / 2, 0);
    std::vector<char> written(sm.size(), 0);  // a read of an element no writer stored fails
    auto at = [&](int byte) -> uint16_t& { return sm[(size_t)byte / 2]; };
    auto put = [&](int byte, int v) {
        sm[(size_t)byte / 2] = (uint16_t)(int16_t)v;
        written[(size_t)byte / 2] = 1;
    };
    // taps: small integers (exact in every form) as "hi", a few as "lo"
    std::vector<int> hi(K), lo(K);
    for (int j = 0; j < K; ++j) {
        hi[j] = (int)(rng() % 61) - 30;
        lo[j] = (int)(rng() % 7) - 3;
    }
    // A writer: the kernel's loop (one 16-byte core-matrix row per item)
    for (int it = 0; it < 2 * kTcolM * KG; ++it) {
        const int hl = it / (kTcolM * KG), rest = it % (kTcolM * KG);
        const int m = rest % kTcolM, kg = rest / kTcolM;
        for (int e = 0; e < 8; ++e) {
            const int j = 8 * kg + e - m;
            const int v = (j >= 0 && j < K) ? (hl ? lo[j] : hi[j]) : 0;
            const int off = tcol_off_a(hl, K) + tcol_a_off(m, 8 * kg + e);
            if (off < tcol_off_a(hl, K) || off + 2 > tcol_off_a(hl, K) + ob) fail("A write outside", hl, m, kg);
            put(off, v);
        }
    }
    // B writer: producers' stores (16-sample chunk of one row as two 16-byte runs)
    std::vector<int> src((size_t)kTcolN * KR);
    for (auto& x : src) x = (int)(rng() % 256) - 128;
    const int bb = 1;
    for (int kg = 0; kg < KG; ++kg)
        for (int half = 0; half < 2; ++half)
            for (int lane = 0; lane < 32; ++lane) {
                const int r8 = lane & 7, c4 = lane >> 3, n = 64 * half + 16 * c4, k = 8 * kg + r8;
                for (int part = 0; part < 2; ++part)
                    for (int e = 0; e < 8; ++e) {
                        const int nn = n + 8 * part + e;
                        const int off = tcol_off_b(bb, K) + tcol_b_off(n + 8 * part, k) + 2 * e;
                        if (off < tcol_off_b(bb, K) || off + 2 > tcol_off_b(bb, K) + ob) fail("B write outside", n, k, e);
                        put(off, src[(size_t)nn * KR + k]);
                    }
            }
    // emulate: halo steps (N = 16 GH at the slab's edges) and the full step
    for (int GH = 1; GH <= 2; ++GH) {
        const int steps[3][2] = {{kTcolN - 16 * GH, 16 * GH}, {0, kTcolN}, {0, 16 * GH}};
        for (auto& stp : steps) {
            const int n0 = stp[0], nn = stp[1];
            const uint32_t idesc = tcol_idesc(nn);
            const int c_fmt = (idesc >> 4) & 3, a_fmt = (idesc >> 7) & 7, b_fmt = (idesc >> 10) & 7;
            const int a_major = (idesc >> 15) & 1, b_major = (idesc >> 16) & 1;
            const int N = (int)((idesc >> 17) & 63) * 8, M = (int)((idesc >> 24) & 31) * 16;
            if (c_fmt != 1 || a_fmt != 0 || b_fmt != 0 || a_major != 0 || b_major != 1 || N != nn || M != kTcolM)
                fail("instruction descriptor", nn, M, N);
            std::vector<long long> D((size_t)kTcolM * nn, 0);
            for (int ks = 0; ks < KR / 16; ++ks)
                for (int hl = 0; hl < 2; ++hl) {
                    const uint64_t ad = tcol_desc_a((uint32_t)tcol_off_a(hl, K), ks);
                    const uint64_t bd = tcol_desc_b((uint32_t)tcol_off_b(bb, K), ks, n0);
                    auto dec = [](uint64_t d, int& start, int& lbo, int& sbo, int& ver, int& lay) {
                        start = (int)(d & 0x3fff) << 4;
                        lbo = (int)((d >> 16) & 0x3fff) << 4;
                        sbo = (int)((d >> 32) & 0x3fff) << 4;
                        ver = (int)((d >> 46) & 3);
                        lay = (int)((d >> 61) & 7);
                    };
                    int as, al, asb, av, alay, bs, bl, bsb, bv, blay;
                    dec(ad, as, al, asb, av, alay);
                    dec(bd, bs, bl, bsb, bv, blay);
                    if (av != 1 || bv != 1 || alay != 0 || blay != 0) fail("descriptor version/layout", ks, av, bv);
                    for (int m = 0; m < M; ++m)
                        for (int n = 0; n < N; ++n)
                            for (int kk = 0; kk < 16; ++kk) {
                                const int aoff = as + (m / 8) * asb + (kk / 8) * al + (m % 8) * 16 + (kk % 8) * 2;
                                const int boff = bs + (n / 8) * bsb + (kk / 8) * bl + (kk % 8) * 16 + (n % 8) * 2;
                                if (aoff < tcol_off_a(hl, K) || aoff + 2 > tcol_off_a(hl, K) + ob) {
                                    fail("A read outside", m, kk, ks);
                                    continue;
                                }
                                if (boff < tcol_off_b(bb, K) || boff + 2 > tcol_off_b(bb, K) + ob) {
                                    fail("B read outside", n, kk, ks);
                                    continue;
                                }
                                if (!written[(size_t)aoff / 2] || !written[(size_t)boff / 2]) {
                                    fail("read of an unwritten element", m, n, kk);
                                    continue;
                                }
                                const int16_t av2 = (int16_t)at(aoff), bv2 = (int16_t)at(boff);
                                D[(size_t)m * nn + n] += (long long)av2 * bv2;
                            }
                }
            for (int m = 0; m < M; ++m)
                for (int n = 0; n < N; ++n) {
                    long long want = 0;
                    for (int j = 0; j < K; ++j)
                        if (m + j < KR) want += (long long)(hi[j] + lo[j]) * src[(size_t)(n0 + n) * KR + m + j];
                    ++cases;
                    if (D[(size_t)m * nn + n] != want) fail("D mismatch", m, n, K);
                }
        }
    }
}

// The host's bottleneck unit split: contiguous, every range non-empty,
// range costs as tcol_range_cost sums them, and no range costing more than
// the mean plus one costliest unit (the split's granularity).
static void check_split(std::mt19937& rng) {
    for (int t = 0; t < 3000; ++t) {
        const int nb = 1 + (int)(rng() % 40), ns = 1 + (int)(rng() % 120);
        const int units = nb * ns;
        const int grid = 1 + (int)(rng() % std::min(units, 160));
        std::vector<int> split(grid + 1, -1);
        tcol_split_units(units, ns, grid, split.data());
        if (split[0] != 0 || split[grid] != units) fail("split ends", split[0], split[grid], units);
        double total = 0, worst = 0;
        for (int b = 0; b < grid; ++b) {
            if (split[b + 1] <= split[b]) fail("empty or reversed range", b, split[b], split[b + 1]);
            // the range cost against a unit-by-unit sum
            double c = 2 * kTcolHaloCost;
            for (int u = split[b]; u < split[b + 1]; ++u) {
                c += 1.0;
                if (u % ns == ns - 1) c += kTcolRightEdgeCost;
                if (u % ns == 0) c += kTcolLeftEdgeCost + (u == split[b] ? 0.0 : kTcolBandCrossCost);
            }
            if (std::fabs(c - tcol_range_cost(split[b], split[b + 1], ns)) > 1e-9) fail("range cost", b, split[b], split[b + 1]);
            total += c;
            worst = std::max(worst, c);
        }
        ++cases;
        // the bottleneck stays within one costliest unit of the mean
        if (worst > total / grid + 1.0 + kTcolLeftEdgeCost + kTcolRightEdgeCost + 1e-9)
            fail("unbalanced split", units, grid, (int)worst);
    }
}

static void check_walk(std::mt19937& rng) {
    for (int t = 0; t < 3000; ++t) {
        const int nb = 1 + (int)(rng() % 20), ns = 1 + (int)(rng() % 100);
        const int units = nb * ns;
        const int grid = 1 + (int)(rng() % (units + 5));
        std::vector<int> seen(units, 0);
        for (int b = 0; b < grid && b < units; ++b) {
            const int u0 = (int)((long long)b * units / std::min(grid, units));
            const int u1 = (int)((long long)(b + 1) * units / std::min(grid, units));
            TcolWalk w(u0, u1, ns);
            TcolStep st;
            int state = 0, band = -1, last = -2;  // state: 0 expect left halo, 1 inside a run
            while (w.next(st)) {
                ++cases;
                if (st.kind == 0) {
                    if (state != 0) fail("left halo inside a run", b, st.band, st.slab);
                    state = 1;
                    band = st.band;
                    last = st.slab;
                } else if (st.kind == 1) {
                    if (state != 1 || st.band != band || st.slab != last + 1) fail("slab order", b, st.band, st.slab);
                    if (st.slab < 0 || st.slab >= ns) fail("slab out of range", b, st.band, st.slab);
                    else seen[st.band * ns + st.slab]++;
                    last = st.slab;
                } else {
                    if (state != 1 || st.band != band || st.slab != last + 1) fail("right halo", b, st.band, st.slab);
                    state = 0;
                }
            }
            if (state != 0) fail("run not closed", b, u0, u1);
        }
        for (int u = 0; u < units; ++u)
            if (seen[u] != 1) fail("unit coverage", u, seen[u], units);
    }
}

int main() {
    std::mt19937 rng(12345);
    for (int K : {3, 5, 7, 9, 11, 13, 15, 17, 21, 25, 31}) check_k(K, rng);
    check_split(rng);
    check_walk(rng);
    if (bad) {
        std::printf("%lld failures\n", bad);
        return 1;
    }
    std::printf("ok %lld\n", cases);
    return 0;
}
