// sep_tcol.cuh -- geometry of the separable kernel whose column (vertical)
// pass runs on the 5th-generation tensor cores (tcgen05) and whose row
// (horizontal) pass runs on CUDA cores straight out of tensor memory
// (sep_tcol.cu).  Shared by the kernel and a host-side layout check.
//
// For a band of 128 output rows y0 .. y0+127 and a slab of 128 interleaved
// samples x0 .. x0+127 of uint8 source S, one group of MMAs computes
//
//   D[m][n] = sum_k A[m][k] * B[n][k]                   (M = 128, N = 128)
//   A[m][k] = ky[k - m] * 2^e   for 0 <= k - m < K, else 0 (banded taps)
//   B[n][k] = S[y0 - K/2 + k][x0 + n] - 128            (rows and samples
//                                                         border-resolved)
//
// so D[m][n] = 2^e * (sum_j ky[j] S[y0 + m + j - K/2][x0 + n] - 128 sum ky):
// tensor-memory lane m holds output row m, column n holds sample n -- each
// thread of the row pass reads its own output row's column sums as
// consecutive registers and runs the horizontal taps without leaving them.
// The horizontal taps reach C*(K/2) samples either side, so the row pass of
// one slab also reads the last columns of the previous slab and the first of
// the next: four slab buffers of 128 columns live in tensor memory.
//
// Split precision: uint8 - 128 is exact in FP16; each vertical tap is split
// into hi = fp16(w 2^e) and lo = fp16(w 2^e - hi) and the MMA runs twice per
// K step (A_hi, A_lo) into the same FP32 accumulator.  Products are exact in
// FP32; centring keeps the accumulator small.
//
// Shared-memory operands, both without swizzle (8 x 16-byte core matrices):
//  * A, K-major: element (m, k) at (m/8)*128 + (k/8)*2048 + (m%8)*16 + (k%8)*2
//    -- 8-row groups 128 B apart (SBO), 8-element K groups 2048 B apart (LBO);
//  * B, MN-major: element (n, k) at (n/8)*128 + (k/8)*2048 + (k%8)*16 + (n%8)*2
//    -- 8-sample groups 128 B apart (SBO), 8-row K groups 2048 B apart (LBO);
//    a 16-byte run is 8 consecutive samples of one source row, so the
//    producers write each converted 16-sample chunk of a row as two stores.
// K step j (16 source rows) starts 2j * 2048 bytes into both operands.
#pragma once

#include <stdint.h>

namespace ipfc {

constexpr int kTcolM = 128;                   // output rows per band (MMA M)
constexpr int kTcolN = 128;                   // samples per slab (MMA N)
constexpr int kTcolMaxK = 31;
constexpr int kTcolProdWarps = 6;             // convert uint8 rows into B
constexpr int kTcolRowWarps = 12;             // row pass (3 per tensor-memory lane quarter)
// The 8 chunks of 16 columns of a slab, split 3 / 3 / 2 among the three
// row-pass warps of a lane quarter: first chunk of part p.
__host__ __device__ constexpr int tcol_row_chunk0(int p) { return p <= 0 ? 0 : p == 1 ? 3 : p == 2 ? 6 : 8; }
constexpr int kTcolThreads = 32 * (1 + kTcolProdWarps + kTcolRowWarps);
constexpr int kTcolTmemCols = 4 * kTcolN;     // four slab buffers
constexpr int kTcolKGroupBytes = 2048;        // 16 core matrices of 128 B

// Staged source rows per band (a multiple of 16: one MMA K step each).
__host__ __device__ constexpr int tcol_kr(int K) { return (kTcolM + K - 1 + 15) / 16 * 16; }
// One operand (A_hi, A_lo or one B buffer) in bytes.
__host__ __device__ constexpr int tcol_operand_bytes(int K) { return tcol_kr(K) / 8 * kTcolKGroupBytes; }
// Raw source bytes of one step as copied from the image (KR rows x 128
// samples); kTcolStages of them let the copies run two steps ahead.
constexpr int kTcolStages = 0;
__host__ __device__ constexpr int tcol_stage_bytes(int K) { return tcol_kr(K) * kTcolN; }
// Shared layout: A_hi, A_lo, B[0], B[1], the stages, then 13 mbarriers, the
// abort flag and the tensor-memory slot (128 bytes), then the FP16 taps
// (2 x 32).
__host__ __device__ constexpr int tcol_off_a(int hl, int K) { return hl * tcol_operand_bytes(K); }
__host__ __device__ constexpr int tcol_off_b(int b, int K) { return (2 + b) * tcol_operand_bytes(K); }
__host__ __device__ constexpr int tcol_off_s(int st, int K) { return 4 * tcol_operand_bytes(K) + st * tcol_stage_bytes(K); }
__host__ __device__ constexpr int tcol_off_bar(int K) { return tcol_off_s(kTcolStages, K); }
__host__ __device__ constexpr int tcol_smem(int K) { return tcol_off_bar(K) + 256; }
// Byte offset of the 16-sample chunk at sample n (a multiple of 16) of
// staged row k: chunks XOR-swizzled by the row so that the 8 rows a
// quarter-warp reads at one n fall in distinct banks.
__host__ __device__ constexpr int tcol_s_off(int k, int n) { return k * kTcolN + (((n >> 4) ^ (k & 7)) << 4); }

__host__ __device__ inline int tcol_a_off(int m, int k) {
    return (m >> 3) * 128 + (k >> 3) * kTcolKGroupBytes + (m & 7) * 16 + (k & 7) * 2;
}
__host__ __device__ inline int tcol_b_off(int n, int k) {
    return (n >> 3) * 128 + (k >> 3) * kTcolKGroupBytes + (k & 7) * 16 + (n & 7) * 2;
}

// Shared-memory matrix descriptor, no swizzle, version 1 (sm_100):
// start, leading-dimension byte offset, stride-dimension byte offset.
__host__ __device__ inline uint64_t tcol_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | ((uint64_t)1 << 46);
}
// A: K-major (LBO = K-group stride, SBO = 8-row stride).
__host__ __device__ inline uint64_t tcol_desc_a(uint32_t a_addr, int kstep) {
    return tcol_desc(a_addr + (uint32_t)(2 * kstep * kTcolKGroupBytes), kTcolKGroupBytes, 128);
}
// B: MN-major without swizzle (LBO = K-group stride, SBO = 8-sample stride),
// starting at sample n0 (a multiple of 8).
__host__ __device__ inline uint64_t tcol_desc_b(uint32_t b_addr, int kstep, int n0) {
    return tcol_desc(b_addr + (uint32_t)(2 * kstep * kTcolKGroupBytes + (n0 >> 3) * 128), kTcolKGroupBytes, 128);
}

// Instruction descriptor, kind::f16: D FP32, A and B FP16, A K-major, B
// MN-major, M = 128, N = n (a multiple of 16, 16..256).
__host__ __device__ constexpr uint32_t tcol_idesc(int n) {
    return (1u << 4) | (1u << 16) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcolM >> 4) << 24);
}

// Horizontal reach of the row pass in 16-column groups: C*(K/2) samples.
__host__ __device__ constexpr int tcol_halo_groups(int K, int C) { return (C * (K / 2) + 15) / 16; }

// The steps a CTA walks: its share of the (band, slab) units, each maximal
// run of one band bracketed by a left and a right halo step (the previous
// and next slab's edge columns, which the row pass of the run's first and
// last slab reads).  Every role of the kernel walks the same sequence.
struct TcolStep {
    int band, slab;
    int kind;  // 0 left halo, 1 slab, 2 right halo
};
struct TcolWalk {
    int u, u1, ns;
    int pending;  // 0: next is a left halo (or done), 1: next is slab u, 2: right halo after u-1
    __host__ __device__ TcolWalk(int u0, int u1_, int ns_) : u(u0), u1(u1_), ns(ns_), pending(0) {}
    __host__ __device__ bool next(TcolStep& st) {
        if (pending == 0) {
            if (u >= u1) return false;
            st = TcolStep{u / ns, u % ns - 1, 0};
            pending = 1;
            return true;
        }
        if (pending == 1) {
            st = TcolStep{u / ns, u % ns, 1};
            ++u;
            // the run ends at the walk's end or where the band changes
            pending = (u >= u1 || u % ns == 0) ? 2 : 1;
            return true;
        }
        st = TcolStep{(u - 1) / ns, (u - 1) % ns + 1, 2};
        pending = 0;
        return true;
    }
};

// Splits the (band, slab) units into `grid` contiguous ranges whose
// largest estimated cost is as small as it can be: split[b] .. split[b+1]-1
// is range b (split has grid + 1 entries); every range gets at least one
// unit (grid <= units).  The kernel's time is its slowest CTA's, so the
// split minimises the bottleneck rather than matching an average share.
// Costs are in slab steps, from per-CTA timings of 4K RGB launches: a unit
// costs one step; a range starting at a band's first slab pays the left
// image-edge halo step (border-resolved gathers), kTcolLeftEdgeCost more; a
// band's last slab pays the right one, kTcolRightEdgeCost more; a range that
// runs on into the next band pays that band's left edge with
// kTcolBandCrossCost off (the two edge steps overlap in the pipeline); and
// every range pays its own left and right halo steps.
constexpr double kTcolLeftEdgeCost = 1.9;
constexpr double kTcolRightEdgeCost = 1.3;
constexpr double kTcolBandCrossCost = -0.6;
constexpr double kTcolHaloCost = 0.3;
// Cost of units [0, u) counted as later units of a range (no range start).
inline double tcol_cost_prefix(int u, int ns) {
    return (double)u + kTcolRightEdgeCost * (double)(u / ns) +
           (kTcolLeftEdgeCost + kTcolBandCrossCost) * (double)((u + ns - 1) / ns);
}
// Estimated cost of the range of units [u0, u1), u0 < u1.
inline double tcol_range_cost(int u0, int u1, int ns) {
    return 2 * kTcolHaloCost + tcol_cost_prefix(u1, ns) - tcol_cost_prefix(u0, ns) -
           (u0 % ns == 0 ? kTcolBandCrossCost : 0.0);
}
// Greedy fill under a cost cap: each range takes the most units whose cost
// stays within cap (at least one, and one left for every later range).
// Returns whether the ranges hold every unit.
inline bool tcol_fill_units(int units, int ns, int grid, double cap, int* split) {
    split[0] = 0;
    for (int b = 0; b < grid; ++b) {
        const int u0 = split[b];
        int lo = u0 + 1, hi = units - (grid - 1 - b);  // the range's possible ends
        while (lo < hi) {  // the range cost grows with its end
            const int mid = lo + (hi - lo + 1) / 2;
            if (tcol_range_cost(u0, mid, ns) <= cap) lo = mid;
            else hi = mid - 1;
        }
        split[b + 1] = lo;
    }
    return split[grid] == units;
}
inline void tcol_split_units(int units, int ns, int grid, int* split) {
    // a cap above the whole image's cost always fits: bisect down from it
    double lo = 0.0, hi = tcol_range_cost(0, units, ns) + 1.0 + kTcolLeftEdgeCost + kTcolRightEdgeCost;
    while (hi - lo > 1e-3 * (1.0 + lo)) {
        const double mid = 0.5 * (lo + hi);
        if (tcol_fill_units(units, ns, grid, mid, split)) hi = mid;
        else lo = mid;
    }
    tcol_fill_units(units, ns, grid, hi, split);
}
}  // namespace ipfc
