// filter2d_tc.cuh -- geometry of the tensor-core (tcgen05) form of filter2D:
// shared-memory layouts, descriptors and tile sizes, shared by the kernel
// (filter2d_tc.cu) and host-side checks.
//
// The correlation out[y][x] = sum_{j,i} w[j][i] P[y + j - ay][x + i - ax]
// (include/ipf/filter.hpp:159-194, single channel) becomes, for one CTA tile
// of 128 output pixels (x = tx0 + m) by NG x 16 output rows
// (y = ty0 + 16 g + n), NG groups of MMAs
//
//   D_g[m][n] = sum_i sum_k A_{g,i}[m][k] * B_i[n][k]          (M=128, N=32)
//   A_{g,i}[m][k] = T[m + sh_i][16 g + k],   sh_i = i + (axa - ax)
//   B_i[n][k]     = w_hi[k - n][i],  B_i[16 + n][k] = w_lo[k - n][i]
//                   for 0 <= k - n < kh and n < 16, else 0
//
// where T[x'][r] = P[ty0 - ay + r][tx0 - axa + x'] is the source tile stored
// transposed (x' major, source rows r contiguous) and axa = ax rounded up to
// a multiple of 4 (so staged pixel quads start 4-aligned in the image).
// Images of C > 1 interleaved channels are the same correlation over the row
// of W*C samples with the horizontal taps C samples apart: x counts samples,
// the anchor is ax*C samples and tap column i shifts A by i*C rows.
// Both operands are K-major without swizzle: 8 x 16-byte core matrices,
// rows 16 bytes apart, so shifting A by one pixel (the tap offset i) is a
// 16-byte move of the descriptor's start address -- one staged tile serves
// all kw horizontal offsets, and the vertical taps live in the banded B.
//
// Split precision: uint8 pixels are exact in FP16; float pixels are split
// into hi = fp16(p * 2^e) and lo = fp16(p * 2^e - hi) with a per-tile power
// of two 2^e; taps into hi = fp16(w * 2^s), lo = fp16(w * 2^s - hi).  The
// products hi*hi + hi*lo + lo*hi (lo*lo dropped; uint8: A*hi + A*lo) are
// accumulated in FP32 in tensor memory and scaled back by 2^-(e+s).  The hi
// and lo taps sit side by side in B's N dimension, so one N = 32 MMA reads
// the pixel tile once and fills both the hi x hi ("main", columns 0-15) and
// the correction (columns 16-31) accumulator of its group.  Pixels
// are centred first (uint8: p - 128, exact; float: about the tile's mid-range)
// and hi*hi goes to its own accumulator, apart from the small correction
// products, which keeps the accumulators small and their rounding low.
#pragma once

#include <stdint.h>

namespace ipfc {

constexpr int kTcM = 128;          // output pixels per tile (MMA M)
constexpr int kTcN = 16;           // output rows per MMA group (N = 2 x 16: hi and lo taps)
constexpr int kTcGroups = 4;       // MMA groups per tile
constexpr int kTcRows = kTcN * kTcGroups;
constexpr int kTcWorkers = 256;                // staging and epilogue threads (8 warps)
constexpr int kTcThreads = kTcWorkers + 32;    // + the MMA-issuing warp
constexpr int kTcMaxKw = 32;
constexpr int kTcMaxKh = 33;

struct TcGeom {
    int kw, kh, ax, ay;
    int C;       // channels: the row is W*C interleaved samples, tap column i sits i*C samples away
    int axs;     // the anchor in samples (ax * C)
    int axa;     // axs rounded up to a multiple of 4
    int Kt;      // K of one group's window (>= kh + 15, multiple of 16)
    int XR;      // staged pixels per tile row (multiple of 8)
    int KR;      // staged source rows (multiple of 8)
    int lboA;    // bytes between A's 8-row K slabs (= XR * 16)
    int bytesA;  // one A part
    int bytesBi; // B of one tap column (32 rows: hi, lo)
    int bytesB;  // B of all kw tap columns
    int partsA;  // 1 (uint8) or 2 (float hi, lo)
    int offA;    // shared offsets
    int offBar;
    int smem;

    __host__ __device__ TcGeom(int kw_, int kh_, int ax_, int ay_, bool float_src, int C_ = 1) {
        kw = kw_;
        kh = kh_;
        ax = ax_;
        ay = ay_;
        C = C_;
        axs = ax * C;
        axa = (axs + 3) / 4 * 4;
        Kt = (kh + 15 + 15) / 16 * 16;
        XR = (kTcM + (kw - 1) * C + (axa - axs) + 7) / 8 * 8;
        KR = 16 * (kTcGroups - 1) + Kt;
        lboA = XR * 16;
        bytesA = (KR / 8) * lboA;
        bytesBi = (Kt / 8) * 512;
        bytesB = kw * bytesBi;
        partsA = float_src ? 2 : 1;
        offA = bytesB;                              // A: 2 buffers x partsA parts
        offBar = offA + 2 * partsA * bytesA;
        smem = offBar + 192;
    }
    // shared offset of A buffer b, part p
    __host__ __device__ int a_buf(int b, int p) const { return offA + (b * partsA + p) * bytesA; }
    // byte offset of T[x'][r] in an A part
    __host__ __device__ int a_off(int xr, int r) const { return (r >> 3) * lboA + xr * 16 + (r & 7) * 2; }
    // byte offset of B_i[n][k], n in [0, 32)
    __host__ __device__ int b_off(int i, int n, int k) const {
        return i * bytesBi + (k >> 3) * 512 + (n >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2;
    }
};

// tcgen05 shared-memory descriptor: no swizzle, K-major, version 1.
__host__ __device__ inline uint64_t tc_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: D f32, A and B f16, both K-major,
// M = 128, N = n.
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
}

}  // namespace ipfc
