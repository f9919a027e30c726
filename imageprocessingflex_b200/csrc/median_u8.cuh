// median_u8.cuh -- exact 3x3 and 5x5 median of uint8 images on packed
// samples: the tile used by the per-image kernel and the batch kernel.
//
// Same result as median_tile (median.cuh, after include/ipf/filter.hpp:
// 302-332): the sample of rank k*k/2 of the border-extended k x k window,
// per channel (order statistics, so any exact selection agrees with the
// reference's histogram / nth_element).
//
//  * staging: each source row of the tile (rows border-mapped) is copied
//    with 16-byte cp.async from the 16-byte-aligned address at or below the
//    row's first sample, all of a thread's rows in flight at once, keeping
//    the row's offset (0..15) into its staged copy;
//    16-byte chunks that leave the row are read byte by byte through the
//    border mapping (border_sample, channel preserved);
//  * selection: 4 adjacent samples per 32-bit word.  Each window word (the
//    4 bytes at staged offset 4t + i*C + delta of row j) is spread over two
//    words of 16-bit lanes (bytes 0, 2 and bytes 1, 3), and both are
//    reduced with min/max.u16x2 (two samples per instruction):
//      k = 3: each window column sorted (3 compare-exchanges), then the
//             median of (max of minima, median of middles, min of maxima);
//      k = 5: columns then rows sorted, then the 7th smallest of the 13
//             entries that can still be the median (forgetful selection:
//             keep m + 2 live values, drop the current minimum and maximum,
//             pull the next);
//  * store: one 32-bit store per 4 outputs where the destination address is
//    4-byte aligned, byte stores otherwise.
#pragma once

#include "common.cuh"
#include "kernels.cuh"
#include "morph_u8.cuh"

namespace ipfc {

constexpr int kMedianU8Threads = 256;

// Geometry of one tile: TX output samples (a multiple of 4) x TY rows.
struct MedianU8Geom {
    int RY;  // staged rows
    int SP;  // staged row stride (bytes, multiple of 16)
    int TW;  // words per output row (TX / 4)
    __host__ __device__ MedianU8Geom(int TX, int TY, int k, int C) {
        RY = TY + k - 1;
        const int SWB = TX + (k - 1) * C;
        SP = ((SWB + 15 + 16) / 16) * 16 + 16;  // delta + samples + the last word's neighbour
        TW = TX / 4;
    }
    __host__ __device__ size_t bytes() const { return (size_t)RY * SP + (size_t)RY * 4; }
};

__host__ __device__ inline size_t median_u8_tile_bytes(int TX, int TY, int k, int C) {
    return MedianU8Geom(TX, TY, k, C).bytes();
}

__host__ __device__ __forceinline__ void ce2(unsigned& a, unsigned& b) {
    const unsigned lo = umin2(a, b), hi = umax2(a, b);
    a = lo;
    b = hi;
}

__host__ __device__ __forceinline__ unsigned med3_2(unsigned a, unsigned b, unsigned c) {
    return umax2(umin2(a, b), umin2(umax2(a, b), c));
}

// median of 9 lane-words: v[dy * 3 + dx]
__host__ __device__ __forceinline__ unsigned median9_2(unsigned (&v)[9]) {
#pragma unroll
    for (int dx = 0; dx < 3; ++dx) {  // sort each column
        ce2(v[dx], v[3 + dx]);
        ce2(v[3 + dx], v[6 + dx]);
        ce2(v[dx], v[3 + dx]);
    }
    const unsigned lo = umax2(umax2(v[0], v[1]), v[2]);
    const unsigned mid = med3_2(v[3], v[4], v[5]);
    const unsigned hi = umin2(umin2(v[6], v[7]), v[8]);
    return med3_2(lo, mid, hi);
}

// Sorts v[i0], v[i0 + st], .. v[i0 + 4 st] ascending (9 compare-exchanges,
// a minimal 5-input network).
template <int N>
__host__ __device__ __forceinline__ void sort5_2(unsigned (&v)[N], int i0, int st) {
    unsigned& a = v[i0];
    unsigned& b = v[i0 + st];
    unsigned& c = v[i0 + 2 * st];
    unsigned& d = v[i0 + 3 * st];
    unsigned& e = v[i0 + 4 * st];
    ce2(a, b);
    ce2(d, e);
    ce2(c, e);
    ce2(c, d);
    ce2(a, d);
    ce2(a, c);
    ce2(b, e);
    ce2(b, d);
    ce2(b, c);
}

// Forgetful selection over v[0..N), N = 2m + 1 (see median.cuh).
template <int N>
__host__ __device__ __forceinline__ unsigned forgetful_2(unsigned (&v)[N]) {
    constexpr int m = N / 2;
#pragma unroll
    for (int round = 0; round < m - 1; ++round) {
        const int a = round, L = m + 2 - round, u = m + 2 + round;
#pragma unroll
        for (int i = a + 1; i < a + L; ++i) ce2(v[a], v[i]);  // minimum to v[a]
#pragma unroll
        for (int i = a + 1; i < a + L - 1; ++i) ce2(v[i], v[a + L - 1]);  // maximum to v[a + L - 1]
        v[a + L - 1] = v[u];
    }
    return med3_2(v[m - 1], v[m], v[m + 1]);
}

// Median of 25 lane-words v[row * 5 + col].  Sort the columns, then the
// rows: in a matrix sorted both ways the entry at (r, c) has at least
// (r+1)(c+1) - 1 entries at or below it and (5-r)(5-c) - 1 at or above it,
// so 6 entries are certainly below the median (rank 13), 6 certainly above,
// and the median is the 7th smallest of the other 13.  45 + 45 + 45
// compare-exchanges instead of forgetful selection's 165 over all 25.
__host__ __device__ __forceinline__ unsigned median25_2(unsigned (&v)[25]) {
#pragma unroll
    for (int c = 0; c < 5; ++c) sort5_2(v, c, 5);  // columns
#pragma unroll
    for (int r = 0; r < 5; ++r) sort5_2(v, 5 * r, 1);  // rows
    unsigned w[13] = {v[3],  v[4],  v[7],  v[8],  v[9],  v[11], v[12],
                      v[13], v[15], v[16], v[17], v[20], v[21]};
    return forgetful_2<13>(w);
}

template <int K>
__device__ __forceinline__ void median_u8_tile_k(const MedianArgs& a, int TX, int TY, int bx, int by,
                                                 unsigned char* smem) {
    const MedianU8Geom g(TX, TY, K, a.C);
    unsigned char* stage = smem;
    int* delta = reinterpret_cast<int*>(smem + (size_t)g.RY * g.SP);
    const int C = a.C;
    const int rowlen = a.W * C;
    const int q0 = bx * TX, y0 = by * TY;
    const int g0 = q0 - (K / 2) * C;  // global sample of staged sample 0
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kMedianU8Threads / 32;

    // ---- staging (rows and samples border-mapped; Constant is not accepted)
    for (int r = warp; r < g.RY; r += nwarp) {
        const int sy = border_index(y0 - K / 2 + r, a.H, a.border);
        const unsigned char* p = reinterpret_cast<const unsigned char*>(a.src) + (long long)sy * a.spitch;
        const int d = (int)(((uintptr_t)p + (uintptr_t)(long long)g0) & 15);
        if (lane == 0) delta[r] = d;
        uint4* dst = reinterpret_cast<uint4*>(stage + (size_t)r * g.SP);
        const int gc0 = g0 - d;
        for (int c = lane; c < g.SP / 16; c += 32) {
            const int gc = gc0 + 16 * c;
            if (gc >= 0 && gc + 16 <= rowlen) {
                cp_async16(dst + c, p + gc);  // all of this thread's rows in flight at once
            } else {
                uint4 v;
                unsigned w[4];
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    unsigned x = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int gg = gc + 4 * kk + b;
                        const int src = ((unsigned)gg < (unsigned)rowlen) ? gg : border_sample(gg, a.W, C, a.border);
                        x |= (unsigned)__ldg(p + (src < 0 ? 0 : src)) << (8 * b);
                    }
                    w[kk] = x;
                }
                v = make_uint4(w[0], w[1], w[2], w[3]);
                dst[c] = v;
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // ---- selection and store (a warp per output row, a lane per word: no index division)
    for (int y = warp; y < TY; y += nwarp) {
        const int gy = y0 + y;
        if (gy >= a.H) break;  // rows only grow with y
        unsigned char* drow = reinterpret_cast<unsigned char*>(a.dst) + (long long)gy * a.dpitch;
        const bool aligned = (((uintptr_t)(drow + q0)) & 3) == 0;  // q0 and 4t are multiples of 4
        for (int t = lane; t < g.TW; t += 32) {
            const int q = q0 + 4 * t;
            if (q >= rowlen) break;
            unsigned raw[K * K];
#pragma unroll
            for (int j = 0; j < K; ++j) {
                const unsigned* w = reinterpret_cast<const unsigned*>(stage + (size_t)(y + j) * g.SP);
                const int s0 = 4 * t + delta[y + j];
#pragma unroll
                for (int i = 0; i < K; ++i) raw[j * K + i] = staged_word(w, s0 + i * C);
            }
            unsigned ev[K * K], od[K * K];
#pragma unroll
            for (int e = 0; e < K * K; ++e) {
                ev[e] = lanes_even(raw[e]);
                od[e] = lanes_odd(raw[e]);
            }
            unsigned me, mo;
            if constexpr (K == 3) {
                me = median9_2(ev);
                mo = median9_2(od);
            } else {
                me = median25_2(ev);
                mo = median25_2(od);
            }
            const unsigned acc = lanes_pack(me, mo);
            if (aligned && q + 4 <= rowlen) {
                *reinterpret_cast<unsigned*>(drow + q) = acc;
            } else {
                const int n = min(4, rowlen - q);
                for (int b = 0; b < n; ++b) drow[q + b] = (unsigned char)(acc >> (8 * b));
            }
        }
    }
    __syncthreads();
}

// k = 3 or 5 (the caller checks); one tile at tile coordinates (bx, by).
__device__ __forceinline__ void median_u8_tile(const MedianArgs& a, int TX, int TY, int bx, int by,
                                               unsigned char* smem) {
    if (a.ksize == 3) median_u8_tile_k<3>(a, TX, TY, bx, by, smem);
    else median_u8_tile_k<5>(a, TX, TY, bx, by, smem);
}

}  // namespace ipfc
