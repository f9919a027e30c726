// morph_u8.cuh -- erosion / dilation of uint8 images by an all-ones element:
// the packed-byte tile used by both the per-image kernel and the batch kernel.
//
// Same definition as morph_rect_tile (morph.cuh, after
// include/ipf/morphology.hpp:60-84): min (erode) or max (dilate) over the
// sw x sh window anchored at (sw/2, sh/2); pixels outside the image never
// count, which for an all-ones element equals padding with the identity
// (255 for min, 0 for max) because the window always holds its in-image
// centre.
//
// Memory path (the op is bound by HBM bandwidth):
//  * staging: each source row of the tile is copied with 16-byte cp.async
//    from the 16-byte-aligned address at or below the row's first sample, so
//    rows of any pitch and alignment move in full-width copies, all of a
//    thread's rows in flight at once (a load then store would wait for each
//    row in turn); the row's
//    offset into its staged copy (0..15 bytes) is kept per row.  16-byte
//    chunks that leave the row are read byte by byte, with the identity
//    outside the image;
//  * compute: 4 adjacent samples per 32-bit word.  The row pass takes, for
//    each window column i, the 4 bytes at staged offset 4t + i*C + delta
//    (two aligned shared words and one byte permute), spreads them over two
//    words of 16-bit lanes (bytes 0, 2 and bytes 1, 3) and folds them with
//    min/max.u16x2 (native; per-byte forms are emulated); the column pass
//    folds sh row-pass word pairs and packs the bytes back once;
//  * store: one 32-bit store per 4 outputs when the destination address is
//    4-byte aligned, byte stores otherwise (rows of odd pitch).
#pragma once

#include "kernels.cuh"

namespace ipfc {

constexpr int kMorphU8Threads = 256;

// 16-bit lane min / max (two lanes per instruction).  The host form, lane
// by lane, lets host programs run the selection networks built on these.
__host__ __device__ __forceinline__ unsigned umin2(unsigned a, unsigned b) {
#ifdef __CUDA_ARCH__
    unsigned r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
#else
    const unsigned lo = (a & 0xffffu) < (b & 0xffffu) ? (a & 0xffffu) : (b & 0xffffu);
    const unsigned hi = (a >> 16) < (b >> 16) ? (a >> 16) : (b >> 16);
    return (hi << 16) | lo;
#endif
}
__host__ __device__ __forceinline__ unsigned umax2(unsigned a, unsigned b) {
#ifdef __CUDA_ARCH__
    unsigned r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
#else
    const unsigned lo = (a & 0xffffu) > (b & 0xffffu) ? (a & 0xffffu) : (b & 0xffffu);
    const unsigned hi = (a >> 16) > (b >> 16) ? (a >> 16) : (b >> 16);
    return (hi << 16) | lo;
#endif
}
// bytes (b0, b1, b2, b3) -> lanes (b0, b2) and (b1, b3), and back
__device__ __forceinline__ unsigned lanes_even(unsigned w) { return __byte_perm(w, 0u, 0x4240u); }
__device__ __forceinline__ unsigned lanes_odd(unsigned w) { return __byte_perm(w, 0u, 0x4341u); }
__device__ __forceinline__ unsigned lanes_pack(unsigned ev, unsigned od) { return __byte_perm(ev, od, 0x6240u); }

// Bytes [s, s+4) of the staged row `w` (32-bit words), s >= 0.
__device__ __forceinline__ unsigned staged_word(const unsigned* w, int s) {
    const unsigned lo = w[s >> 2], hi = w[(s >> 2) + 1];
    return __byte_perm(lo, hi, 0x3210u + 0x1111u * (unsigned)(s & 3));
}

// Geometry of one tile: TX output samples (a multiple of 4) x TY rows.
struct MorphU8Geom {
    int RY;  // staged rows
    int SP;  // staged row stride (bytes, multiple of 16)
    int TW;  // words per row-pass row (TX / 4)
    __host__ __device__ MorphU8Geom(int TX, int TY, int sw, int sh, int C) {
        RY = TY + sh - 1;
        const int SWB = TX + (sw - 1) * C;
        SP = ((SWB + 15 + 16) / 16) * 16 + 16;  // delta + samples + the last word's neighbour
        TW = TX / 4;
    }
    // staged rows, row-pass rows (two words of 16-bit lanes per 4 samples), per-row offsets
    __host__ __device__ size_t bytes() const {
        return (size_t)RY * SP + (size_t)RY * TW * 8 + (size_t)RY * 4;
    }
};

__host__ __device__ inline size_t morph_u8_tile_bytes(int TX, int TY, int sw, int sh, int C) {
    return MorphU8Geom(TX, TY, sw, sh, C).bytes();
}

template <bool IS_MIN>
__device__ __forceinline__ unsigned fold2(unsigned a, unsigned b) {
    return IS_MIN ? umin2(a, b) : umax2(a, b);
}

// SW, SH: the window at compile time (3 x 3, the common element), or 0 for
// the sizes in `a`.
template <bool IS_MIN, int SW, int SH>
__device__ __forceinline__ void morph_u8_tile_impl(const MorphCore& a, int TX, int TY, int bx, int by,
                                                   unsigned char* smem) {
    const int sw = SW > 0 ? SW : a.sw, sh = SH > 0 ? SH : a.sh;
    const MorphU8Geom g(TX, TY, sw, sh, a.C);
    unsigned char* stage = smem;
    uint2* hrow = reinterpret_cast<uint2*>(smem + (size_t)g.RY * g.SP);
    int* delta = reinterpret_cast<int*>(hrow + (size_t)g.RY * g.TW);
    const int C = a.C;
    const int rowlen = a.W * C;
    const int q0 = bx * TX, y0 = by * TY;
    const int g0 = q0 - a.ax * C;  // global sample of staged sample 0
    const unsigned fill = IS_MIN ? 0xffffffffu : 0u;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kMorphU8Threads / 32;

    // ---- staging
    for (int r = warp; r < g.RY; r += nwarp) {
        const int gy = y0 - a.ay + r;
        uint4* dst = reinterpret_cast<uint4*>(stage + (size_t)r * g.SP);
        const int nch = g.SP / 16;
        if ((unsigned)gy >= (unsigned)a.H) {
            for (int c = lane; c < nch; c += 32) dst[c] = make_uint4(fill, fill, fill, fill);
            if (lane == 0) delta[r] = 0;
            continue;
        }
        const unsigned char* p = reinterpret_cast<const unsigned char*>(a.src) + (long long)gy * a.spitch;
        const int d = (int)(((uintptr_t)p + (uintptr_t)(long long)g0) & 15);
        if (lane == 0) delta[r] = d;
        const int gc0 = g0 - d;  // global sample of the first staged chunk's first byte
        for (int c = lane; c < nch; c += 32) {
            const int gc = gc0 + 16 * c;
            if (gc >= 0 && gc + 16 <= rowlen) {
                cp_async16(dst + c, p + gc);  // all of this thread's rows in flight at once
            } else {
                uint4 v;
                unsigned w[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    unsigned x = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int gg = gc + 4 * k + b;
                        const unsigned byte = ((unsigned)gg < (unsigned)rowlen) ? (unsigned)__ldg(p + gg) : (fill & 0xffu);
                        x |= byte << (8 * b);
                    }
                    w[k] = x;
                }
                v = make_uint4(w[0], w[1], w[2], w[3]);
                dst[c] = v;
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();

    // ---- row pass: hrow[r][t] = fold over i of staged bytes [4t + i*C + delta_r, +4)
    // (a warp per row, a lane per word: no index division)
    for (int r = warp; r < g.RY; r += nwarp) {
        const unsigned* w = reinterpret_cast<const unsigned*>(stage + (size_t)r * g.SP);
        const int dr = delta[r];
        uint2* hr = hrow + (size_t)r * g.TW;
        if constexpr (SW > 0) {
            // window column i of word t starts at byte 4t + dr + i*C: its word
            // offset and byte selector depend on the row only
            int off[SW];
            unsigned sel[SW];
#pragma unroll
            for (int i = 0; i < SW; ++i) {
                const int b = dr + i * C;
                off[i] = b >> 2;
                sel[i] = 0x3210u + 0x1111u * (unsigned)(b & 3);
            }
            for (int t = lane; t < g.TW; t += 32) {
                const unsigned* wt = w + t;
                const unsigned w0 = __byte_perm(wt[off[0]], wt[off[0] + 1], sel[0]);
                unsigned ev = lanes_even(w0), od = lanes_odd(w0);
#pragma unroll
                for (int i = 1; i < SW; ++i) {
                    const unsigned wi = __byte_perm(wt[off[i]], wt[off[i] + 1], sel[i]);
                    ev = fold2<IS_MIN>(ev, lanes_even(wi));
                    od = fold2<IS_MIN>(od, lanes_odd(wi));
                }
                hr[t] = make_uint2(ev, od);
            }
        } else {
            for (int t = lane; t < g.TW; t += 32) {
                const int s0 = 4 * t + dr;
                const unsigned w0 = staged_word(w, s0);
                unsigned ev = lanes_even(w0), od = lanes_odd(w0);
                for (int i = 1; i < sw; ++i) {
                    const unsigned wi = staged_word(w, s0 + i * C);
                    ev = fold2<IS_MIN>(ev, lanes_even(wi));
                    od = fold2<IS_MIN>(od, lanes_odd(wi));
                }
                hr[t] = make_uint2(ev, od);
            }
        }
    }
    __syncthreads();

    // ---- column pass and store (a warp per output row, a lane per word)
    for (int y = warp; y < TY; y += nwarp) {
        const int gy = y0 + y;
        if (gy >= a.H) break;  // rows only grow with y
        unsigned char* drow = reinterpret_cast<unsigned char*>(a.dst) + (long long)gy * a.dpitch;
        const bool aligned = (((uintptr_t)(drow + q0)) & 3) == 0;  // q0 and 4t are multiples of 4
        const uint2* hr = hrow + (size_t)y * g.TW;
        for (int t = lane; t < g.TW; t += 32) {
            const int q = q0 + 4 * t;
            if (q >= rowlen) break;
            uint2 h = hr[t];
            auto fold_row = [&](int j) {
                const uint2 hj = hr[t + j * g.TW];
                h.x = fold2<IS_MIN>(h.x, hj.x);
                h.y = fold2<IS_MIN>(h.y, hj.y);
            };
            if constexpr (SH > 0) {
#pragma unroll
                for (int j = 1; j < SH; ++j) fold_row(j);
            } else {
                for (int j = 1; j < sh; ++j) fold_row(j);
            }
            const unsigned acc = lanes_pack(h.x, h.y);
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

__device__ __forceinline__ void morph_u8_tile(const MorphCore& a, int TX, int TY, int bx, int by,
                                              unsigned char* smem) {
    const bool w3 = a.sw == 3 && a.sh == 3;
    if (a.is_min) {
        if (w3) morph_u8_tile_impl<true, 3, 3>(a, TX, TY, bx, by, smem);
        else morph_u8_tile_impl<true, 0, 0>(a, TX, TY, bx, by, smem);
    } else {
        if (w3) morph_u8_tile_impl<false, 3, 3>(a, TX, TY, bx, by, smem);
        else morph_u8_tile_impl<false, 0, 0>(a, TX, TY, bx, by, smem);
    }
}

}  // namespace ipfc
