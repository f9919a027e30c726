// morph3_stream.cu -- erode / dilate of uint8 images by the 3 x 3 all-ones
// element (include/ipf/morphology.hpp:60-84 with the default element of
// getStructuringElement, morphology.hpp:24-49) as a register-streaming
// kernel: no shared memory, one 16-byte load and one 16-byte store per lane
// per row.
//
// Each warp owns a slice of 32 16-byte chunks (512 samples) of the
// interleaved row and walks a band of rows down the image:
//  * per row, lane t loads chunk t (16 samples) and gets the word left of
//    it and the word right of it from its neighbours with shuffles (the
//    slice's two edge lanes load theirs); the horizontal min / max of
//    samples x - C, x, x + C is formed per 32-bit word from byte permutes of
//    adjacent words and `min/max.u16x2` over the even and odd bytes;
//  * the vertical min / max of the last three rows' horizontal results
//    gives one output row, packed back to bytes and stored.
// Rows outside the image and samples outside the row never count: they
// enter as the identity (255 for min, 0 for max), which for an all-ones
// element is the definition (the window always holds its in-image centre).
// The source row is read only inside [0, rowlen): a chunk that crosses the
// row's end is read word by word.
#include <cuda_runtime.h>

#include "common.cuh"
#include "kernels.cuh"
#include "morph_u8.cuh"

namespace ipfc {

namespace {

constexpr int kM3Warps = 8;
constexpr int kM3Band = 8;   // rows per warp

// Bytes [s, s + 4) of the 8-byte pair (lo, hi), 0 <= s <= 4.
__device__ __forceinline__ unsigned bytes_at(unsigned lo, unsigned hi, int s) {
    return __byte_perm(lo, hi, 0x3210u + 0x1111u * (unsigned)s);
}

struct Row {
    unsigned w[4];
};

// One source row's chunk for lane `lane` at sample x0 (a multiple of 16):
// the words, identity outside [0, rowlen).
__device__ __forceinline__ Row load_chunk(const unsigned char* row, int x0, int rowlen, unsigned ident) {
    Row r;
    if (x0 + 16 <= rowlen) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(row + x0));
        r.w[0] = q.x;
        r.w[1] = q.y;
        r.w[2] = q.z;
        r.w[3] = q.w;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            unsigned v = ident;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int x = x0 + 4 * j + b;
                if (x < rowlen) v = (v & ~(0xffu << (8 * b))) | ((unsigned)__ldg(row + x) << (8 * b));
            }
            r.w[j] = v;
        }
    }
    return r;
}

// The word of source row `row` at sample x (a multiple of 4), identity
// outside [0, rowlen).
__device__ __forceinline__ unsigned load_word(const unsigned char* row, int x, int rowlen, unsigned ident) {
    if (x < 0 || x >= rowlen) return ident;
    if (x + 4 <= rowlen) return __ldg(reinterpret_cast<const unsigned*>(row + x));
    unsigned v = ident;
    for (int b = 0; b < 4 && x + b < rowlen; ++b) v = (v & ~(0xffu << (8 * b))) | ((unsigned)__ldg(row + x + b) << (8 * b));
    return v;
}

// Horizontal 3-tap min / max (taps C samples apart) of one chunk, as even
// and odd 16-bit lanes per word.
template <bool IS_MIN, int C>
__device__ __forceinline__ void hpass(const Row& r, unsigned left, unsigned right, unsigned (&he)[4],
                                      unsigned (&ho)[4]) {
    const unsigned w[6] = {left, r.w[0], r.w[1], r.w[2], r.w[3], right};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const unsigned cm = bytes_at(w[j], w[j + 1], 4 - C);  // samples x - C
        const unsigned cp = bytes_at(w[j + 1], w[j + 2], C);  // samples x + C
        const unsigned c0 = w[j + 1];
        he[j] = fold2<IS_MIN>(fold2<IS_MIN>(lanes_even(cm), lanes_even(c0)), lanes_even(cp));
        ho[j] = fold2<IS_MIN>(fold2<IS_MIN>(lanes_odd(cm), lanes_odd(c0)), lanes_odd(cp));
    }
}

template <bool IS_MIN, int C>
__global__ void __launch_bounds__(32 * kM3Warps) morph3_stream_kernel(const MorphCore a, int nslices, int nbands) {
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * kM3Warps + (threadIdx.x >> 5);
    if (wid >= nslices * nbands) return;  // warp-uniform
    const int slice = wid % nslices, band = wid / nslices;
    const int rowlen = a.W * C;
    const int x0 = 512 * slice + 16 * lane;
    const int y0 = band * kM3Band, y1 = min(y0 + kM3Band, a.H);
    const unsigned ident = IS_MIN ? 0xffffffffu : 0u;
    const unsigned char* src = static_cast<const unsigned char*>(a.src);
    unsigned char* dst = static_cast<unsigned char*>(a.dst);

    // A row's chunk as loaded (the slice's edge lanes also load the word
    // beyond their chunk); rows are loaded two ahead of their use, so every
    // warp keeps two rows of loads in flight while it computes.
    struct Raw {
        Row r;
        unsigned edge;  // lane 0: the word left of the slice; lane 31: the word right of it
    };
    auto load = [&](int y) {
        Raw w;
        if (y < 0 || y >= a.H) {
#pragma unroll
            for (int j = 0; j < 4; ++j) w.r.w[j] = ident;
            w.edge = ident;
            return w;
        }
        const unsigned char* row = src + (long long)y * a.spitch;
        w.r = load_chunk(row, x0, rowlen, ident);
        w.edge = lane == 0 ? load_word(row, x0 - 4, rowlen, ident)
                           : (lane == 31 ? load_word(row, x0 + 16, rowlen, ident) : ident);
        return w;
    };
    auto hrow = [&](const Raw& w, unsigned (&he)[4], unsigned (&ho)[4]) {
        unsigned left = __shfl_up_sync(0xffffffffu, w.r.w[3], 1);
        unsigned right = __shfl_down_sync(0xffffffffu, w.r.w[0], 1);
        if (lane == 0) left = w.edge;
        if (lane == 31) right = w.edge;
        hpass<IS_MIN, C>(w.r, left, right, he, ho);
    };
    // horizontal results of rows y-1 (p) and y (c); row y+1 is computed in the loop
    unsigned pe[4], po[4], ce[4], co[4];
    hrow(load(y0 - 1), pe, po);
    hrow(load(y0), ce, co);
    Raw r1 = load(y0 + 1), r2 = load(y0 + 2);
    // Unrolled over the band, so the row registers rotate by renaming: a
    // copy of r2 into r1 would wait for r2's loads to land.
#pragma unroll
    for (int i = 0; i < kM3Band; ++i) {
        const int y = y0 + i;
        if (y >= y1) break;
        unsigned ne[4], no[4];
        hrow(r1, ne, no);
        r1 = r2;
        r2 = load(y + 3);
        if (x0 < rowlen) {
            unsigned out[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
                out[j] = lanes_pack(fold2<IS_MIN>(fold2<IS_MIN>(pe[j], ce[j]), ne[j]),
                                    fold2<IS_MIN>(fold2<IS_MIN>(po[j], co[j]), no[j]));
            unsigned char* drow = dst + (long long)y * a.dpitch;
            if (x0 + 16 <= rowlen) {
                *reinterpret_cast<uint4*>(drow + x0) = make_uint4(out[0], out[1], out[2], out[3]);
            } else {
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    if (x0 + e < rowlen) drow[x0 + e] = (unsigned char)(out[e >> 2] >> (8 * (e & 3)));
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            pe[j] = ce[j];
            po[j] = co[j];
            ce[j] = ne[j];
            co[j] = no[j];
        }
    }
}

template <bool IS_MIN>
cudaError_t launch_c(const MorphCore& a, cudaStream_t s) {
    const int rowlen = a.W * a.C;
    const int nslices = (rowlen + 511) / 512, nbands = (a.H + kM3Band - 1) / kM3Band;
    const long long warps = (long long)nslices * nbands;
    const int grid = (int)((warps + kM3Warps - 1) / kM3Warps);
    switch (a.C) {
        case 1: morph3_stream_kernel<IS_MIN, 1><<<grid, 32 * kM3Warps, 0, s>>>(a, nslices, nbands); break;
        case 2: morph3_stream_kernel<IS_MIN, 2><<<grid, 32 * kM3Warps, 0, s>>>(a, nslices, nbands); break;
        case 3: morph3_stream_kernel<IS_MIN, 3><<<grid, 32 * kM3Warps, 0, s>>>(a, nslices, nbands); break;
        case 4: morph3_stream_kernel<IS_MIN, 4><<<grid, 32 * kM3Warps, 0, s>>>(a, nslices, nbands); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

// The 3 x 3 all-ones element, centred, on uint8 images of 1 to 4 channels
// whose source and destination rows start 16-byte aligned; false when the
// call is outside that (the tile kernel runs instead).
bool morph3_stream_launch(const MorphCore& a, cudaStream_t s, cudaError_t* e) {
    if (!(a.is_rect && a.sw == 3 && a.sh == 3 && a.ax == 1 && a.ay == 1)) return false;
    if (a.C < 1 || a.C > 4 || a.W <= 0 || a.H <= 0) return false;
    if ((long long)a.W * a.C > 0x3fffffffLL) return false;
    if (((uintptr_t)a.src & 15) || ((uintptr_t)a.dst & 15) || (a.spitch & 15) || (a.dpitch & 15)) return false;
    *e = a.is_min ? launch_c<true>(a, s) : launch_c<false>(a, s);
    return true;
}

}  // namespace ipfc
