// morph.cuh -- grey erosion / dilation (include/ipf/morphology.hpp:53-127).
//
// Pixels outside the image never take part (no border mode).  The source
// tile is staged in shared memory with the operation's identity element
// (+inf for erosion, -inf for dilation) outside the image, which is exactly
// "outside never counts" for an all-ones element, since its window always
// holds the in-image centre.
//   all-ones element : row pass then column pass (morphology.hpp:60-84),
//                      running min/max over the window in shared memory;
//   other elements   : the member offsets in row-major order; an offset
//                      outside the image is skipped, the first in-image one
//                      replaces the starting centre value, later ones replace
//                      it when better (morphology.hpp:85-106), so an element
//                      with no in-image member leaves the centre sample.
#pragma once

#include "kernels.cuh"

namespace ipfc {

template <typename T>
__device__ __forceinline__ void load_morph_tile(float* tile, int RY, int SW, const MorphCore& a, int gq0, int gy0,
                                                float identity) {
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, nrow = (blockDim.x * blockDim.y) >> 5;
    for (int r = tid >> 5; r < RY; r += nrow) {
        const int gy = gy0 + r;
        float* dst = tile + (size_t)r * SW;
        if ((unsigned)gy >= (unsigned)a.H) {
            for (int s = lane; s < SW; s += 32) dst[s] = identity;
            continue;
        }
        const T* srow = row_ptr<T>(a.src, a.spitch, gy);
        for (int s = lane; s < SW; s += 32) {
            const int g = gq0 + s;
            dst[s] = ((unsigned)g < (unsigned)rowlen) ? to_f(srow[g]) : identity;
        }
    }
}

// Shared memory of one TX x TY tile (flat samples x rows), in bytes.
__host__ __device__ inline size_t morph_tile_bytes(int TX, int TY, int sw, int sh, int C, bool rect) {
    const size_t RY = (size_t)TY + sh - 1, SW = (size_t)TX + (size_t)(sw - 1) * C;
    return sizeof(float) * (RY * SW + (rect ? RY * (size_t)TX : 0));
}

// All-ones element: row pass then column pass over the staged tile.  One tile
// at tile coordinates (bx, by); used by morph_kernel and the batch kernel.
template <typename T>
__device__ __forceinline__ void morph_rect_tile(const MorphCore& a, int TX, int TY, int bx, int by, float* smem) {
    const int RY = TY + a.sh - 1;
    const int SW = TX + (a.sw - 1) * a.C;
    float* tile = smem;
    const int q0 = bx * TX, y0 = by * TY;
    const float identity = a.is_min ? __int_as_float(0x7f800000) : __int_as_float(0xff800000);
    load_morph_tile<T>(tile, RY, SW, a, q0 - a.ax * a.C, y0 - a.ay, identity);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    float* th = smem + (size_t)RY * SW;
    for (int idx = tid; idx < RY * TX; idx += nt) {
        const int r = idx / TX, t = idx - r * TX;
        const float* p = tile + (size_t)r * SW + t;
        float v = p[0];
        if (a.is_min)
            for (int i = 1; i < a.sw; ++i) v = fminf(v, p[i * a.C]);
        else
            for (int i = 1; i < a.sw; ++i) v = fmaxf(v, p[i * a.C]);
        th[idx] = v;
    }
    __syncthreads();
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const float* p = th + (size_t)y * TX + t;
        float v = p[0];
        if (a.is_min)
            for (int j = 1; j < a.sh; ++j) v = fminf(v, p[(size_t)j * TX]);
        else
            for (int j = 1; j < a.sh; ++j) v = fmaxf(v, p[(size_t)j * TX]);
        row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(v);
    }
    __syncthreads();
}

// Any element: the member list in row-major order.
template <typename T>
__device__ __forceinline__ void morph_list_tile(const MorphArgs& a, int TX, int TY, int bx, int by, float* smem) {
    const int RY = TY + a.sh - 1;
    const int SW = TX + (a.sw - 1) * a.C;
    float* tile = smem;
    const int q0 = bx * TX, y0 = by * TY;
    const float identity = a.is_min ? __int_as_float(0x7f800000) : __int_as_float(0xff800000);
    load_morph_tile<T>(tile, RY, SW, a, q0 - a.ax * a.C, y0 - a.ay, identity);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const int px = gq / a.C;
        float v = tile[(size_t)(y + a.ay) * SW + t + a.ax * a.C];
        bool any = false;
        for (int k = 0; k < a.noffs; ++k) {
            const short2 o = a.offs[k];
            const int sx = px + o.x, sy = gy + o.y;
            if ((unsigned)sx >= (unsigned)a.W || (unsigned)sy >= (unsigned)a.H) continue;
            const float sv = tile[(size_t)(y + a.ay + o.y) * SW + t + (a.ax + o.x) * a.C];
            const bool better = a.is_min ? (sv < v) : (v < sv);
            if (!any || better) v = sv;
            any = true;
        }
        row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(v);
    }
    __syncthreads();
}

}  // namespace ipfc
