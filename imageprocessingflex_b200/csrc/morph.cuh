// morph.cuh -- grey erosion / dilation (include/ipf/morphology.hpp:53-127).
//
// Pixels outside the image never take part (no border mode).  The source
// tile is staged in shared memory with the operation's identity element
// (+inf for erosion, -inf for dilation) outside the image, which is exactly
// "outside never counts" for an all-ones element, since its window always
// holds the in-image centre.
//   all-ones element : row pass then column pass (morphology.hpp:60-84),
//                      per pass the direct window scan for short windows,
//                      van Herk / Gil-Werman block prefix and suffix extrema
//                      from kMorphVhgwMin members on;
//   other elements   : the member offsets in row-major order; an offset
//                      outside the image is skipped, the first in-image one
//                      replaces the starting centre value, later ones replace
//                      it when better (morphology.hpp:85-106), so an element
//                      with no in-image member leaves the centre sample.
#pragma once

#include "kernels.cuh"

namespace ipfc {

// Storage of the shared tile: float holds uint8/uint16/int16/float exactly;
// int32 and double keep their own type.  The identity element of erosion is
// the storage type's largest value (+inf for floating types), of dilation
// its smallest.
template <typename T> struct MorphStore { using type = float; };
template <> struct MorphStore<int32_t> { using type = int32_t; };
template <> struct MorphStore<double> { using type = double; };

template <typename V> __device__ __forceinline__ V morph_identity(bool is_min);
template <> __device__ __forceinline__ float morph_identity<float>(bool is_min) {
    return is_min ? __int_as_float(0x7f800000) : __int_as_float(0xff800000);
}
template <> __device__ __forceinline__ double morph_identity<double>(bool is_min) {
    return is_min ? __longlong_as_double(0x7ff0000000000000ll) : __longlong_as_double((long long)0xfff0000000000000ull);
}
template <> __device__ __forceinline__ int32_t morph_identity<int32_t>(bool is_min) {
    return is_min ? 0x7fffffff : (int32_t)0x80000000;
}
__device__ __forceinline__ float mmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ float mmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double mmin(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ double mmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ int32_t mmin(int32_t a, int32_t b) { return a < b ? a : b; }
__device__ __forceinline__ int32_t mmax(int32_t a, int32_t b) { return a < b ? b : a; }

template <typename T, typename V>
__device__ __forceinline__ void load_morph_tile(V* tile, int RY, int SW, const MorphCore& a, int gq0, int gy0,
                                                V identity) {
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = tid & 31, nrow = (blockDim.x * blockDim.y) >> 5;
    for (int r = tid >> 5; r < RY; r += nrow) {
        const int gy = gy0 + r;
        V* dst = tile + (size_t)r * SW;
        if ((unsigned)gy >= (unsigned)a.H) {
            for (int s = lane; s < SW; s += 32) dst[s] = identity;
            continue;
        }
        const T* srow = row_ptr<T>(a.src, a.spitch, gy);
        for (int s = lane; s < SW; s += 32) {
            const int g = gq0 + s;
            dst[s] = ((unsigned)g < (unsigned)rowlen) ? static_cast<V>(srow[g]) : identity;
        }
    }
}

// From this many members along an axis, a rectangular element's pass runs
// van Herk / Gil-Werman (block prefix and suffix extrema, about three
// operations per sample whatever the length) instead of the direct
// window scan (length - 1 operations per sample).
constexpr int kMorphVhgwMin = 7;

// Shared memory of one TX x TY tile (flat samples x rows), in bytes, for tile
// elements of `esize` bytes: the source tile plus the row-pass result, and
// for a van Herk / Gil-Werman pass one more tile-sized array of suffixes.
__host__ __device__ inline size_t morph_tile_bytes(int TX, int TY, int sw, int sh, int C, bool rect,
                                                   size_t esize = sizeof(float)) {
    const size_t RY = (size_t)TY + sh - 1, SW = (size_t)TX + (size_t)(sw - 1) * C;
    const bool vhgw = rect && (sw >= kMorphVhgwMin || sh >= kMorphVhgwMin);
    return esize * (RY * SW + (rect ? RY * (size_t)TX : 0) + (vhgw ? RY * SW : 0));
}

// All-ones element: row pass then column pass over the staged tile.  One tile
// at tile coordinates (bx, by); used by morph_kernel and the batch kernel.
template <typename T>
__device__ __forceinline__ void morph_rect_tile(const MorphCore& a, int TX, int TY, int bx, int by, float* smem_raw) {
    using V = typename MorphStore<T>::type;
    V* smem = reinterpret_cast<V*>(smem_raw);
    const int RY = TY + a.sh - 1;
    const int SW = TX + (a.sw - 1) * a.C;
    V* tile = smem;
    const int q0 = bx * TX, y0 = by * TY;
    const bool is_min = a.is_min != 0;
    const V identity = morph_identity<V>(is_min);
    load_morph_tile<T, V>(tile, RY, SW, a, q0 - a.ax * a.C, y0 - a.ay, identity);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    V* th = smem + (size_t)RY * SW;
    V* aux = th + (size_t)RY * TX;  // van Herk / Gil-Werman suffixes (RY * SW elements)
    // ---- row pass: th[r][t] = extremum of tile[r][t + i C], i < sw
    if (a.sw >= kMorphVhgwMin) {
        // sequences: (row r, residue c mod C), index j -> sample c + j C
        const int nseq = RY * a.C;
        const int len = (SW + a.C - 1) / a.C;
        const int nb = (len + a.sw - 1) / a.sw;
        for (int it = tid; it < nseq * nb; it += nt) {
            const int q = it % nseq, b = it / nseq;
            const int r = q / a.C, c = q - r * a.C;
            V* row = tile + (size_t)r * SW;
            V* srow = aux + (size_t)r * SW;
            const int j0 = b * a.sw;
            const int j1 = min(j0 + a.sw, (SW - c + a.C - 1) / a.C);
            if (j0 >= j1) continue;
            // suffixes first (from the source), then prefixes in place
            V run = row[c + (j1 - 1) * a.C];
            srow[c + (j1 - 1) * a.C] = run;
            for (int j = j1 - 2; j >= j0; --j) {
                const V x = row[c + j * a.C];
                run = is_min ? mmin(run, x) : mmax(run, x);
                srow[c + j * a.C] = run;
            }
            run = row[c + j0 * a.C];
            for (int j = j0 + 1; j < j1; ++j) {
                V* p = row + c + j * a.C;
                run = is_min ? mmin(run, *p) : mmax(run, *p);
                *p = run;
            }
        }
        __syncthreads();
        for (int idx = tid; idx < RY * TX; idx += nt) {
            const int r = idx / TX, t = idx - r * TX;
            const V s0 = aux[(size_t)r * SW + t], p1 = tile[(size_t)r * SW + t + (a.sw - 1) * a.C];
            th[idx] = is_min ? mmin(s0, p1) : mmax(s0, p1);
        }
    } else {
        for (int idx = tid; idx < RY * TX; idx += nt) {
            const int r = idx / TX, t = idx - r * TX;
            const V* p = tile + (size_t)r * SW + t;
            V v = p[0];
            if (is_min)
                for (int i = 1; i < a.sw; ++i) v = mmin(v, p[i * a.C]);
            else
                for (int i = 1; i < a.sw; ++i) v = mmax(v, p[i * a.C]);
            th[idx] = v;
        }
    }
    __syncthreads();
    // ---- column pass: out[y][t] = extremum of th[y + j][t], j < sh
    if (a.sh >= kMorphVhgwMin) {
        const int nb = (RY + a.sh - 1) / a.sh;
        for (int it = tid; it < TX * nb; it += nt) {
            const int t = it % TX, b = it / TX;
            const int j0 = b * a.sh, j1 = min(j0 + a.sh, RY);
            V run = th[(size_t)(j1 - 1) * TX + t];
            aux[(size_t)(j1 - 1) * TX + t] = run;
            for (int j = j1 - 2; j >= j0; --j) {
                const V x = th[(size_t)j * TX + t];
                run = is_min ? mmin(run, x) : mmax(run, x);
                aux[(size_t)j * TX + t] = run;
            }
            run = th[(size_t)j0 * TX + t];
            for (int j = j0 + 1; j < j1; ++j) {
                V* p = th + (size_t)j * TX + t;
                run = is_min ? mmin(run, *p) : mmax(run, *p);
                *p = run;
            }
        }
        __syncthreads();
        for (int idx = tid; idx < TY * TX; idx += nt) {
            const int y = idx / TX, t = idx - y * TX;
            const int gy = y0 + y, gq = q0 + t;
            if (gy >= a.H || gq >= rowlen) continue;
            const V s0 = aux[(size_t)y * TX + t], p1 = th[(size_t)(y + a.sh - 1) * TX + t];
            row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(is_min ? mmin(s0, p1) : mmax(s0, p1));
        }
    } else {
        for (int idx = tid; idx < TY * TX; idx += nt) {
            const int y = idx / TX, t = idx - y * TX;
            const int gy = y0 + y, gq = q0 + t;
            if (gy >= a.H || gq >= rowlen) continue;
            const V* p = th + (size_t)y * TX + t;
            V v = p[0];
            if (is_min)
                for (int j = 1; j < a.sh; ++j) v = mmin(v, p[(size_t)j * TX]);
            else
                for (int j = 1; j < a.sh; ++j) v = mmax(v, p[(size_t)j * TX]);
            row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(v);
        }
    }
    __syncthreads();
}

// Any element: the member list in row-major order.
template <typename T>
__device__ __forceinline__ void morph_list_tile(const MorphArgs& a, int TX, int TY, int bx, int by, float* smem_raw) {
    using V = typename MorphStore<T>::type;
    V* tile = reinterpret_cast<V*>(smem_raw);
    const int RY = TY + a.sh - 1;
    const int SW = TX + (a.sw - 1) * a.C;
    const int q0 = bx * TX, y0 = by * TY;
    const V identity = morph_identity<V>(a.is_min != 0);
    load_morph_tile<T, V>(tile, RY, SW, a, q0 - a.ax * a.C, y0 - a.ay, identity);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const int px = gq / a.C;
        V v = tile[(size_t)(y + a.ay) * SW + t + a.ax * a.C];
        bool any = false;
        for (int k = 0; k < a.noffs; ++k) {
            const short2 o = a.offs[k];
            const int sx = px + o.x, sy = gy + o.y;
            if ((unsigned)sx >= (unsigned)a.W || (unsigned)sy >= (unsigned)a.H) continue;
            const V sv = tile[(size_t)(y + a.ay + o.y) * SW + t + (a.ax + o.x) * a.C];
            const bool better = a.is_min ? (sv < v) : (v < sv);
            if (!any || better) v = sv;
            any = true;
        }
        row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(v);
    }
    __syncthreads();
}

}  // namespace ipfc
