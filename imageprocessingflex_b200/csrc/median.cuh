// median.cuh -- exact k x k median (medianBlur, include/ipf/filter.hpp:302-332).
//
// The reference returns the sample of rank k*k/2 of the border-extended
// window, per channel: a sliding histogram for uint8 with k >= 5
// (filter.hpp:271-297), nth_element otherwise.  Both are order statistics, so
// any exact selection gives the same value.  Here:
//   k = 3, 5 : the window is held in registers and reduced by forgetful
//              selection: of a live set of m+2 values (n = 2m+1) the minimum
//              and the maximum can never be the median, so both are dropped
//              and the next window value pulled in, until three remain.  Only
//              min/max, no branches, exact for every type;
//   k >= 7   : radix selection on order-preserving integer keys read from the
//              shared-memory tile, one key bit per round.
// The source tile is staged in shared memory with the border resolved at load
// (tile.cuh); Constant is rejected by the API layer as in the reference.
#pragma once

#include "common.cuh"
#include "kernels.cuh"
#include "tile.cuh"

namespace ipfc {

namespace median_detail {

// Storage type of the shared tile: float holds uint8/uint16/int16/float
// exactly; int32 and double keep their own type.
template <typename T> struct Store { using type = float; };
template <> struct Store<int32_t> { using type = int32_t; };
template <> struct Store<double> { using type = double; };

__host__ __device__ __forceinline__ float vmin(float a, float b) { return fminf(a, b); }
__host__ __device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__host__ __device__ __forceinline__ double vmin(double a, double b) { return fmin(a, b); }
__host__ __device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__host__ __device__ __forceinline__ int32_t vmin(int32_t a, int32_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int32_t vmax(int32_t a, int32_t b) { return a < b ? b : a; }

template <typename V>
__host__ __device__ __forceinline__ V med3(V a, V b, V c) {
    return vmax(vmin(a, b), vmin(vmax(a, b), c));
}

// Forgetful selection over v[0..N), N = 2m+1.  Live set v[a .. a+L), next
// unseen value v[u].  Each round bubbles the live minimum to v[a] and the live
// maximum to v[a+L-1], drops both, and moves v[u] into the freed maximum slot.
template <int N, typename V>
__host__ __device__ __forceinline__ V median_forgetful(V (&v)[N]) {
    constexpr int m = N / 2;
#pragma unroll
    for (int round = 0; round < m - 1; ++round) {
        const int a = round, L = m + 2 - round, u = m + 2 + round;
#pragma unroll
        for (int i = a + 1; i < a + L; ++i) {
            const V x = v[a], y = v[i];
            v[a] = vmin(x, y);
            v[i] = vmax(x, y);
        }
#pragma unroll
        for (int i = a + 1; i < a + L - 1; ++i) {
            const V x = v[i], y = v[a + L - 1];
            v[i] = vmin(x, y);
            v[a + L - 1] = vmax(x, y);
        }
        v[a + L - 1] = v[u];
    }
    return med3(v[m - 1], v[m], v[m + 1]);
}

template <int K, typename V>
__device__ __forceinline__ V median_small(const V* tile, int SW, int y, int t, int C) {
    V v[K * K];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int i = 0; i < K; ++i) v[j * K + i] = tile[(size_t)(y + j) * SW + t + i * C];
    return median_forgetful<K * K>(v);
}

// Key of a tile value: integers map to value + offset (order-preserving,
// `bits` wide); floats map through the IEEE sign-flip trick (32 or 64 bits).
template <typename T>
struct MedianKey {
    using V = typename Store<T>::type;
    using K = typename std::conditional<std::is_same<T, double>::value, unsigned long long, unsigned>::type;
    static constexpr int bits = sizeof(T) == 1 ? 8 : (sizeof(T) == 2 ? 16 : (sizeof(T) == 4 ? 32 : 64));
    __device__ static K key(V v) {
        if constexpr (std::is_same<T, float>::value) {
            const unsigned b = __float_as_uint(v);
            return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
        } else if constexpr (std::is_same<T, double>::value) {
            const unsigned long long b = (unsigned long long)__double_as_longlong(v);
            return (b >> 63) ? ~b : (b | (1ull << 63));
        } else if constexpr (std::is_same<T, int32_t>::value) {
            return (unsigned)v ^ 0x80000000u;
        } else if constexpr (std::is_same<T, int16_t>::value) {
            return (unsigned)((int)v + 32768);
        } else {
            return (unsigned)(int)v;
        }
    }
    __device__ static V value(K k) {
        if constexpr (std::is_same<T, float>::value) {
            return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
        } else if constexpr (std::is_same<T, double>::value) {
            return __longlong_as_double((long long)((k >> 63) ? (k & ~(1ull << 63)) : ~k));
        } else if constexpr (std::is_same<T, int32_t>::value) {
            return (int32_t)(k ^ 0x80000000u);
        } else if constexpr (std::is_same<T, int16_t>::value) {
            return (float)((int)k - 32768);
        } else {
            return (float)k;
        }
    }
};

template <typename T>
__device__ typename MedianKey<T>::V median_radix(const typename MedianKey<T>::V* tile, int SW, int y, int t, int C,
                                                 int k) {
    using Key = MedianKey<T>;
    using KT = typename Key::K;
    unsigned rank = (unsigned)(k * k / 2);
    KT prefix = 0;
    for (int bit = Key::bits - 1; bit >= 0; --bit) {
        // count window keys whose bits above `bit` equal prefix's and whose
        // bit `bit` is 0
        const KT hi_mask = (bit == Key::bits - 1) ? (KT)0 : ((~(KT)0) << (bit + 1));
        unsigned cnt = 0;
        for (int j = 0; j < k; ++j) {
            const typename Key::V* row = tile + (size_t)(y + j) * SW + t;
            for (int i = 0; i < k; ++i) {
                const KT kk = Key::key(row[i * C]);
                cnt += ((kk & hi_mask) == prefix) && !((kk >> bit) & (KT)1);
            }
        }
        if (rank >= cnt) {
            rank -= cnt;
            prefix |= (KT)1 << bit;
        }
    }
    return Key::value(prefix);
}

}  // namespace median_detail

// Shared memory of one TX x TY median tile (flat samples x rows), in bytes,
// for tile elements of `esize` bytes (4: uint8/uint16/int16/float/int32; 8: double).
__host__ __device__ inline size_t median_tile_bytes(int TX, int TY, int k, int C, size_t esize = sizeof(float)) {
    return esize * (size_t)(TY + k - 1) * (size_t)(TX + (k - 1) * C);
}

// One TX x TY tile (flat samples x rows) at tile coordinates (bx, by); `tile`
// holds (TY + k - 1) x (TX + (k - 1) C) floats of shared memory.  Used by
// median_kernel (one tile per CTA) and the persistent batch kernel.
template <typename T>
__device__ __forceinline__ void median_tile(const MedianArgs& a, int TX, int TY, int bx, int by, float* tile_raw) {
    using V = typename median_detail::Store<T>::type;
    V* tile = reinterpret_cast<V*>(tile_raw);
    const int k = a.ksize, r = k / 2;
    const int RY = TY + k - 1;
    const int SW = TX + (k - 1) * a.C;
    const int q0 = bx * TX, y0 = by * TY;
    load_tile<T, V>(tile, RY, SW, a.src, a.spitch, a.W, a.H, a.C, q0 - r * a.C, y0 - r, a.border, V(0));
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        V m;
        if (k == 3) m = median_detail::median_small<3>(tile, SW, y, t, a.C);
        else if (k == 5) m = median_detail::median_small<5>(tile, SW, y, t, a.C);
        else m = median_detail::median_radix<T>(tile, SW, y, t, a.C, k);
        row_ptr_mut<T>(a.dst, a.dpitch, gy)[gq] = static_cast<T>(m);
    }
    __syncthreads();
}
}  // namespace ipfc
