// common.cuh -- device-side helpers shared by every neighbourhood kernel.
//
// Element types, border-index resolution and saturating stores with ipf's
// rounding rule.  Written for sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/ipfc.h"

namespace ipfc {

// ---------------------------------------------------------------------------
// Border index.  Same mapping as ipf::borderIndex (include/ipf/core.hpp:187-214):
// Constant -> -1, Replicate clamps, Reflect mirrors with the edge sample
// repeated (period 2n), Reflect101 mirrors without it (period 2n-2, n==1 -> 0),
// Wrap is periodic.  Works for p arbitrarily far outside [0, n).
// ---------------------------------------------------------------------------
// 16-byte asynchronous copy global -> shared, both addresses 16-byte
// aligned, through L2 only.  No register holds the data, so a thread can
// have many in flight; cp_async_wait_all() waits for all of its own.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__host__ __device__ __forceinline__ int border_index(int p, int n, int mode) {
    if ((unsigned)p < (unsigned)n) return p;
    if (n <= 0) return -1;
    switch (mode) {
        case IPFC_BORDER_REPLICATE:
            return p < 0 ? 0 : n - 1;
        case IPFC_BORDER_REFLECT: {
            const int per = 2 * n;
            int q = p % per;
            q += (q < 0) ? per : 0;
            return q < n ? q : per - 1 - q;
        }
        case IPFC_BORDER_REFLECT101: {
            if (n == 1) return 0;
            const int per = 2 * n - 2;
            int q = p % per;
            q += (q < 0) ? per : 0;
            return q < n ? q : per - q;
        }
        case IPFC_BORDER_WRAP: {
            int q = p % n;
            return q < 0 ? q + n : q;
        }
        default:
            return -1;
    }
}

// Floor division for possibly negative numerators (positive divisor).
__host__ __device__ __forceinline__ int floor_div(int a, int b) {
    const int q = a / b;
    return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

// Resolves a flat interleaved sample index s = x*C + c of a row of `width`
// pixels to the flat index of its border source, or -1 (Constant outside).
__host__ __device__ __forceinline__ int border_sample(int s, int width, int C, int mode) {
    const int x = floor_div(s, C);
    const int c = s - x * C;
    const int sx = border_index(x, width, mode);
    return sx < 0 ? -1 : sx * C + c;
}

// ---------------------------------------------------------------------------
// Element traits: load any supported element as float (exact for u8, u16,
// i16), store from float with ipf::saturate_cast semantics
// (core.hpp:69-103): round half away from zero, clamp, NaN -> 0.
// ---------------------------------------------------------------------------
template <typename T> struct Elem;
template <> struct Elem<uint8_t> {
    static constexpr int code = IPFC_U8;
    static constexpr float lo = 0.f, hi = 255.f;
    static constexpr bool is_int = true;
};
template <> struct Elem<uint16_t> {
    static constexpr int code = IPFC_U16;
    static constexpr float lo = 0.f, hi = 65535.f;
    static constexpr bool is_int = true;
};
template <> struct Elem<int16_t> {
    static constexpr int code = IPFC_I16;
    static constexpr float lo = -32768.f, hi = 32767.f;
    static constexpr bool is_int = true;
};
template <> struct Elem<int32_t> {
    static constexpr int code = IPFC_I32;
    static constexpr float lo = -2147483648.f, hi = 2147483647.f;  // float form: not used for rounding
    static constexpr double dlo = -2147483648.0, dhi = 2147483647.0;
    static constexpr bool is_int = true;
};
template <> struct Elem<float> {
    static constexpr int code = IPFC_F32;
    static constexpr float lo = -3.402823466e38f, hi = 3.402823466e38f;
    static constexpr bool is_int = false;
};
template <> struct Elem<double> {
    static constexpr int code = IPFC_F64;
    static constexpr bool is_int = false;
};

// Accumulator of the generic kernels: FP64 when either side is a 32-bit
// integer or double image (the reference accumulates in FP64 throughout; FP32
// cannot hold int32 samples exactly), FP32 otherwise.
template <typename Tin, typename Tout>
struct AccOf {
    static constexpr bool wide = std::is_same<Tin, int32_t>::value || std::is_same<Tin, double>::value ||
                                 std::is_same<Tout, int32_t>::value || std::is_same<Tout, double>::value;
    using type = typename std::conditional<wide, double, float>::type;
};

template <typename T>
__device__ __forceinline__ float to_f(T v) {
    return static_cast<float>(v);
}

// Round half away from zero.  truncf() is exact; the remainder x - t is exact
// for |x| < 2^24 and for larger |x| it is 0, so no rounding step is involved.
__host__ __device__ __forceinline__ float round_half_away(float x) {
    const float t = truncf(x);
    return fabsf(x - t) >= 0.5f ? t + copysignf(1.0f, x) : t;
}

template <typename T>
__host__ __device__ __forceinline__ T sat_from_f(float v) {
    if constexpr (Elem<T>::is_int) {
        // fmaxf/fminf return the non-NaN operand, so NaN lands on lo or hi:
        // pin NaN to 0 explicitly as the reference does.
        float r = round_half_away(v);
        r = fminf(fmaxf(r, Elem<T>::lo), Elem<T>::hi);
        if (v != v) r = 0.f;
        return static_cast<T>(static_cast<int>(r));
    } else {
        return static_cast<T>(v);
    }
}

// saturate_cast<T>(double) exactly as the reference evaluates it
// (include/ipf/core.hpp:69-103): NaN -> 0; integers add -0.5 or +0.5 in FP64
// (one rounding, as in the reference), saturate at the type's limits, then
// truncate toward zero; float narrows with round-to-nearest; double is kept.
template <typename T>
__host__ __device__ __forceinline__ T sat_from_d(double v) {
    if constexpr (std::is_same<T, double>::value) {
        return v;
    } else if constexpr (std::is_same<T, float>::value) {
        return static_cast<float>(v);
    } else {
        if (!(v == v)) return T(0);
        double lo, hi;
        if constexpr (std::is_same<T, int32_t>::value) {
            lo = Elem<T>::dlo;
            hi = Elem<T>::dhi;
        } else {
            lo = (double)Elem<T>::lo;
            hi = (double)Elem<T>::hi;
        }
        const double d = v < 0 ? v - 0.5 : v + 0.5;
        if (d <= lo) return static_cast<T>(lo);
        if (d >= hi) return static_cast<T>(hi);
        return static_cast<T>(d);
    }
}

// Row pointer helper for pitched images.
template <typename T>
__device__ __forceinline__ const T* row_ptr(const void* base, long long pitch, int y) {
    return reinterpret_cast<const T*>(static_cast<const char*>(base) + (long long)y * pitch);
}
template <typename T>
__device__ __forceinline__ T* row_ptr_mut(void* base, long long pitch, int y) {
    return reinterpret_cast<T*>(static_cast<char*>(base) + (long long)y * pitch);
}

}  // namespace ipfc
