// filter2d.cu -- dense 2-D correlation on the CUDA cores, FP32 accumulation.
//
// filter2D (include/ipf/filter.hpp:159-194): out = saturate(delta +
// sum over non-zero taps w(i,j) * P(x + i - ax, y + j - ay)), taps float32,
// zero taps skipped (so an Inf/NaN source sample under a zero tap does not
// reach the sum, as in the reference), P border-extended with borderValue
// under Constant.
//
// One CTA owns a TX x TY output tile; the source tile with its halo is staged
// in shared memory with the border resolved at load.  Two FP32 forms: the
// register-tiled one (below) for the kernel sizes it is built for, and the
// general one, where each thread produces kRows vertically adjacent outputs
// of one column so every tap weight read (a warp-uniform, L1-broadcast load)
// feeds kRows FMAs.
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"
#include "tile.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;
constexpr int kRows = 4;

template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kThreads) filter2d_kernel(const F2DArgs a, int TX, int TY) {
    extern __shared__ float tile[];
    const int RY = TY + a.kh - 1;
    const int SW = TX + (a.kw - 1) * a.C;
    const int q0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    load_tile<Tin, float>(tile, RY, SW, a.src, a.spitch, a.W, a.H, a.C, q0 - a.ax * a.C, y0 - a.ay, a.border,
                          a.bv);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    const int groups = (TY / kRows) * TX;
    for (int idx = tid; idx < groups; idx += nt) {
        const int yb = (idx / TX) * kRows, t = idx - (idx / TX) * TX;
        float acc[kRows];
#pragma unroll
        for (int r = 0; r < kRows; ++r) acc[r] = a.delta;
        const float* base = tile + (size_t)yb * SW + t;
        for (int k = 0; k < a.ntaps; ++k) {
            const float4 tp = __ldg(a.taps + k);
            const float* p = base + (int)tp.z * SW + (int)tp.y * a.C;
#pragma unroll
            for (int r = 0; r < kRows; ++r) acc[r] = fmaf(tp.x, p[r * SW], acc[r]);
        }
        const int gq = q0 + t;
        if (gq >= rowlen) continue;
#pragma unroll
        for (int r = 0; r < kRows; ++r) {
            const int gy = y0 + yb + r;
            if (gy < a.H) row_ptr_mut<Tout>(a.dst, a.dpitch, gy)[gq] = sat_from_f<Tout>(acc[r]);
        }
    }
}

// FP64 form for int32 and double images: the reference's sum, delta first,
// then each non-zero tap in row-major order as a rounded product and a
// rounded sum (no fused multiply-add), so results match it bit for bit.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kThreads) filter2d_kernel_d(const F2DArgs a, int TX, int TY) {
    extern __shared__ __align__(16) unsigned char f2d_raw[];
    double* tile = reinterpret_cast<double*>(f2d_raw);
    const int RY = TY + a.kh - 1;
    const int SW = TX + (a.kw - 1) * a.C;
    const int q0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    load_tile<Tin, double>(tile, RY, SW, a.src, a.spitch, a.W, a.H, a.C, q0 - a.ax * a.C, y0 - a.ay, a.border,
                           a.bvd);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const double* base = tile + (size_t)y * SW + t;
        double acc = a.deltad;
        for (int k = 0; k < a.ntaps; ++k) {
            const float4 tp = __ldg(a.taps + k);
            acc = __dadd_rn(acc, __dmul_rn((double)tp.x, base[(int)tp.z * SW + (int)tp.y * a.C]));
        }
        row_ptr_mut<Tout>(a.dst, a.dpitch, gy)[gq] = sat_from_d<Tout>(acc);
    }
}

// ---------------------------------------------------------------------------
// Register-tiled form (FP32): each thread owns kRtR rows x kRtP samples of
// outputs.  Per source row of its band it loads one window of the staged
// tile (kRtP + (KWB-1) C samples) into registers with 16-byte shared loads
// and applies the taps of every output row that source row feeds, four taps
// per 16-byte load of the tap table.  Every output still accumulates delta,
// then the taps in row-major order with FMAs -- the CUDA-core form's own
// sequence -- so results are bit-identical to it: zero taps are included,
// which adds exactly zero for finite samples (the caller takes this form for
// integer sources, and for float sources only when no tap is zero).  KWB is
// the tap-row capacity (kw <= KWB, taps past kw are skipped by a uniform
// test), C the channel count (tap i sits i*C samples away).
constexpr int kRtR = 4, kRtP = 8;
constexpr int kRtTX = 128, kRtTY = 64;  // 16 x 16 threads

__host__ __device__ constexpr int rt_row_stride(int kw, int C) { return (kRtTX + (kw - 1) * C + 3) / 4 * 4; }
template <int KWB, int C>
__host__ __device__ constexpr int rt_window() { return (kRtP + (KWB - 1) * C + 3) / 4 * 4; }

template <typename Tin, typename Tout, int KWB, int C>
__global__ void __launch_bounds__(kThreads, 2) filter2d_rt_kernel(const F2DArgs a) {
    extern __shared__ __align__(16) float rt_smem[];
    constexpr int WIN = rt_window<KWB, C>();
    const int SW = rt_row_stride(a.kw, C);
    const int RY = kRtTY + a.kh - 1;
    float* tile = rt_smem;
    float* taps = rt_smem + (size_t)RY * SW + WIN;  // after the tile and the last row's over-read slack
    const int q0 = blockIdx.x * kRtTX, y0 = blockIdx.y * kRtTY;
    // dense tap table [kh][KWB], zero past kw and where the list has no tap
    for (int i = threadIdx.x; i < a.kh * KWB; i += kThreads) taps[i] = 0.f;
    __syncthreads();
    for (int k = threadIdx.x; k < a.ntaps; k += kThreads) {
        const float4 t = __ldg(a.taps + k);
        taps[(int)t.z * KWB + (int)t.y] = t.x;
    }
    load_tile<Tin, float>(tile, RY, SW, a.src, a.spitch, a.W, a.H, C, q0 - a.ax * C, y0 - a.ay, a.border, a.bv);
    // the slack past the last row is read by the last windows and never used
    for (int i = threadIdx.x; i < WIN; i += kThreads) tile[(size_t)RY * SW + i] = 0.f;
    __syncthreads();
    const int tc = threadIdx.x % (kRtTX / kRtP), tr = threadIdx.x / (kRtTX / kRtP);
    float acc[kRtR][kRtP];
#pragma unroll
    for (int r = 0; r < kRtR; ++r)
#pragma unroll
        for (int u = 0; u < kRtP; ++u) acc[r][u] = a.delta;
    const int nsrc = kRtR + a.kh - 1;
    for (int sr = 0; sr < nsrc; ++sr) {
        float win[WIN];
        const float4* p4 = reinterpret_cast<const float4*>(tile + (size_t)(tr * kRtR + sr) * SW + tc * kRtP);
#pragma unroll
        for (int q = 0; q < WIN / 4; ++q) {
            const float4 v = p4[q];
            win[4 * q] = v.x;
            win[4 * q + 1] = v.y;
            win[4 * q + 2] = v.z;
            win[4 * q + 3] = v.w;
        }
#pragma unroll
        for (int r = 0; r < kRtR; ++r) {
            const int j = sr - r;  // tap row feeding output row r from this source row
            if (j < 0 || j >= a.kh) continue;
            const float4* t4 = reinterpret_cast<const float4*>(taps + j * KWB);
#pragma unroll
            for (int i4 = 0; i4 < KWB / 4; ++i4) {
                if (4 * i4 >= a.kw) break;
                const float4 w4 = t4[i4];
                const float w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int i = 4 * i4 + e;
                    if (i >= a.kw) break;
#pragma unroll
                    for (int u = 0; u < kRtP; ++u) acc[r][u] = fmaf(w[e], win[u + i * C], acc[r][u]);
                }
            }
        }
    }
    const int rowlen = a.W * C;
#pragma unroll
    for (int r = 0; r < kRtR; ++r) {
        const int gy = y0 + tr * kRtR + r;
        if (gy >= a.H) continue;
        Tout* drow = row_ptr_mut<Tout>(a.dst, a.dpitch, gy);
#pragma unroll
        for (int u = 0; u < kRtP; ++u) {
            const int gq = q0 + tc * kRtP + u;
            if (gq < rowlen) drow[gq] = sat_from_f<Tout>(acc[r][u]);
        }
    }
}

template <typename Tin, typename Tout, int KWB, int C>
cudaError_t launch_rt(const F2DArgs& a, cudaStream_t s) {
    const size_t smem = sizeof(float) * ((size_t)(kRtTY + a.kh - 1) * rt_row_stride(a.kw, C) + rt_window<KWB, C>() +
                                         (size_t)a.kh * KWB);
    if (smem > 160 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)filter2d_rt_kernel<Tin, Tout, KWB, C>, 160 * 1024, &done);
    if (e != cudaSuccess) return e;
    dim3 grid((a.W * C + kRtTX - 1) / kRtTX, (a.H + kRtTY - 1) / kRtTY);
    filter2d_rt_kernel<Tin, Tout, KWB, C><<<grid, kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

// The register-tiled form where it is built (1 or 3 channels; kernels of
// 9 to 32 taps per row; at most 33 rows) and exact to use (integer source,
// or every tap non-zero); false otherwise.
// IPFC_F2D_TILED=0 turns the register-tiled form off (read once), so tests
// can compare it with the general form.
bool rt_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("IPFC_F2D_TILED");
        return !(v && std::strcmp(v, "0") == 0);
    }();
    return on;
}

template <typename Tin, typename Tout>
bool try_rt(const F2DArgs& a, cudaStream_t s, cudaError_t* e) {
    if (!rt_enabled()) return false;
    constexpr bool built = (std::is_same<Tin, uint8_t>::value || std::is_same<Tin, float>::value) &&
                           (std::is_same<Tout, uint8_t>::value || std::is_same<Tout, float>::value);
    if constexpr (!built) {
        return false;
    } else {
        if (a.kh > 33 || a.kw < 9 || a.kw > 32) return false;
        if (!Elem<Tin>::is_int && !a.dense) return false;
        if (a.C == 1) {
            *e = a.kw <= 16 ? launch_rt<Tin, Tout, 16, 1>(a, s) : launch_rt<Tin, Tout, 32, 1>(a, s);
            return true;
        }
        if (a.C == 3 && a.kw <= 16) {
            *e = launch_rt<Tin, Tout, 16, 3>(a, s);
            return true;
        }
        return false;
    }
}

template <typename Tin, typename Tout>
cudaError_t f2d_typed(const F2DArgs& a, cudaStream_t s) {
    {
        cudaError_t e = cudaSuccess;
        if (try_rt<Tin, Tout>(a, s, &e)) return e;
    }
    constexpr bool wide = AccOf<Tin, Tout>::wide;
    constexpr size_t es = wide ? sizeof(double) : sizeof(float);
    int TX = 128, TY = 32;
    size_t smem;
    for (;;) {
        smem = es * (size_t)(TY + a.kh - 1) * (TX + (a.kw - 1) * a.C);
        if (smem <= 160 * 1024 || TY <= kRows) break;
        TY /= 2;
    }
    while (smem > 160 * 1024 && TX > 32) {
        TX /= 2;
        smem = es * (size_t)(TY + a.kh - 1) * (TX + (a.kw - 1) * a.C);
    }
    if (smem > 160 * 1024) return cudaErrorInvalidConfiguration;
    const void* kern = wide ? (const void*)filter2d_kernel_d<Tin, Tout> : (const void*)filter2d_kernel<Tin, Tout>;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr(kern, 160 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    if constexpr (wide)
        filter2d_kernel_d<Tin, Tout><<<grid, dim3(32, kThreads / 32), smem, s>>>(a, TX, TY);
    else
        filter2d_kernel<Tin, Tout><<<grid, dim3(32, kThreads / 32), smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

template <typename Tin>
cudaError_t f2d_out(int ddt, const F2DArgs& a, cudaStream_t s) {
    switch (ddt) {
        case IPFC_U8: return f2d_typed<Tin, uint8_t>(a, s);
        case IPFC_U16: return f2d_typed<Tin, uint16_t>(a, s);
        case IPFC_I16: return f2d_typed<Tin, int16_t>(a, s);
        case IPFC_I32: return f2d_typed<Tin, int32_t>(a, s);
        case IPFC_F32: return f2d_typed<Tin, float>(a, s);
        case IPFC_F64: return f2d_typed<Tin, double>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t filter2d_launch(int sdt, int ddt, const F2DArgs& a, cudaStream_t s) {
    switch (sdt) {
        case IPFC_U8: return f2d_out<uint8_t>(ddt, a, s);
        case IPFC_U16: return f2d_out<uint16_t>(ddt, a, s);
        case IPFC_I16: return f2d_out<int16_t>(ddt, a, s);
        case IPFC_I32: return f2d_out<int32_t>(ddt, a, s);
        case IPFC_F32: return f2d_out<float>(ddt, a, s);
        case IPFC_F64: return f2d_out<double>(ddt, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ipfc
