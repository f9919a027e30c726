// filter2d.cu -- dense 2-D correlation on the CUDA cores, FP32 accumulation.
//
// filter2D (include/ipf/filter.hpp:159-194): out = saturate(delta +
// sum over non-zero taps w(i,j) * P(x + i - ax, y + j - ay)), taps float32,
// zero taps skipped (so an Inf/NaN source sample under a zero tap does not
// reach the sum, as in the reference), P border-extended with borderValue
// under Constant.
//
// One CTA owns a TX x TY output tile; the source tile with its halo is staged
// in shared memory with the border resolved at load.  Each thread produces
// kRows vertically adjacent outputs of one column, so every tap weight read
// (a warp-uniform, L1-broadcast load) feeds kRows FMAs.
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

template <typename Tin, typename Tout>
cudaError_t f2d_typed(const F2DArgs& a, cudaStream_t s) {
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
