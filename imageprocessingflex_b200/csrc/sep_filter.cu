// sep_filter.cu -- separable correlation and box filter, generic forms.
//
// Semantics follow detail::sepFilterImpl (include/ipf/filter.hpp:37-90):
// out = saturate(delta + sum_j ky[j] * sum_i kx[i] * P(x + i - ax, y + j - ay))
// with P the border-extended source; Constant rows and columns read
// borderValue.  Channels are independent: on the interleaved row, tap i sits
// i*C samples away (filter.hpp:67-71).
//
// Generic fused form: one CTA owns a TX-sample x TY-row output tile.  The
// source tile with its halo is staged in shared memory with the border
// resolved at load (tile.cuh); the row pass writes an FP32 intermediate tile
// in shared memory; the column pass reads it and stores saturated outputs.
// Nothing but the source and the destination touches global memory.
//
// Two-pass form (taps longer than kSepMaxParamTaps or a halo that does not fit
// in shared memory): a row pass into an FP32 scratch image of H rows, then a
// column pass that resolves the vertical border through border_index.
#include "sep_filter.cuh"
#include "tile.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;

struct FusedGeom {
    int TX, TY;
    size_t smem;
};

FusedGeom fused_geom(const SepArgs& a, size_t esize) {
    FusedGeom g{128, 32, 0};
    for (;;) {
        const int RY = g.TY + a.kh - 1, SW = g.TX + (a.kw - 1) * a.C;
        g.smem = esize * ((size_t)RY * SW + (size_t)RY * g.TX);
        if (g.smem <= 96 * 1024 || g.TY <= 4) return g;
        g.TY /= 2;
    }
}

// One multiply-add of the accumulation.  FP32: fused.  FP64: a rounded
// product then a rounded sum, the reference's own sequence (it is built
// without FMA contraction), so FP64 results match it bit for bit.
__device__ __forceinline__ float acc_madd(float acc, float k, float x) { return fmaf(k, x, acc); }
__device__ __forceinline__ double acc_madd(double acc, double k, double x) {
    return __dadd_rn(acc, __dmul_rn(k, x));
}

template <typename Tacc> __device__ __forceinline__ Tacc tap_x(const SepArgs& a, int i);
template <> __device__ __forceinline__ float tap_x<float>(const SepArgs& a, int i) { return a.kx[i]; }
template <> __device__ __forceinline__ double tap_x<double>(const SepArgs& a, int i) { return a.kxd[i]; }
template <typename Tacc> __device__ __forceinline__ Tacc tap_y(const SepArgs& a, int j);
template <> __device__ __forceinline__ float tap_y<float>(const SepArgs& a, int j) { return a.ky[j]; }
template <> __device__ __forceinline__ double tap_y<double>(const SepArgs& a, int j) { return a.kyd[j]; }

template <typename Tout>
__device__ __forceinline__ Tout sat_acc(float v) { return sat_from_f<Tout>(v); }
template <typename Tout>
__device__ __forceinline__ Tout sat_acc(double v) { return sat_from_d<Tout>(v); }

template <typename Tin, typename Tout, typename Tacc>
__global__ void __launch_bounds__(kThreads) sep_fused_kernel(const SepArgs a, int TX, int TY) {
    extern __shared__ __align__(16) unsigned char smem_raw_sep[];
    Tacc* smem = reinterpret_cast<Tacc*>(smem_raw_sep);
    const int RY = TY + a.kh - 1;
    const int SW = TX + (a.kw - 1) * a.C;
    Tacc* tin = smem;
    Tacc* th = smem + (size_t)RY * SW;
    const int rowlen = a.W * a.C;
    const int q0 = blockIdx.x * TX;
    const int y0 = blockIdx.y * TY;
    const Tacc bv = std::is_same<Tacc, double>::value ? (Tacc)a.bvd : (Tacc)a.bv;
    load_tile<Tin, Tacc>(tin, RY, SW, a.src, a.spitch, a.W, a.H, a.C, q0 - a.ax * a.C, y0 - a.ay, a.border, bv);
    __syncthreads();
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < RY * TX; idx += nt) {
        const int r = idx / TX, t = idx - r * TX;
        const Tacc* p = tin + (size_t)r * SW + t;
        Tacc acc = 0;
        for (int i = 0; i < a.kw; ++i) acc = acc_madd(acc, tap_x<Tacc>(a, i), p[i * a.C]);
        th[idx] = acc;
    }
    __syncthreads();
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const Tacc* p = th + (size_t)y * TX + t;
        Tacc acc = std::is_same<Tacc, double>::value ? (Tacc)a.deltad : (Tacc)a.delta;
        for (int j = 0; j < a.kh; ++j) acc = acc_madd(acc, tap_y<Tacc>(a, j), p[(size_t)j * TX]);
        row_ptr_mut<Tout>(a.dst, a.dpitch, gy)[gq] = sat_acc<Tout>(acc);
    }
}

// Row pass of the two-pass form: h[y][q] for every in-image row y.
template <typename Tin, typename Tacc>
__global__ void __launch_bounds__(kThreads) sep_rows_kernel(const SepArgs a, const Tacc* __restrict__ kx,
                                                            Tacc* __restrict__ h) {
    const int rowlen = a.W * a.C;
    const int y = blockIdx.y;
    const Tin* srow = row_ptr<Tin>(a.src, a.spitch, y);
    const Tacc bv = std::is_same<Tacc, double>::value ? (Tacc)a.bvd : (Tacc)a.bv;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) {
        Tacc acc = 0;
        const int base = q - a.ax * a.C;
        for (int i = 0; i < a.kw; ++i) {
            const int g = base + i * a.C;
            const int idx = ((unsigned)g < (unsigned)rowlen) ? g : border_sample(g, a.W, a.C, a.border);
            acc = acc_madd(acc, kx[i], idx < 0 ? bv : static_cast<Tacc>(srow[idx]));
        }
        h[(size_t)y * rowlen + q] = acc;
    }
}

// Column pass: a row outside the image reads borderValue * sum(kx) (the row
// pass of a row that is borderValue everywhere), accumulated in tap order.
template <typename Tout, typename Tacc>
__global__ void __launch_bounds__(kThreads) sep_cols_kernel(const SepArgs a, const Tacc* __restrict__ kx,
                                                            const Tacc* __restrict__ ky,
                                                            const Tacc* __restrict__ h) {
    const int rowlen = a.W * a.C;
    const int y = blockIdx.y;
    const Tacc bv = std::is_same<Tacc, double>::value ? (Tacc)a.bvd : (Tacc)a.bv;
    Tacc const_row = 0;
    for (int i = 0; i < a.kw; ++i) const_row = acc_madd(const_row, kx[i], bv);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) {
        Tacc acc = std::is_same<Tacc, double>::value ? (Tacc)a.deltad : (Tacc)a.delta;
        for (int j = 0; j < a.kh; ++j) {
            const int sy = border_index(y + j - a.ay, a.H, a.border);
            acc = acc_madd(acc, ky[j], sy < 0 ? const_row : h[(size_t)sy * rowlen + q]);
        }
        row_ptr_mut<Tout>(a.dst, a.dpitch, y)[q] = sat_acc<Tout>(acc);
    }
}

template <typename Tin, typename Tout, typename Tacc>
cudaError_t launch_acc(const SepArgs& a, const void* dkx, const void* dky, void* scratch, cudaStream_t s) {
    const int rowlen = a.W * a.C;
    if (!sep_needs_scratch(a, std::is_same<Tacc, double>::value)) {
        const FusedGeom g = fused_geom(a, sizeof(Tacc));
        static unsigned done = 0;  // per instantiation, one bit per device
        cudaError_t e = ensure_smem_attr((const void*)sep_fused_kernel<Tin, Tout, Tacc>, 96 * 1024, &done);
        if (e != cudaSuccess) return e;
        dim3 grid((rowlen + g.TX - 1) / g.TX, (a.H + g.TY - 1) / g.TY);
        dim3 block(32, kThreads / 32);
        sep_fused_kernel<Tin, Tout, Tacc><<<grid, block, g.smem, s>>>(a, g.TX, g.TY);
        return cudaGetLastError();
    }
    if (!dkx || !dky || !scratch) return cudaErrorInvalidValue;
    const int bx = (rowlen + kThreads - 1) / kThreads;
    dim3 grid(bx < 64 ? bx : 64, a.H);
    sep_rows_kernel<Tin, Tacc><<<grid, kThreads, 0, s>>>(a, static_cast<const Tacc*>(dkx), static_cast<Tacc*>(scratch));
    sep_cols_kernel<Tout, Tacc><<<grid, kThreads, 0, s>>>(a, static_cast<const Tacc*>(dkx),
                                                          static_cast<const Tacc*>(dky),
                                                          static_cast<const Tacc*>(scratch));
    return cudaGetLastError();
}

// Accumulator: FP64 for int32 / double images or when asked, FP32 otherwise.
template <typename Tin, typename Tout>
cudaError_t launch_typed(const SepArgs& a, const void* dkx, const void* dky, void* scratch, cudaStream_t s,
                         bool fp64) {
    if constexpr (AccOf<Tin, Tout>::wide) {
        return launch_acc<Tin, Tout, double>(a, dkx, dky, scratch, s);
    } else {
        if (fp64) return launch_acc<Tin, Tout, double>(a, dkx, dky, scratch, s);
        return launch_acc<Tin, Tout, float>(a, dkx, dky, scratch, s);
    }
}

template <typename Tin>
cudaError_t launch_out(int ddt, const SepArgs& a, const void* dkx, const void* dky, void* scratch, cudaStream_t s,
                       bool fp64) {
    switch (ddt) {
        case IPFC_U8: return launch_typed<Tin, uint8_t>(a, dkx, dky, scratch, s, fp64);
        case IPFC_U16: return launch_typed<Tin, uint16_t>(a, dkx, dky, scratch, s, fp64);
        case IPFC_I16: return launch_typed<Tin, int16_t>(a, dkx, dky, scratch, s, fp64);
        case IPFC_I32: return launch_typed<Tin, int32_t>(a, dkx, dky, scratch, s, fp64);
        case IPFC_F32: return launch_typed<Tin, float>(a, dkx, dky, scratch, s, fp64);
        case IPFC_F64: return launch_typed<Tin, double>(a, dkx, dky, scratch, s, fp64);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool sep_needs_scratch(const SepArgs& a, bool wide) {
    if (a.kw > kSepMaxParamTaps || a.kh > kSepMaxParamTaps) return true;
    return fused_geom(a, wide ? sizeof(double) : sizeof(float)).smem > 96 * 1024;
}

cudaError_t sep_launch(int sdt, int ddt, const SepArgs& a, const void* dkx, const void* dky, void* scratch,
                       cudaStream_t s, bool force_fp64) {
    switch (sdt) {
        case IPFC_U8: return launch_out<uint8_t>(ddt, a, dkx, dky, scratch, s, force_fp64);
        case IPFC_U16: return launch_out<uint16_t>(ddt, a, dkx, dky, scratch, s, force_fp64);
        case IPFC_I16: return launch_out<int16_t>(ddt, a, dkx, dky, scratch, s, force_fp64);
        case IPFC_I32: return launch_out<int32_t>(ddt, a, dkx, dky, scratch, s, force_fp64);
        case IPFC_F32: return launch_out<float>(ddt, a, dkx, dky, scratch, s, force_fp64);
        case IPFC_F64: return launch_out<double>(ddt, a, dkx, dky, scratch, s, force_fp64);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Box filter (filter.hpp:206-253).  The reference sums the window in FP64 with
// running sums and multiplies by fl64(1/(kw*kh)).  For integer sources every
// sum is an integer, so here it is formed exactly in int32 and the rounding is
// done on the exact quotient; the only inputs where the FP64 product can round
// differently from the exact quotient are exact ties S/n = t + 1/2 (n even),
// whose outcome the host precomputes per t with the reference's own double
// expression into tie_up.  Float destinations get fl32 of S * fl64(1/n)
// through a two-float product.  Float sources are summed in FP32.
// ---------------------------------------------------------------------------
namespace {

template <typename Tin, typename Tout, typename Tacc>
__global__ void __launch_bounds__(kThreads) box_kernel(const BoxArgs a, int TX, int TY) {
    extern __shared__ unsigned char smem_raw[];
    Tacc* tin = reinterpret_cast<Tacc*>(smem_raw);
    const int RY = TY + a.kh - 1;
    const int SW = TX + (a.kw - 1) * a.C;
    Tacc* th = tin + (size_t)RY * SW;
    const int rowlen = a.W * a.C;
    const int q0 = blockIdx.x * TX;
    const int y0 = blockIdx.y * TY;
    load_tile<Tin, Tacc>(tin, RY, SW, a.src, a.spitch, a.W, a.H, a.C, q0 - a.ax * a.C, y0 - a.ay, a.border,
                         std::is_same<Tacc, double>::value ? static_cast<Tacc>(a.bvd) : static_cast<Tacc>(a.bv));
    __syncthreads();
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nt = blockDim.x * blockDim.y;
    for (int idx = tid; idx < RY * TX; idx += nt) {
        const int r = idx / TX, t = idx - r * TX;
        const Tacc* p = tin + (size_t)r * SW + t;
        Tacc acc = 0;
        for (int i = 0; i < a.kw; ++i) acc += p[i * a.C];
        th[idx] = acc;
    }
    __syncthreads();
    const int n = a.kw * a.kh;
    for (int idx = tid; idx < TY * TX; idx += nt) {
        const int y = idx / TX, t = idx - y * TX;
        const int gy = y0 + y, gq = q0 + t;
        if (gy >= a.H || gq >= rowlen) continue;
        const Tacc* p = th + (size_t)y * TX + t;
        Tacc S = 0;
        for (int j = 0; j < a.kh; ++j) S += p[(size_t)j * TX];
        Tout out;
        if constexpr (std::is_same<Tacc, int>::value) {
            if (!a.normalize) {
                if constexpr (Elem<Tout>::is_int) {
                    const int lo = (int)Elem<Tout>::lo, hi = (int)Elem<Tout>::hi;
                    out = static_cast<Tout>(S < lo ? lo : (S > hi ? hi : S));
                } else {
                    out = static_cast<Tout>(S);
                }
            } else if constexpr (Elem<Tout>::is_int) {
                const int mag = S < 0 ? -S : S;
                int tq = mag / n;
                const int r2 = 2 * (mag - tq * n);
                if (r2 > n) {
                    ++tq;
                } else if (r2 == n) {
                    const bool up = tq >= 65536 ? true : ((a.tie_up[tq >> 5] >> (tq & 31)) & 1u);
                    tq += up ? 1 : 0;
                }
                const int v = S < 0 ? -tq : tq;
                const int lo = (int)Elem<Tout>::lo, hi = (int)Elem<Tout>::hi;
                out = static_cast<Tout>(v < lo ? lo : (v > hi ? hi : v));
            } else {
                const float fs = static_cast<float>(S);
                const float p0 = fs * a.scale_hi;
                const float e = fmaf(fs, a.scale_hi, -p0);
                out = static_cast<Tout>(p0 + fmaf(fs, a.scale_lo, e));
            }
        } else if constexpr (std::is_same<Tacc, double>::value) {
            // the reference's sum times fl64(1/(kw*kh)), one rounding
            out = sat_from_d<Tout>(a.normalize ? __dmul_rn(S, a.scaled) : S);
        } else {
            const float v = a.normalize ? S * (a.scale_hi + a.scale_lo) : S;
            out = sat_from_f<Tout>(v);
        }
        row_ptr_mut<Tout>(a.dst, a.dpitch, gy)[gq] = out;
    }
}

template <typename Tin, typename Tout, typename Tacc>
cudaError_t box_typed(const BoxArgs& a, cudaStream_t s) {
    int TX = 128, TY = 32;
    size_t smem;
    for (;;) {
        const int RY = TY + a.kh - 1, SW = TX + (a.kw - 1) * a.C;
        smem = sizeof(Tacc) * ((size_t)RY * SW + (size_t)RY * TX);
        if (smem <= 96 * 1024 || TY <= 1) break;
        TY /= 2;
    }
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)box_kernel<Tin, Tout, Tacc>, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    box_kernel<Tin, Tout, Tacc><<<grid, dim3(32, kThreads / 32), smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

template <typename Tin, typename Tacc>
cudaError_t box_out(int ddt, const BoxArgs& a, cudaStream_t s) {
    switch (ddt) {
        case IPFC_U8: return box_typed<Tin, uint8_t, Tacc>(a, s);
        case IPFC_U16: return box_typed<Tin, uint16_t, Tacc>(a, s);
        case IPFC_I16: return box_typed<Tin, int16_t, Tacc>(a, s);
        case IPFC_F32: return box_typed<Tin, float, Tacc>(a, s);
        case IPFC_I32: return box_typed<Tin, int32_t, double>(a, s);
        case IPFC_F64: return box_typed<Tin, double, double>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t box_launch(int sdt, int ddt, const BoxArgs& a, bool exact_int, cudaStream_t s, bool force_fp64) {
    if (force_fp64 || sep_wide(sdt, ddt)) {  // FP64 sums
        switch (sdt) {
            case IPFC_U8: return box_out<uint8_t, double>(ddt, a, s);
            case IPFC_U16: return box_out<uint16_t, double>(ddt, a, s);
            case IPFC_I16: return box_out<int16_t, double>(ddt, a, s);
            case IPFC_I32: return box_out<int32_t, double>(ddt, a, s);
            case IPFC_F32: return box_out<float, double>(ddt, a, s);
            case IPFC_F64: return box_out<double, double>(ddt, a, s);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (sdt) {
        case IPFC_U8: return exact_int ? box_out<uint8_t, int>(ddt, a, s) : box_out<uint8_t, float>(ddt, a, s);
        case IPFC_U16: return exact_int ? box_out<uint16_t, int>(ddt, a, s) : box_out<uint16_t, float>(ddt, a, s);
        case IPFC_I16: return exact_int ? box_out<int16_t, int>(ddt, a, s) : box_out<int16_t, float>(ddt, a, s);
        case IPFC_F32: return box_out<float, float>(ddt, a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned bit = dev >= 0 && dev < 32 ? 1u << dev : 0u;  // devices past 32 are set every call
    if (__atomic_load_n(done_mask, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) __atomic_fetch_or(done_mask, bit, __ATOMIC_ACQ_REL);
    return e;
}

}  // namespace ipfc
