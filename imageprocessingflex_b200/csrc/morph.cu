// morph.cu -- grey erosion / dilation (include/ipf/morphology.hpp:53-127).
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
#include "kernels.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ void load_morph_tile(float* tile, int RY, int SW, const MorphArgs& a, int gq0, int gy0,
                                                float identity) {
    const int rowlen = a.W * a.C;
    for (int r = threadIdx.y; r < RY; r += blockDim.y) {
        const int gy = gy0 + r;
        float* dst = tile + (size_t)r * SW;
        if ((unsigned)gy >= (unsigned)a.H) {
            for (int s = threadIdx.x; s < SW; s += blockDim.x) dst[s] = identity;
            continue;
        }
        const T* srow = row_ptr<T>(a.src, a.spitch, gy);
        for (int s = threadIdx.x; s < SW; s += blockDim.x) {
            const int g = gq0 + s;
            dst[s] = ((unsigned)g < (unsigned)rowlen) ? to_f(srow[g]) : identity;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) morph_kernel(const MorphArgs a, int TX, int TY) {
    extern __shared__ float smem[];
    const int RY = TY + a.sh - 1;
    const int SW = TX + (a.sw - 1) * a.C;
    float* tile = smem;
    const int q0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const float identity = a.is_min ? __int_as_float(0x7f800000) : __int_as_float(0xff800000);
    load_morph_tile<T>(tile, RY, SW, a, q0 - a.ax * a.C, y0 - a.ay, identity);
    __syncthreads();
    const int rowlen = a.W * a.C;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nt = blockDim.x * blockDim.y;
    if (a.is_rect) {
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
        return;
    }
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
}

template <typename T>
cudaError_t morph_typed(const MorphArgs& a, cudaStream_t s) {
    int TX = 128, TY = 32;
    size_t smem;
    for (;;) {
        const int RY = TY + a.sh - 1, SW = TX + (a.sw - 1) * a.C;
        smem = sizeof(float) * ((size_t)RY * SW + (a.is_rect ? (size_t)RY * TX : 0));
        if (smem <= 96 * 1024 || TY <= 1) break;
        TY /= 2;
    }
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)morph_kernel<T>, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    morph_kernel<T><<<grid, dim3(32, kThreads / 32), smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

}  // namespace

cudaError_t morph_launch(int dt, const MorphArgs& a, cudaStream_t s) {
    switch (dt) {
        case IPFC_U8: return morph_typed<uint8_t>(a, s);
        case IPFC_U16: return morph_typed<uint16_t>(a, s);
        case IPFC_I16: return morph_typed<int16_t>(a, s);
        case IPFC_F32: return morph_typed<float>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ipfc
