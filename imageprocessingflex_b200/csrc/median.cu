// median.cu -- launcher of the k x k median kernel (tile code: median.cuh).
#include "median.cuh"
#include "median_u8.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads) median_kernel(const MedianArgs a, int TX, int TY) {
    extern __shared__ __align__(16) float tile[];
    median_tile<T>(a, TX, TY, blockIdx.x, blockIdx.y, tile);
}

// uint8 with k = 3 or 5: the packed tile (median_u8.cuh).
__global__ void __launch_bounds__(kMedianU8Threads) median_u8_kernel(const MedianArgs a, int TX, int TY) {
    extern __shared__ __align__(128) unsigned char smem_u8[];
    median_u8_tile(a, TX, TY, blockIdx.x, blockIdx.y, smem_u8);
}

cudaError_t median_u8(const MedianArgs& a, cudaStream_t s) {
    const int TX = 128, TY = 32;
    const size_t smem = median_u8_tile_bytes(TX, TY, a.ksize, a.C);
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)median_u8_kernel, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    median_u8_kernel<<<grid, kMedianU8Threads, smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

template <typename T>
cudaError_t median_typed(const MedianArgs& a, cudaStream_t s) {
    constexpr size_t es = sizeof(typename median_detail::Store<T>::type);
    int TX = 128, TY = 32;
    size_t smem;
    for (;;) {
        smem = median_tile_bytes(TX, TY, a.ksize, a.C, es);
        if (smem <= 96 * 1024 || TY <= 1) break;
        TY /= 2;
    }
    while (smem > 96 * 1024 && TX > 32) {
        TX /= 2;
        smem = median_tile_bytes(TX, TY, a.ksize, a.C, es);
    }
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)median_kernel<T>, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    median_kernel<T><<<grid, kThreads, smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

}  // namespace

cudaError_t median_launch(int dt, const MedianArgs& a, cudaStream_t s) {
    if (dt == IPFC_U8 && (a.ksize == 3 || a.ksize == 5) && median_u8_tile_bytes(128, 32, a.ksize, a.C) <= 96 * 1024)
        return median_u8(a, s);
    switch (dt) {
        case IPFC_U8: return median_typed<uint8_t>(a, s);
        case IPFC_U16: return median_typed<uint16_t>(a, s);
        case IPFC_I16: return median_typed<int16_t>(a, s);
        case IPFC_I32: return median_typed<int32_t>(a, s);
        case IPFC_F32: return median_typed<float>(a, s);
        case IPFC_F64: return median_typed<double>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ipfc
