// morph.cu -- launcher of the erosion / dilation kernel (tile code: morph.cuh).
#include "morph.cuh"
#include "morph_u8.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;
constexpr int kMorphU8VhgwFrom = 11;  // uint8 rect members per axis from which the generic tile takes over

template <typename T>
__global__ void __launch_bounds__(kThreads) morph_kernel(const MorphArgs a, int TX, int TY) {
    extern __shared__ __align__(16) float smem[];
    if (a.is_rect) morph_rect_tile<T>(a, TX, TY, blockIdx.x, blockIdx.y, smem);
    else morph_list_tile<T>(a, TX, TY, blockIdx.x, blockIdx.y, smem);
}

// uint8 with an all-ones element: the packed-byte tile (morph_u8.cuh).
__global__ void __launch_bounds__(kMorphU8Threads) morph_u8_kernel(const MorphCore a, int TX, int TY) {
    extern __shared__ __align__(128) unsigned char smem_u8[];
    morph_u8_tile(a, TX, TY, blockIdx.x, blockIdx.y, smem_u8);
}

cudaError_t morph_u8_rect(const MorphCore& a, cudaStream_t s) {
    const int TX = 256, TY = 32;
    const size_t smem = morph_u8_tile_bytes(TX, TY, a.sw, a.sh, a.C);
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)morph_u8_kernel, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    morph_u8_kernel<<<grid, kMorphU8Threads, smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

template <typename T>
cudaError_t morph_typed(const MorphArgs& a, cudaStream_t s) {
    constexpr size_t es = sizeof(typename MorphStore<T>::type);
    int TX = 128, TY = 32;
    size_t smem;
    for (;;) {
        smem = morph_tile_bytes(TX, TY, a.sw, a.sh, a.C, a.is_rect != 0, es);
        if (smem <= 96 * 1024 || TY <= 1) break;
        TY /= 2;
    }
    while (smem > 96 * 1024 && TX > 32) {
        TX /= 2;
        smem = morph_tile_bytes(TX, TY, a.sw, a.sh, a.C, a.is_rect != 0, es);
    }
    if (smem > 96 * 1024) return cudaErrorInvalidConfiguration;
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)morph_kernel<T>, 96 * 1024, &done);
    if (e != cudaSuccess) return e;
    const int rowlen = a.W * a.C;
    dim3 grid((rowlen + TX - 1) / TX, (a.H + TY - 1) / TY);
    morph_kernel<T><<<grid, kThreads, smem, s>>>(a, TX, TY);
    return cudaGetLastError();
}

}  // namespace

bool morph3_stream_launch(const MorphCore& a, cudaStream_t s, cudaError_t* e);

cudaError_t morph_launch(int dt, const MorphArgs& a, cudaStream_t s) {
    // uint8, the 3 x 3 element with 16-byte aligned rows: the streaming
    // kernel (morph3_stream.cu), no shared-memory staging
    if (dt == IPFC_U8) {
        cudaError_t e = cudaSuccess;
        if (morph3_stream_launch(a, s, &e)) return e;
    }
    // uint8 rectangles: the packed-byte tile's direct scans up to 9 members
    // per axis; longer ones run van Herk / Gil-Werman in the generic tile
    if (dt == IPFC_U8 && a.is_rect && a.sw < kMorphU8VhgwFrom && a.sh < kMorphU8VhgwFrom &&
        morph_u8_tile_bytes(256, 32, a.sw, a.sh, a.C) <= 96 * 1024)
        return morph_u8_rect(a, s);
    switch (dt) {
        case IPFC_U8: return morph_typed<uint8_t>(a, s);
        case IPFC_U16: return morph_typed<uint16_t>(a, s);
        case IPFC_I16: return morph_typed<int16_t>(a, s);
        case IPFC_I32: return morph_typed<int32_t>(a, s);
        case IPFC_F32: return morph_typed<float>(a, s);
        case IPFC_F64: return morph_typed<double>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ipfc
