// batch_kernel.cuh -- body of the persistent batch kernel, instantiated once
// per register class (batch_light.cu, batch_heavy.cu).
#pragma once

#include "batch.cuh"

namespace ipfc {

// The current tile's item and the tile bodies' buffer: file-scope shared
// variables, so that the out-of-line tile functions below address them as
// shared memory directly.
__shared__ BatchItem g_batch_item;
extern __shared__ __align__(128) float g_batch_smem[];

// Each tile body is its own function: the compiler allocates registers per
// function, and one kernel body with every variant inlined is many times
// slower to compile and no faster to run (a call per tile costs nothing).

static __device__ __noinline__ void batch_median_tile(int x, int y) {
    median_tile<uint8_t>(g_batch_item.u.med, g_batch_item.tx, g_batch_item.ty, x, y, g_batch_smem);
}

// 3x3 and 5x5 (the memory-bound class)
static __device__ __noinline__ void batch_median_u8_tile(int x, int y) {
    median_u8_tile(g_batch_item.u.med, g_batch_item.tx, g_batch_item.ty, x, y,
                   reinterpret_cast<unsigned char*>(g_batch_smem));
}

static __device__ __noinline__ void batch_morph_tile(int x, int y) {
    morph_u8_tile(g_batch_item.u.morph, g_batch_item.tx, g_batch_item.ty, x, y,
                  reinterpret_cast<unsigned char*>(g_batch_smem));
}

// Queue tiles: median k >= 7 (light class), 3x3 / 5x5 median and
// morphology (memory-bound class).  Separable tiles run as group launches.
template <int CLS>
__device__ __forceinline__ void batch_run_tile(int kind, int k, int c, int x, int y) {
    if constexpr (CLS == kBatchLight) {
        batch_median_tile(x, y);
    } else if constexpr (CLS == kBatchMem) {
        if (kind == kBatchMedian) batch_median_u8_tile(x, y);
        else batch_morph_tile(x, y);
    }
}

// ---- separable group launches --------------------------------------------------
template <int K, int C>
__global__ void __launch_bounds__(kFastThreads, K <= kBatchLightMaxTaps ? 2 : 1)
    batch_sep_group_kernel(const __grid_constant__ SepGroup g) {
    const SepFastArgs& a = g.it[blockIdx.y];
    const int chunks = (a.H + a.rows_per_cta - 1) / a.rows_per_cta;
    if ((int)blockIdx.x >= a.strips * chunks) return;  // CTA-uniform
    sep_fast_tile<K, C, uint8_t, uint8_t>(a, g_batch_smem, blockIdx.x % a.strips, blockIdx.x / a.strips);
}

cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

template <int K, int C>
cudaError_t batch_sep_group_launch_kc(const SepGroup& g, int n, int max_tiles, cudaStream_t s) {
    using G = FastGeom<K, C, 4>;
    static unsigned done = 0;  // one bit per device
    cudaError_t e = ensure_smem_attr((const void*)batch_sep_group_kernel<K, C>, (int)G::SMEM, &done);
    if (e != cudaSuccess) return e;
    batch_sep_group_kernel<K, C><<<dim3(max_tiles, n), kFastThreads, G::SMEM, s>>>(g);
    return cudaGetLastError();
}

template <int K>
bool batch_sep_group_case(int k, int c, const SepGroup& g, int n, int max_tiles, cudaStream_t s, cudaError_t* e) {
    if (k != K) return false;
    *e = c == 1   ? batch_sep_group_launch_kc<K, 1>(g, n, max_tiles, s)
         : c == 3 ? batch_sep_group_launch_kc<K, 3>(g, n, max_tiles, s)
                  : batch_sep_group_launch_kc<K, 4>(g, n, max_tiles, s);
    return true;
}

// The tile loop.  Thread 0 takes the next tile index; the whole CTA reads it
// after a barrier, so every exit and item switch is CTA-uniform.
template <int CLS>
__global__ void __launch_bounds__(kFastThreads, CLS == kBatchLight ? 2 : 4)
    batch_kernel(const BatchItem* __restrict__ items, const BatchTile* __restrict__ tiles, int ntiles,
                 unsigned* __restrict__ counter) {
    __shared__ int next;
    int cur = -1;
    for (;;) {
        if (threadIdx.x == 0) next = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = next;
        if (t >= ntiles) break;
        const BatchTile tl = tiles[t];
        if (tl.item != cur) {
            const uint4* from = reinterpret_cast<const uint4*>(items + tl.item);
            uint4* to = reinterpret_cast<uint4*>(&g_batch_item);
            for (int i = threadIdx.x; i < (int)(sizeof(BatchItem) / 16); i += kFastThreads) to[i] = from[i];
            cur = tl.item;
            __syncthreads();
        }
        batch_run_tile<CLS>(g_batch_item.kind, g_batch_item.K, g_batch_item.C, tl.x, tl.y);
        __syncthreads();  // tile done with the item, `next` and the buffer
    }
}

// Opens the kernel to all the dynamic shared memory a block may have (once
// per device): batches differ in what they need.
template <int CLS>
cudaError_t batch_prepare_class() {
    static unsigned done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned bit = 1u << (dev & 31);
    if (__atomic_load_n(&done, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
    int optin = 0;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, (const void*)batch_kernel<CLS>)) != cudaSuccess) return e;
    e = cudaFuncSetAttribute((const void*)batch_kernel<CLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             optin - (int)fa.sharedSizeBytes);
    if (e == cudaSuccess) __atomic_fetch_or(&done, bit, __ATOMIC_ACQ_REL);
    return e;
}

template <int CLS>
cudaError_t batch_launch_class(const BatchItem* items, const BatchTile* tiles, int ntiles, unsigned* counter,
                               int grid, size_t smem, cudaStream_t s) {
    cudaError_t e = batch_prepare_class<CLS>();
    if (e != cudaSuccess) return e;
    batch_kernel<CLS><<<grid, kFastThreads, smem, s>>>(items, tiles, ntiles, counter);
    return cudaGetLastError();
}

template <int CLS>
cudaError_t batch_occupancy_class(size_t smem, int* occ) {
    cudaError_t e = batch_prepare_class<CLS>();
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, batch_kernel<CLS>, kFastThreads, smem);
}

}  // namespace ipfc
