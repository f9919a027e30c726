// kernels.cuh -- argument blocks and launchers of the dense, median and
// morphology kernels (the separable ones live in sep_filter.cuh).
#pragma once

#include "common.cuh"
#include "sep_filter.cuh"

namespace ipfc {

struct MedianArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C;
    int ksize;
    int border;
};

cudaError_t median_launch(int dt, const MedianArgs& a, cudaStream_t s);

// Morphology: one erosion or dilation pass.  Offsets of the structuring
// element's members relative to its anchor, packed (dx, dy) as int16 pairs in
// row-major order, carried in the launch parameters.
constexpr int kMorphMaxOffsets = 1024;

// Everything but the member list (all an all-ones element needs).
struct MorphCore {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C;
    int sw, sh, ax, ay;
    int is_rect;
    int is_min;
    int noffs;
};

struct MorphArgs : MorphCore {
    short2 offs[kMorphMaxOffsets];
};

cudaError_t morph_launch(int dt, const MorphArgs& a, cudaStream_t s);

// Dense correlation with FP32 accumulation on the CUDA cores.
struct F2DArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C;
    int kw, kh, ax, ay;
    int border;
    float delta, bv;
    double deltad, bvd;  // the same in FP64 (int32 / double images accumulate in FP64)
    int ntaps;       // non-zero taps
    int dense;       // 1 when every tap is non-zero (taps = kw*kh, row-major)
    const float4* taps;  // device: {w, dx, dy, 0} per non-zero tap, row-major order
};

cudaError_t filter2d_launch(int sdt, int ddt, const F2DArgs& a, cudaStream_t s);

}  // namespace ipfc
