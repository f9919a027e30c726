// sep_filter.cuh -- separable correlation kernels (declarations shared with the API layer).
#pragma once

#include "common.cuh"

namespace ipfc {

// Taps carried in the launch parameters up to this length per axis; longer
// kernels use the two-pass form with taps in device memory.
constexpr int kSepMaxParamTaps = 64;

struct SepArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C;       // pixels, rows, channels
    int kw, kh;        // tap counts
    int ax, ay;        // anchors
    int border;
    float delta;
    float bv;          // border value (Constant)
    float kx[kSepMaxParamTaps];
    float ky[kSepMaxParamTaps];
};

// Launches the separable correlation described by `a` (taps in a.kx/a.ky when
// kw, kh <= kSepMaxParamTaps).  dkx/dky: the same taps in device memory, used
// by the two-pass form; scratch: H*W*C floats of device memory for that form
// (may be null when the fused form applies, see sep_needs_scratch).
cudaError_t sep_launch(int sdt, int ddt, const SepArgs& a, const float* dkx, const float* dky, float* scratch,
                       cudaStream_t s);

bool sep_needs_scratch(const SepArgs& a);

// Box filter over integer or float sources (exact integer sums for integer
// sources).  tie_up: bit t set when the reference rounds an exact x.5 window
// mean t + 0.5 up (see the box kernel).
struct BoxArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C;
    int kw, kh, ax, ay;
    int border;
    int normalize;
    float bv;
    float scale_hi, scale_lo;  // fl64(1/(kw*kh)) split into two floats
    unsigned tie_up[2048];      // bit t: exact tie t + 1/2 rounds up (t < 65536)
};

// exact_int: integer source summed exactly in int32 (the host checks that the
// border value is integral and that no window sum can overflow).
cudaError_t box_launch(int sdt, int ddt, const BoxArgs& a, bool exact_int, cudaStream_t s);

// Raises a kernel's dynamic shared-memory limit once per device.
cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

}  // namespace ipfc
