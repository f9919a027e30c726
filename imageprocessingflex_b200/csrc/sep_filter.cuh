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
    // FP64 forms of the same (int32 or double images accumulate in FP64)
    double deltad, bvd;
    double kxd[kSepMaxParamTaps];
    double kyd[kSepMaxParamTaps];
};

// True when the call accumulates in FP64: a 32-bit integer or double image on
// either side.
inline bool sep_wide(int sdt, int ddt) {
    return sdt == IPFC_I32 || sdt == IPFC_F64 || ddt == IPFC_I32 || ddt == IPFC_F64;
}

// Launches the separable correlation described by `a` (taps in a.kx/a.ky, or
// a.kxd/a.kyd for FP64 calls, when kw, kh <= kSepMaxParamTaps).  dkx/dky: the
// same taps in device memory (float, or double for FP64 calls), used by the
// two-pass form; scratch: H*W*C accumulator elements (float or double) of
// device memory for that form (may be null when the fused form applies, see
// sep_needs_scratch).
cudaError_t sep_launch(int sdt, int ddt, const SepArgs& a, const void* dkx, const void* dky, void* scratch,
                       cudaStream_t s, bool force_fp64 = false);

bool sep_needs_scratch(const SepArgs& a, bool wide);

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
    double scaled, bvd;         // fl64(1/(kw*kh)) and the border value, for FP64 sums
    unsigned tie_up[2048];      // bit t: exact tie t + 1/2 rounds up (t < 65536)
};

// exact_int: integer source summed exactly in int32 (the host checks that the
// border value is integral and that no window sum can overflow).  int32 and
// double images are summed in FP64 (exact for integer windows below 2^53).
cudaError_t box_launch(int sdt, int ddt, const BoxArgs& a, bool exact_int, cudaStream_t s, bool force_fp64 = false);

// Raises a kernel's dynamic shared-memory limit once per device.
cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

}  // namespace ipfc
