// filter2d_noalloc.cu -- filter2D for callers that cannot allocate memory.
//
// ipfc_filter2d stages its list of non-zero taps in a small device buffer
// that it allocates per call.  Some callers cannot allocate: code running
// where the allocator must not be entered (inside a custom memory manager,
// or on a device whose memory a host framework has fully reserved), code
// that must not touch the allocator once set up (real-time pipelines that
// forbid allocation after start-up), or foreign runtimes with no allocation
// hook.  ipfc_filter2d_noalloc serves them: the tap list lives in the
// file-scope device array below (kNoAllocMaxTaps entries, 64 KB, held by
// every GPU that loads the library until the process exits), and nothing is
// allocated per call.  The caller passes device images only (host images
// would need staging buffers).  It always runs the FP32 CUDA-core form, the
// same kernel as ipfc_filter2d_fp32 (ipfc_filter2d may pick the tensor-core
// form for single-channel uint8 images from 15 x 15 taps, whose uint8
// results can differ from this one by 1 LSB; both stay within 1 LSB of ipf).
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress while that device is current.  The taps travel
// from a per-thread pageable host buffer with cudaMemcpyAsync, which a
// capturing stream refuses, and a captured copy would replay the buffer's
// contents at replay time; so a call on a capturing stream is rejected with
// IPFC_ERR_UNSUPPORTED before anything is enqueued.  The array is shared by
// every call and keeps the last call's taps: any two calls whose streams the
// caller has not ordered (by using the same stream, an event or a
// synchronisation) race on it, even when their kernels would not run at the
// same time, because the second call's copy may land before the first call's
// kernel starts.  Each call writes exactly the entries its kernel reads, so
// nothing has to start at zero.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/ipfc.h"
#include "kernels.cuh"

namespace ipfc {
int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* fn);
size_t elem_bytes(int dt);
}  // namespace ipfc

namespace {

constexpr int kNoAllocMaxTaps = 4096;  // 64 KB of {w, dx, dy, 0}

// In host code this name is only a stand-in for the symbol, not a device
// address: kernels get the address looked up below.
static __device__ __align__(256) float4 g_noalloc_taps[kNoAllocMaxTaps];

// Per-device address of the array; threads may race to fill an entry, and
// every racer stores the same value, so acquire/release atomics suffice.
float4* g_taps_addr[32] = {nullptr};

// Device address of g_noalloc_taps on the current device (looked up once).
int taps_address(float4** out, const char* fn) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return ipfc::cuda_status(e, fn);
    if (dev < 0 || dev >= 32)
        return ipfc::set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: device index %d out of range", fn, dev);
    float4* addr = __atomic_load_n(&g_taps_addr[dev], __ATOMIC_ACQUIRE);
    if (!addr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_taps);
        if (e != cudaSuccess) return ipfc::cuda_status(e, fn);
        addr = static_cast<float4*>(p);
        __atomic_store_n(&g_taps_addr[dev], addr, __ATOMIC_RELEASE);
    }
    *out = addr;
    return IPFC_OK;
}

bool supported(int dt) { return dt == IPFC_U8 || dt == IPFC_U16 || dt == IPFC_I16 || dt == IPFC_F32; }

}  // namespace

extern "C" IPFC_API int ipfc_filter2d_noalloc(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw,
                                               int kh, int ax, int ay, int border, double delta,
                                               double border_value, void* stream) {
    using namespace ipfc;
    const char* fn = "filter2D (no-alloc)";
    if (!kernel || kw <= 0 || kh <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: filter2D: kernel must be a non-empty single-channel image");
    if (ax < 0) ax = kw / 2;
    if (ay < 0) ay = kh / 2;
    if (!(ax < kw && ay < kh)) return set_error(IPFC_ERR_INVALID, "ipf: filter2D: anchor outside kernel");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (src->mem != IPFC_MEM_DEVICE || dst->mem != IPFC_MEM_DEVICE)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: images must be in device memory (host images need staging)", fn);
    if (src->width < 0 || src->height < 0 || src->channels < 1)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid source dimensions", fn);
    if (dst->width != src->width || dst->height != src->height || dst->channels != src->channels)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: destination shape does not match source", fn);
    if (!supported(src->dtype) || !supported(dst->dtype))
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: element type not provided by this build (u8, u16, i16, f32)",
                         fn);
    const long long srow = (long long)src->width * src->channels * (long long)elem_bytes(src->dtype);
    const long long drow = (long long)dst->width * dst->channels * (long long)elem_bytes(dst->dtype);
    if ((src->pitch != 0 && src->pitch < srow) || (dst->pitch != 0 && dst->pitch < drow))
        return set_error(IPFC_ERR_INVALID, "ipf: %s: pitch smaller than a row", fn);
    if ((long long)src->width * src->channels > 0x3fffffffLL || (long long)src->height > 0x3fffffffLL)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: image too large", fn);
    // Non-zero taps in row-major order, as the reference builds them
    // (include/ipf/filter.hpp:171-178); the list must fit the static array.
    int ntaps = 0;
    for (long long i = 0; i < (long long)kw * kh; ++i) ntaps += kernel[i] != 0.f ? 1 : 0;
    if (ntaps > kNoAllocMaxTaps)
        return set_error(IPFC_ERR_INVALID,
                         "ipf: %s: %d non-zero taps exceed this entry point's fixed capacity of %d (use ipfc_filter2d)",
                         fn, ntaps, kNoAllocMaxTaps);
    if (src->width == 0 || src->height == 0) return IPFC_OK;
    if (!src->data || !dst->data) return set_error(IPFC_ERR_INVALID, "ipf: %s: null pixel pointer", fn);
    if (src->data == dst->data) return set_error(IPFC_ERR_INVALID, "ipf: %s: in-place operation is not supported", fn);
    cudaStream_t s = (cudaStream_t)stream;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing(s, &cap);
    if (ce != cudaSuccess) return cuda_status(ce, fn);
    if (cap != cudaStreamCaptureStatusNone)
        return set_error(IPFC_ERR_UNSUPPORTED,
                         "ipf: %s: cannot be called while its stream is capturing (the taps are copied from a "
                         "per-thread host buffer)",
                         fn);
    float4* taps = nullptr;
    int rc = taps_address(&taps, fn);
    if (rc) return rc;
    // Host copy of the list, copied into the static array on the stream.  A
    // copy from pageable memory returns once the source has been read, so
    // this thread may reuse the buffer on its next call.
    static thread_local float4 host[kNoAllocMaxTaps];
    int n = 0;
    for (int j = 0; j < kh; ++j)
        for (int i = 0; i < kw; ++i) {
            const float w = kernel[(size_t)j * kw + i];
            if (w != 0.f) host[n++] = make_float4(w, (float)i, (float)j, 0.f);
        }
    cudaError_t e = cudaSuccess;
    if (n > 0) e = cudaMemcpyAsync(taps, host, sizeof(float4) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, fn);
    F2DArgs a;
    std::memset(&a, 0, sizeof(a));
    a.src = src->data;
    a.spitch = src->pitch > 0 ? src->pitch : srow;
    a.dst = dst->data;
    a.dpitch = dst->pitch > 0 ? dst->pitch : drow;
    a.W = src->width;
    a.H = src->height;
    a.C = src->channels;
    a.kw = kw;
    a.kh = kh;
    a.ax = ax;
    a.ay = ay;
    a.border = border;
    a.delta = (float)delta;
    a.bv = (float)border_value;
    a.ntaps = n;
    a.dense = n == kw * kh;
    a.taps = taps;
    e = filter2d_launch(src->dtype, dst->dtype, a, s);
    return e == cudaSuccess ? IPFC_OK : cuda_status(e, fn);
}
