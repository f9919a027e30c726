// api.cu -- the extern "C" entry points of include/ipfc.h.
//
// Host responsibilities: argument checks with the reference's messages, tap
// generation in FP64 exactly as the reference computes it, staging of host
// images through stream-ordered device allocations, and dispatch to the
// kernels.  No compute runs on the host and nothing falls back to it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ipfc.h"
#include "api_internal.h"
#include "filter2d_tc.cuh"
#include "kernels.cuh"
#include "sep_fast_launch.cuh"
#include "tma.cuh"

namespace ipfc {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_status(cudaError_t e, const char* fn) {
    if (e == cudaSuccess) return IPFC_OK;
    cudaGetLastError();  // clear sticky-free errors so the next call starts clean
    if (e == cudaErrorMemoryAllocation)
        return set_error(IPFC_ERR_NOMEM, "ipf: %s: device allocation failed (%s)", fn, cudaGetErrorString(e));
    return set_error(IPFC_ERR_CUDA, "ipf: %s: CUDA error: %s", fn, cudaGetErrorString(e));
}

#define IPFC_TRY_CUDA(expr, fn)                          \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return cuda_status(e_, fn); \
    } while (0)

size_t elem_bytes(int dt) {
    switch (dt) {
        case IPFC_U8: return 1;
        case IPFC_U16: case IPFC_I16: return 2;
        case IPFC_I32: case IPFC_F32: return 4;
        case IPFC_F64: return 8;
        default: return 0;
    }
}

static bool dtype_supported(int dt) { return dt >= IPFC_U8 && dt <= IPFC_F64; }

long long row_bytes(const ipfc_image* im) {
    return (long long)im->width * im->channels * (long long)elem_bytes(im->dtype);
}

long long pitch_of(const ipfc_image* im) { return im->pitch > 0 ? im->pitch : row_bytes(im); }

// ---------------------------------------------------------------------------
// Device memory: stream-ordered allocations from the device's default pool,
// kept cached by a maximal release threshold (set once per device) so that
// steady-state calls do not return memory to the driver.  Reuse across
// streams through inserted dependencies is off: a call on one stream never
// waits for another stream's work to reuse its freed staging memory, so
// callers on several streams overlap their copies and kernels.
// ---------------------------------------------------------------------------
static unsigned g_pool_ready = 0;

cudaError_t prepare_device() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned bit = dev >= 0 && dev < 32 ? 1u << dev : 0u;  // devices past 32 are set up every call
    if (__atomic_load_n(&g_pool_ready, __ATOMIC_ACQUIRE) & bit) return cudaSuccess;
    cudaMemPool_t pool;
    e = cudaDeviceGetDefaultMemPool(&pool, dev);
    if (e != cudaSuccess) return e;
    unsigned long long thr = ~0ull;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (e != cudaSuccess) return e;
    int no_internal_deps = 0;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no_internal_deps);
    if (e != cudaSuccess) return e;
    __atomic_fetch_or(&g_pool_ready, bit, __ATOMIC_ACQ_REL);
    return cudaSuccess;
}

// Device error word: kernels with bounded waits record a code here when a
// wait gives up.  One word per device, allocated on the first call that
// launches such a kernel on that device (under a lock: callers may be on
// several threads).
static unsigned* g_err_word[32] = {nullptr};
static std::mutex g_err_word_mu;

unsigned* device_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    // Past the table no word is kept: the kernels skip the error write when
    // given none, and ipfc_check_device then reports nothing.
    if (dev < 0 || dev >= 32) return nullptr;
    std::lock_guard<std::mutex> lk(g_err_word_mu);
    unsigned*& w = g_err_word[dev];
    if (!w) {
        unsigned* p = nullptr;
        if (cudaMalloc((void**)&p, sizeof(unsigned)) != cudaSuccess ||
            cudaMemset(p, 0, sizeof(unsigned)) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        w = p;
    }
    return w;
}

// Bound of the device-side pipeline waits of the tensor-core kernels.
static unsigned long long g_wait_limit_ns = 0;  // 0: the default

unsigned long long device_wait_limit_ns() {
    const unsigned long long v = __atomic_load_n(&g_wait_limit_ns, __ATOMIC_ACQUIRE);
    return v ? v : kWaitNsDefault;
}

// Reads and clears the error word after the stream has drained.
int take_device_error(cudaStream_t s, const char* fn) {
    unsigned* w = device_error_word();
    if (!w) return IPFC_OK;
    unsigned v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, w, sizeof(v), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_status(e, fn);
    if (v == 0) return IPFC_OK;
    cudaMemsetAsync(w, 0, sizeof(unsigned), s);
    cudaStreamSynchronize(s);
    return set_error(IPFC_ERR_TIMEOUT,
                     "ipf: %s: a device-side wait gave up (code 0x%x); results of the affected call are not valid", fn,
                     v);
}

long long round_up(long long v, long long m) { return (v + m - 1) / m * m; }

int view_in(const ipfc_image* im, cudaStream_t s, DevView* v, const char* fn) {
    if (im->mem == IPFC_MEM_DEVICE) {
        v->ptr = im->data;
        v->pitch = pitch_of(im);
        return IPFC_OK;
    }
    const long long rb = row_bytes(im);
    v->pitch = round_up(rb > 0 ? rb : 1, 128);
    IPFC_TRY_CUDA(cudaMallocAsync(&v->ptr, (size_t)(v->pitch * im->height), s), fn);
    v->owned = true;
    IPFC_TRY_CUDA(cudaMemcpy2DAsync(v->ptr, (size_t)v->pitch, im->data, (size_t)pitch_of(im), (size_t)rb,
                                    (size_t)im->height, cudaMemcpyHostToDevice, s),
                  fn);
    return IPFC_OK;
}

int view_out(const ipfc_image* im, cudaStream_t s, DevView* v, const char* fn) {
    if (im->mem == IPFC_MEM_DEVICE) {
        v->ptr = im->data;
        v->pitch = pitch_of(im);
        return IPFC_OK;
    }
    const long long rb = row_bytes(im);
    v->pitch = round_up(rb > 0 ? rb : 1, 128);
    IPFC_TRY_CUDA(cudaMallocAsync(&v->ptr, (size_t)(v->pitch * im->height), s), fn);
    v->owned = true;
    return IPFC_OK;
}

// Copies a staged result back to host memory, releases staging memory and,
// when any side lives in host memory, waits for the stream.
int finish(const ipfc_image* dst, DevView* in, DevView* out, cudaStream_t s, const char* fn) {
    cudaError_t e = cudaSuccess;
    if (out->owned) {
        e = cudaMemcpy2DAsync(dst->data, (size_t)pitch_of(dst), out->ptr, (size_t)out->pitch, (size_t)row_bytes(dst),
                              (size_t)dst->height, cudaMemcpyDeviceToHost, s);
    }
    if (in && in->owned) cudaFreeAsync(in->ptr, s);
    if (out->owned) cudaFreeAsync(out->ptr, s);
    if (e != cudaSuccess) return cuda_status(e, fn);
    if ((in && in->owned) || out->owned) {
        IPFC_TRY_CUDA(cudaStreamSynchronize(s), fn);
        return take_device_error(s, fn);
    }
    return IPFC_OK;
}

// Common checks: both views non-null, supported types, equal shapes, no
// aliasing, a device present.  Returns IPFC_OK, an error, or -1 for "empty
// image: nothing to do" (the reference returns an empty result).
int check_pair(const ipfc_image* src, const ipfc_image* dst, const char* fn, bool same_type) {
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (src->width < 0 || src->height < 0 || src->channels < 1)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid source dimensions", fn);
    if (dst->width != src->width || dst->height != src->height || dst->channels != src->channels)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: destination shape does not match source", fn);
    if (!dtype_supported(src->dtype) || !dtype_supported(dst->dtype))
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: unknown element type code", fn);
    if (same_type && src->dtype != dst->dtype)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: source and destination types differ", fn);
    if ((src->mem != IPFC_MEM_HOST && src->mem != IPFC_MEM_DEVICE) ||
        (dst->mem != IPFC_MEM_HOST && dst->mem != IPFC_MEM_DEVICE))
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid memory kind", fn);
    if ((src->pitch != 0 && src->pitch < row_bytes(src)) || (dst->pitch != 0 && dst->pitch < row_bytes(dst)))
        return set_error(IPFC_ERR_INVALID, "ipf: %s: pitch smaller than a row", fn);
    if ((long long)src->width * src->channels > 0x3fffffffLL || (long long)src->height > 0x3fffffffLL)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: image too large", fn);
    if (src->width == 0 || src->height == 0) return -1;
    if (!src->data || !dst->data) return set_error(IPFC_ERR_INVALID, "ipf: %s: null pixel pointer", fn);
    if (src->data == dst->data) return set_error(IPFC_ERR_INVALID, "ipf: %s: in-place operation is not supported", fn);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(IPFC_ERR_CUDA, "ipf: %s: no CUDA device available", fn);
    }
    cudaError_t e = prepare_device();
    if (e != cudaSuccess) return cuda_status(e, fn);
    return IPFC_OK;
}

// check_pair for a destination whose shape differs from the source's by the
// function's definition (pyramids, the integral image, single-channel edge
// maps): the caller has checked that shape; the destination's own pitch is
// checked against its own row, the rest as check_pair does.
int check_pair_resized(const ipfc_image* src, const ipfc_image* dst, const char* fn, bool same_type) {
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (dtype_supported(dst->dtype) && dst->pitch != 0 && dst->pitch < row_bytes(dst))
        return set_error(IPFC_ERR_INVALID, "ipf: %s: pitch smaller than a row", fn);
    ipfc_image same = *dst;
    same.width = src->width;
    same.height = src->height;
    same.channels = src->channels;
    same.pitch = 0;
    return check_pair(src, &same, fn, same_type);
}

// ---------------------------------------------------------------------------
// Tap generators (FP64, the reference's expressions and order)
// ---------------------------------------------------------------------------
int gaussian_taps(double sigma, int ksize, std::vector<double>& k) {
    if (ksize <= 0) {
        if (!(sigma > 0))
            return set_error(IPFC_ERR_INVALID, "ipf: gaussianKernel1D: need sigma > 0 or ksize > 0");
        const int r = static_cast<int>(3.0 * sigma + 0.5);
        ksize = 2 * (r > 1 ? r : 1) + 1;
    }
    if (ksize % 2 != 1) return set_error(IPFC_ERR_INVALID, "ipf: gaussianKernel1D: ksize must be odd");
    if (sigma <= 0) sigma = 0.3 * ((ksize - 1) * 0.5 - 1) + 0.8;
    k.assign((size_t)ksize, 0.0);
    const int c = ksize / 2;
    double sum = 0;
    for (int i = 0; i < ksize; ++i) {
        k[i] = std::exp(-0.5 * (i - c) * (i - c) / (sigma * sigma));
        sum += k[i];
    }
    for (double& v : k) v /= sum;
    return IPFC_OK;
}

int deriv_taps(int order, int ksize, std::vector<double>& k) {
    if (ksize == 1) {
        if (order == 0) { k = {1.0}; return IPFC_OK; }
        if (order == 1) { k = {-1.0, 0.0, 1.0}; return IPFC_OK; }
        if (order == 2) { k = {1.0, -2.0, 1.0}; return IPFC_OK; }
        return set_error(IPFC_ERR_INVALID, "ipf: derivKernel: order > 2 requires ksize >= 3");
    }
    if (!(ksize % 2 == 1 && ksize >= 3 && ksize <= 31))
        return set_error(IPFC_ERR_INVALID, "ipf: derivKernel: ksize must be odd in [3, 31]");
    if (!(order >= 0 && order < ksize)) return set_error(IPFC_ERR_INVALID, "ipf: derivKernel: invalid derivative order");
    // binomial smoothing (1, 1)^(ksize-1-order) convolved with (-1, 1)^order
    k.assign(1, 1.0);
    for (int step = 0; step < ksize - 1; ++step) {
        const double a = step < ksize - 1 - order ? 1.0 : -1.0;
        std::vector<double> r(k.size() + 1, 0.0);
        for (size_t i = 0; i < k.size(); ++i) {
            r[i] += k[i] * a;
            r[i + 1] += k[i] * 1.0;
        }
        k.swap(r);
    }
    return IPFC_OK;
}

// ---------------------------------------------------------------------------
// Separable path shared by sepFilter2D, gaussianBlur and sobel.
// ---------------------------------------------------------------------------

bool filter2d_tc_eligible(int sdt, int ddt, int C, int kw, int kh);
cudaError_t filter2d_tc_launch(int sdt, int ddt, const void* src, long long spitch, void* dst, long long dpitch, int W,
                               int H, int C, const float* taps, int kw, int kh, int ax, int ay, int border, float delta,
                               float bv, cudaStream_t s);
bool sep_tcol_launch(const void* src, long long spitch, void* dst, long long dpitch, int W, int H, int C,
                     const double* kx, const double* ky, int K, int border, double delta, double bv, int clamp,
                     cudaStream_t s, cudaError_t* err);

// Kernel selection for separable filters.  Default: uint8 -> uint8 calls
// that the tensor-core column-pass kernel covers (sep_tcol.cu) run there
// where it is the faster one (tcol_wins), the rest on the CUDA-core fast
// kernel where it is instantiated, else on the generic kernels.
// IPFC_SEP_PATH=generic forces the generic fused/two-pass kernels; =fast
// keeps uint8 calls off the tensor cores; =tcol takes the tensor-core kernel
// for every size it covers.
//
// The tensor-core kernel costs about 11 us per CTA on top of its per-unit
// work and barely depends on the tap count; the CUDA-core kernel scales
// with samples x taps.  Measured gaussianBlur, uint8, L2-cold inputs (us per
// image, CUDA-core / tensor-core):
//   C = 1: 1920x1080 K 13  16.6 / 22.8   3840x2160 K 9  30.0 / 28.2
//          3840x2160 K 13  29.7 / 28.9   4096x4096 K 9  48.4 / 38.9
//   C = 3: 1920x1080 K 13  21.8 / 27.5   2560x1440 K 9  31.1 / 33.5
//          2560x1440 K 13  35.2 / 35.0   2560x1440 K 15 40.9 / 35.5
//          3840x2160 K 9   59.2 / 48.4   3840x2160 K 13 64.7 / 50.3
//   C = 4: 1920x1080 K 15  27.5 / 28.4   2560x1440 K 13 38.9 / 38.5
//          3840x2160 K 9   68.9 / 59.1
// Below 9 taps the CUDA-core kernel stays (3840x2160x3 K 7 on an earlier
// build of the tensor-core kernel: 49.4 / 51.6).
static bool tcol_wins(int kw, int channels, long long samples) {
    if (kw < 9) return false;
    if (channels == 1) return samples >= 7000000;
    return samples >= 16000000 || (kw >= 13 && samples >= 10000000);
}
// Callers that share the GPU among many streams (the request server) keep
// separable calls on the CUDA-core kernel: the tensor-core kernel is
// persistent, one CTA with 203 KB of shared memory on every SM, so while it
// runs no other stream's kernel gets an SM.
static thread_local bool t_shared_gpu = false;
void set_shared_gpu(bool on) { t_shared_gpu = on; }
static int sep_path_mode() {
    static const int mode = [] {  // read once, thread-safe initialisation
        const char* v = std::getenv("IPFC_SEP_PATH");
        if (!v) return 0;
        if (std::strcmp(v, "generic") == 0) return 1;
        if (std::strcmp(v, "fast") == 0) return 2;
        if (std::strcmp(v, "tcol") == 0) return 4;
        return 0;
    }();
    return mode;
}

// The fast kernel covers equal tap counts up to kFastMaxTaps with centred
// anchors and finite taps; the instantiation table decides the rest.
static bool sep_fast_eligible(const ipfc_image* src, const double* kx, int kw, const double* ky, int kh, int ax,
                              int ay) {
    if (sep_path_mode() == 1) return false;
    if (kw != kh || kw > kFastMaxTaps || ax != kw / 2 || ay != kh / 2) return false;
    if (src->channels != 1 && src->channels != 3 && src->channels != 4) return false;
    for (int i = 0; i < kw; ++i)
        if (!std::isfinite(kx[i]) || !std::isfinite(ky[i]) || !std::isfinite((float)kx[i]) ||
            !std::isfinite((float)ky[i]))
            return false;
    return true;
}

static unsigned long long pack_tap2(double v) {
    const float fv = (float)v;
    unsigned u;
    std::memcpy(&u, &fv, sizeof(u));
    return ((unsigned long long)u << 32) | u;
}

// Argument block of the fast kernel for device views (in_ptr, in_pitch) ->
// (out_ptr, out_pitch); false when the fast kernel does not cover the call.
// The batch layer builds its separable items with this same function, so a
// batched image computes exactly what the per-image call computes.
bool make_sep_fast_args(const ipfc_image* src, const ipfc_image* dst, const void* in_ptr, long long in_pitch,
                        void* out_ptr, long long out_pitch, const double* kx, int kw, const double* ky, int kh, int ax,
                        int ay, int border, double delta, double bv, SepFastArgs* fp) {
    if (!sep_fast_eligible(src, kx, kw, ky, kh, ax, ay)) return false;
    // the kernel forms row offsets as 32 x 32-bit products
    if (in_pitch <= 0 || in_pitch >= (1LL << 31) || out_pitch <= 0 || out_pitch >= (1LL << 31)) return false;
    SepFastArgs& f = *fp;
    std::memset(&f, 0, sizeof(f));
    f.src = in_ptr;
    f.spitch = in_pitch;
    f.dst = out_ptr;
    f.dpitch = out_pitch;
    f.W = src->width;
    f.H = src->height;
    f.border = border;
    f.delta = (float)delta;
    f.bv = (float)bv;
    for (int i = 0; i < kw; ++i) {
        f.kx[i] = (float)kx[i];
        f.kx2[i] = pack_tap2(kx[i]);
    }
    for (int j = 0; j < kh; ++j) f.ky2[j] = pack_tap2(ky[j]);
    const uintptr_t op = (uintptr_t)out_ptr, ip = (uintptr_t)in_ptr;
    f.vec_store = (op % 16 == 0 && out_pitch % 16 == 0) ? 1 : 0;
    const unsigned vec_align = src->dtype == IPFC_F32 ? 8u : 4u;  // 2 floats or 4 bytes per load
    f.vec_load = (ip % vec_align == 0 && in_pitch % vec_align == 0) ? 1 : 0;
    // Saturation is needed unless every output provably stays inside the
    // destination range: non-negative taps bound the result between
    // delta + sum(kx)sum(ky) * min(0, lowest input) and the same with the
    // highest input.
    f.clamp = 1;
    if (dst->dtype == IPFC_U8 || dst->dtype == IPFC_U16) {
        double sx = 0, sy = 0;
        bool nonneg = true;
        for (int i = 0; i < kw; ++i) {
            sx += kx[i];
            nonneg = nonneg && kx[i] >= 0;
        }
        for (int j = 0; j < kh; ++j) {
            sy += ky[j];
            nonneg = nonneg && ky[j] >= 0;
        }
        const double smax = src->dtype == IPFC_U8 ? 255.0 : 65535.0;
        const double hi_in = border == IPFC_BORDER_CONSTANT ? std::fmax(smax, bv) : smax;
        const double lo_in = border == IPFC_BORDER_CONSTANT ? std::fmin(0.0, bv) : 0.0;
        const double dmax = dst->dtype == IPFC_U8 ? 255.0 : 65535.0;
        if (nonneg && (src->dtype == IPFC_U8 || src->dtype == IPFC_U16) && delta + sx * sy * lo_in > -0.25 &&
            delta + sx * sy * hi_in < dmax + 0.25)
            f.clamp = 0;
    }
    return true;
}

// Launches the fast kernel when a fitting instantiation exists; returns
// whether it did (e holds the launch status).
static bool run_sep_fast(const ipfc_image* src, const ipfc_image* dst, const DevView& in, const DevView& out,
                         const double* kx, int kw, const double* ky, int kh, int ax, int ay, int border, double delta,
                         double bv, cudaStream_t s, cudaError_t* e) {
    SepFastArgs f;
    if (!make_sep_fast_args(src, dst, in.ptr, in.pitch, out.ptr, out.pitch, kx, kw, ky, kh, ax, ay, border, delta, bv,
                            &f))
        return false;
    const int mode = sep_path_mode();
    const bool tcol = mode == 4 || (mode == 0 && !t_shared_gpu &&
                                    tcol_wins(kw, src->channels, (long long)src->width * src->channels * src->height));
    if (tcol && src->dtype == IPFC_U8 && dst->dtype == IPFC_U8 &&
        sep_tcol_launch(in.ptr, in.pitch, out.ptr, out.pitch, src->width, src->height, src->channels, kx, ky, kw,
                        border, delta, bv, f.clamp, s, e))
        return true;
    return sep_fast_dispatch(kw, src->channels, src->dtype, dst->dtype, f, s, e);
}
int run_sep(const ipfc_image* src, ipfc_image* dst, const double* kx, int kw, const double* ky, int kh, int ax, int ay,
            int border, double delta, double bv, cudaStream_t s, const char* fn, bool force_fp64) {
    if (!kx || !ky || kw <= 0 || kh <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: separable filter: empty kernel");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    if (ax < 0) ax = kw / 2;
    if (ay < 0) ay = kh / 2;
    if (ax >= kw || ay >= kh) return set_error(IPFC_ERR_INVALID, "ipf: %s: anchor outside kernel", fn);
    int rc = check_pair(src, dst, fn, false);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    SepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.W = src->width;
    a.H = src->height;
    a.C = src->channels;
    a.kw = kw;
    a.kh = kh;
    a.ax = ax;
    a.ay = ay;
    a.border = border;
    a.delta = (float)delta;
    a.bv = (float)bv;
    a.deltad = delta;
    a.bvd = bv;
    for (int i = 0; i < kw && i < kSepMaxParamTaps; ++i) {
        a.kx[i] = (float)kx[i];
        a.kxd[i] = kx[i];
    }
    for (int j = 0; j < kh && j < kSepMaxParamTaps; ++j) {
        a.ky[j] = (float)ky[j];
        a.kyd[j] = ky[j];
    }
    // FP64 accumulation (the reference's own arithmetic, bit-identical
    // results) for int32 / double images, and when a composite op asks for
    // it to reproduce the reference's intermediate exactly
    const bool wide = force_fp64 || sep_wide(src->dtype, dst->dtype);
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    a.src = in.ptr;
    a.spitch = in.pitch;
    a.dst = out.ptr;
    a.dpitch = out.pitch;
    unsigned char* dtaps = nullptr;  // kw + kh taps, float or (FP64 calls) double
    void* scratch = nullptr;
    cudaError_t e = cudaSuccess;
    if (!wide && run_sep_fast(src, dst, in, out, kx, kw, ky, kh, ax, ay, border, delta, bv, s, &e)) {
        rc = finish(dst, &in, &out, s, fn);
        if (e != cudaSuccess) return cuda_status(e, fn);
        return rc;
    }
    const size_t tsz = wide ? sizeof(double) : sizeof(float);
    if (sep_needs_scratch(a, wide)) {
        std::vector<unsigned char> taps(((size_t)kw + kh) * tsz);
        for (int i = 0; i < kw + kh; ++i) {
            const double v = i < kw ? kx[i] : ky[i - kw];
            if (wide) std::memcpy(&taps[(size_t)i * tsz], &v, tsz);
            else {
                const float f = (float)v;
                std::memcpy(&taps[(size_t)i * tsz], &f, tsz);
            }
        }
        e = cudaMallocAsync((void**)&dtaps, taps.size(), s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dtaps, taps.data(), taps.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMallocAsync(&scratch, tsz * (size_t)a.W * a.C * a.H, s);
    }
    if (e == cudaSuccess)
        e = sep_launch(src->dtype, dst->dtype, a, dtaps, dtaps ? dtaps + (size_t)kw * tsz : nullptr, scratch, s,
                       force_fp64);
    if (dtaps) cudaFreeAsync(dtaps, s);
    if (scratch) cudaFreeAsync(scratch, s);
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

}  // namespace ipfc

using namespace ipfc;

extern "C" {

const char* ipfc_last_error(void) { return g_last_error.c_str(); }

int ipfc_version(void) { return (1 << 16) | (0 << 8) | 0; }

unsigned long long ipfc_set_wait_limit_ns(unsigned long long ns) {
    const unsigned long long old = __atomic_exchange_n(&g_wait_limit_ns, ns, __ATOMIC_ACQ_REL);
    return old ? old : kWaitNsDefault;
}

int ipfc_check_device(void* stream) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(IPFC_ERR_CUDA, "ipf: check_device: no CUDA device available");
    }
    cudaStream_t s = (cudaStream_t)stream;
    IPFC_TRY_CUDA(cudaStreamSynchronize(s), "check_device");
    return take_device_error(s, "check_device");
}

int ipfc_gaussian_kernel_1d(double sigma, int ksize, double* out, int cap) {
    std::vector<double> k;
    if (gaussian_taps(sigma, ksize, k)) return -1;
    for (int i = 0; i < (int)k.size() && i < cap; ++i) out[i] = k[i];
    return (int)k.size();
}

int ipfc_deriv_kernel(int order, int ksize, double* out, int cap) {
    std::vector<double> k;
    if (deriv_taps(order, ksize, k)) return -1;
    for (int i = 0; i < (int)k.size() && i < cap; ++i) out[i] = k[i];
    return (int)k.size();
}

int ipfc_structuring_element(int shape, int width, int height, uint8_t* out) {
    if (height <= 0) height = width;
    if (width <= 0 || height <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: getStructuringElement: size must be positive");
    if (shape < IPFC_MORPH_RECT || shape > IPFC_MORPH_ELLIPSE)
        return set_error(IPFC_ERR_INVALID, "ipf: getStructuringElement: invalid shape");
    std::memset(out, 0, (size_t)width * height);
    const int r = height / 2, c = width / 2;
    const double inv_r2 = r ? 1.0 / (static_cast<double>(r) * r) : 0.0;
    for (int i = 0; i < height; ++i) {
        int j1 = 0, j2 = 0;
        if (shape == IPFC_MORPH_RECT || (shape == IPFC_MORPH_CROSS && i == r)) {
            j2 = width;
        } else if (shape == IPFC_MORPH_CROSS) {
            j1 = c;
            j2 = c + 1;
        } else {
            const int dy = i - r;
            if (std::abs(dy) <= r) {
                const double v = c * std::sqrt((r * r - dy * dy) * inv_r2);
                const int dx = (int)(v + 0.5);  // saturate_cast<int>: half away from zero, v >= 0
                j1 = c - dx > 0 ? c - dx : 0;
                j2 = c + dx + 1 < width ? c + dx + 1 : width;
            }
        }
        for (int j = j1; j < j2; ++j) out[(size_t)i * width + j] = 1;
    }
    return IPFC_OK;
}

int ipfc_sep_filter2d(const ipfc_image* src, ipfc_image* dst, const double* kx, int kw, const double* ky, int kh,
                      int ax, int ay, int border, double delta, double border_value, void* stream) {
    return run_sep(src, dst, kx, kw, ky, kh, ax, ay, border, delta, border_value, (cudaStream_t)stream,
                   "sepFilter2D", false);
}

int ipfc_gaussian_blur(const ipfc_image* src, ipfc_image* dst, double sigma_x, double sigma_y, int ksize, int border,
                       void* stream) {
    if (sigma_y <= 0) sigma_y = sigma_x;
    std::vector<double> kx, ky;
    if (gaussian_taps(sigma_x, ksize, kx)) return IPFC_ERR_INVALID;
    if (gaussian_taps(sigma_y, ksize, ky)) return IPFC_ERR_INVALID;
    return run_sep(src, dst, kx.data(), (int)kx.size(), ky.data(), (int)ky.size(), -1, -1, border, 0.0, 0.0,
                   (cudaStream_t)stream, "gaussianBlur", false);
}

int ipfc_sobel(const ipfc_image* src, ipfc_image* dst, int dx, int dy, int ksize, double scale, int border,
               void* stream) {
    if (!(dx >= 0 && dy >= 0 && dx + dy > 0)) return set_error(IPFC_ERR_INVALID, "ipf: sobel: need dx + dy > 0");
    std::vector<double> kx, ky;
    if (deriv_taps(dx, ksize, kx)) return IPFC_ERR_INVALID;
    if (deriv_taps(dy, ksize, ky)) return IPFC_ERR_INVALID;
    if (ksize == 1) {  // keep both kernels 3 long so the anchors stay centred (filter.hpp:401-404)
        if (kx.size() == 1) kx = {0.0, 1.0, 0.0};
        if (ky.size() == 1) ky = {0.0, 1.0, 0.0};
    }
    for (double& v : kx) v *= scale;
    return run_sep(src, dst, kx.data(), (int)kx.size(), ky.data(), (int)ky.size(), -1, -1, border, 0.0, 0.0,
                   (cudaStream_t)stream, "sobel", false);
}

}  // extern "C"

namespace ipfc {

int run_box(const ipfc_image* src, ipfc_image* dst, int kw, int kh, int normalize, int border, double border_value,
            cudaStream_t s, bool force_fp64) {
    const char* fn = "boxFilter";
    if (kw <= 0 || kh <= 0) return set_error(IPFC_ERR_INVALID, "ipf: boxFilter: kernel size must be positive");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = check_pair(src, dst, fn, false);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    BoxArgs a;
    std::memset(&a, 0, sizeof(a));
    a.W = src->width;
    a.H = src->height;
    a.C = src->channels;
    a.kw = kw;
    a.kh = kh;
    a.ax = kw / 2;
    a.ay = kh / 2;
    a.border = border;
    a.normalize = normalize ? 1 : 0;
    a.bv = (float)border_value;
    a.bvd = border_value;
    const double n = (double)kw * kh;
    const double scale = normalize ? 1.0 / n : 1.0;
    a.scale_hi = (float)scale;
    a.scale_lo = (float)(scale - (double)a.scale_hi);
    a.scaled = scale;
    const bool int_src = src->dtype == IPFC_U8 || src->dtype == IPFC_U16 || src->dtype == IPFC_I16;
    const double maxval = src->dtype == IPFC_U8 ? 255.0 : (src->dtype == IPFC_U16 ? 65535.0 : 32768.0);
    const bool bv_int = std::floor(border_value) == border_value && std::fabs(border_value) <= 65535.0;
    const bool exact = int_src && bv_int && n * std::fmax(maxval, std::fabs(border_value)) < 2147483647.0;
    if (exact && normalize && ((long long)kw * kh) % 2 == 0) {
        // Outcome of each exact tie S/n = t + 1/2 under the reference's
        // expression saturate_cast(S * (1.0 / n)) (filter.hpp:238, 246).
        const long long nn = (long long)kw * kh;
        const long long tmax = (long long)std::fmin(65535.0, std::fmax(maxval, std::fabs(border_value)));
        for (long long t = 0; t <= tmax; ++t) {
            const double S = (double)(nn * (2 * t + 1) / 2);
            const double d = S * scale + 0.5;
            if ((long long)d == t + 1) a.tie_up[t >> 5] |= 1u << (t & 31);
        }
    }
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    a.src = in.ptr;
    a.spitch = in.pitch;
    a.dst = out.ptr;
    a.dpitch = out.pitch;
    cudaError_t e = box_launch(src->dtype, dst->dtype, a, exact && !force_fp64, s, force_fp64);
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

}  // namespace ipfc

extern "C" {

int ipfc_box_filter(const ipfc_image* src, ipfc_image* dst, int kw, int kh, int normalize, int border,
                    double border_value, void* stream) {
    return run_box(src, dst, kw, kh, normalize, border, border_value, (cudaStream_t)stream, false);
}

}  // extern "C"

namespace ipfc {

// filter2D forms: the FP32 CUDA-core kernel (filter2d.cu) and the
// split-precision tensor-core kernel (filter2d_tc.cu).
enum F2DForm { kF2DAuto = 0, kF2DFp32 = 1, kF2DSplit = 2 };

// Automatic choice: the tensor-core form for uint8 sources (1, 3 or 4
// channels) and kernels of 15 x 15 taps and more (many times faster than the FP32 form,
// with uint8 pixels exact and an error against the FP64 reference on a par
// with it), the FP32 CUDA-core form otherwise.  IPFC_F2D_PATH=split selects
// the tensor-core form wherever it applies, =fp32 pins the CUDA-core form.
static int f2d_auto_form(const ipfc_image* src, const ipfc_image* dst, int kw, int kh) {
    static const int forced = [] {  // read once, thread-safe initialisation
        const char* v = std::getenv("IPFC_F2D_PATH");
        return (v && std::strcmp(v, "fp32") == 0) ? kF2DFp32 : (v && std::strcmp(v, "split") == 0) ? kF2DSplit : 0;
    }();
    const bool tc_ok = filter2d_tc_eligible(src->dtype, dst->dtype, src->channels, kw, kh);
    if (forced == kF2DSplit && tc_ok) return kF2DSplit;
    if (forced == kF2DFp32) return kF2DFp32;
    return (tc_ok && src->dtype == IPFC_U8 && kw * kh >= 225) ? kF2DSplit : kF2DFp32;
}

static int run_filter2d(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax, int ay,
                        int border, double delta, double border_value, void* stream, int form, const char* fn) {
    if (!kernel || kw <= 0 || kh <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: filter2D: kernel must be a non-empty single-channel image");
    if (ax < 0) ax = kw / 2;
    if (ay < 0) ay = kh / 2;
    if (!(ax < kw && ay < kh)) return set_error(IPFC_ERR_INVALID, "ipf: filter2D: anchor outside kernel");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = check_pair(src, dst, fn, false);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    if (form == kF2DSplit && !filter2d_tc_eligible(src->dtype, dst->dtype, src->channels, kw, kh))
        return set_error(IPFC_ERR_UNSUPPORTED,
                         "ipf: %s: the tensor-core form takes uint8 (to uint8, uint16, int16, float; 1, 3 or 4 "
                         "channels) or single-channel float (to float) images and kernels up to %dx%d",
                         fn, kTcMaxKw, kTcMaxKh);
    if (form == kF2DAuto) form = f2d_auto_form(src, dst, kw, kh);
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<float4> taps;
    for (int j = 0; j < kh; ++j)
        for (int i = 0; i < kw; ++i) {
            const float w = kernel[(size_t)j * kw + i];
            if (w != 0.f) taps.push_back(make_float4(w, (float)i, (float)j, 0.f));
        }
    F2DArgs a;
    std::memset(&a, 0, sizeof(a));
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
    a.deltad = delta;
    a.bvd = border_value;
    a.ntaps = (int)taps.size();
    a.dense = a.ntaps == kw * kh;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    a.src = in.ptr;
    a.spitch = in.pitch;
    a.dst = out.ptr;
    a.dpitch = out.pitch;
    if (form == kF2DSplit) {
        cudaError_t e = filter2d_tc_launch(src->dtype, dst->dtype, in.ptr, in.pitch, out.ptr, out.pitch, a.W, a.H,
                                           a.C, kernel, kw, kh, ax, ay, border, (float)delta, (float)border_value, s);
        rc = finish(dst, &in, &out, s, fn);
        if (e != cudaSuccess) return cuda_status(e, fn);
        return rc;
    }
    float4* dtaps = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dtaps, sizeof(float4) * (taps.size() ? taps.size() : 1), s);
    if (e == cudaSuccess && !taps.empty())
        e = cudaMemcpyAsync(dtaps, taps.data(), sizeof(float4) * taps.size(), cudaMemcpyHostToDevice, s);
    a.taps = dtaps;
    if (e == cudaSuccess) e = filter2d_launch(src->dtype, dst->dtype, a, s);
    if (dtaps) cudaFreeAsync(dtaps, s);
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

}  // namespace ipfc

extern "C" {

int ipfc_filter2d(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax, int ay,
                  int border, double delta, double border_value, void* stream) {
    return run_filter2d(src, dst, kernel, kw, kh, ax, ay, border, delta, border_value, stream, kF2DAuto, "filter2D");
}

int ipfc_filter2d_fp32(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax, int ay,
                       int border, double delta, double border_value, void* stream) {
    return run_filter2d(src, dst, kernel, kw, kh, ax, ay, border, delta, border_value, stream, kF2DFp32, "filter2D");
}

int ipfc_filter2d_split(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax, int ay,
                        int border, double delta, double border_value, void* stream) {
    return run_filter2d(src, dst, kernel, kw, kh, ax, ay, border, delta, border_value, stream, kF2DSplit, "filter2D");
}

int ipfc_median_blur(const ipfc_image* src, ipfc_image* dst, int ksize, int border, void* stream) {
    const char* fn = "medianBlur";
    if (!(ksize >= 1 && ksize % 2 == 1))
        return set_error(IPFC_ERR_INVALID, "ipf: medianBlur: ksize must be odd and positive");
    if (border == IPFC_BORDER_CONSTANT)
        return set_error(IPFC_ERR_INVALID, "ipf: medianBlur: Constant border is not supported");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = check_pair(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    cudaError_t e;
    if (ksize == 1) {  // the reference returns the source unchanged
        e = cudaMemcpy2DAsync(out.ptr, (size_t)out.pitch, in.ptr, (size_t)in.pitch, (size_t)row_bytes(src),
                              (size_t)src->height, cudaMemcpyDeviceToDevice, s);
    } else {
        MedianArgs a{in.ptr, in.pitch, out.ptr, out.pitch, src->width, src->height, src->channels, ksize, border};
        e = median_launch(src->dtype, a, s);
    }
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

static int run_morph(const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int sw, int sh, int iterations,
                     bool is_min, cudaStream_t s) {
    const char* fn = is_min ? "erode" : "dilate";
    if (!se || sw <= 0 || sh <= 0)
        return set_error(IPFC_ERR_INVALID,
                         "ipf: morphology: structuring element must be a non-empty single-channel mask");
    int rc = check_pair(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    MorphArgs a;
    std::memset(&a, 0, sizeof(a));
    a.W = src->width;
    a.H = src->height;
    a.C = src->channels;
    a.sw = sw;
    a.sh = sh;
    a.ax = sw / 2;
    a.ay = sh / 2;
    a.is_min = is_min ? 1 : 0;
    a.is_rect = 1;
    for (int j = 0; j < sh; ++j)
        for (int i = 0; i < sw; ++i) {
            if (!se[(size_t)j * sw + i]) {
                a.is_rect = 0;
                continue;
            }
            if (a.noffs < kMorphMaxOffsets) a.offs[a.noffs] = make_short2((short)(i - a.ax), (short)(j - a.ay));
            ++a.noffs;
        }
    if (!a.is_rect && a.noffs > kMorphMaxOffsets)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: structuring element has more than %d members", fn,
                         kMorphMaxOffsets);
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    cudaError_t e = cudaSuccess;
    const size_t rb = (size_t)row_bytes(src);
    if (iterations <= 0) {
        e = cudaMemcpy2DAsync(out.ptr, (size_t)out.pitch, in.ptr, (size_t)in.pitch, rb, (size_t)src->height,
                              cudaMemcpyDeviceToDevice, s);
    } else {
        // Ping-pong: iteration i writes dst when (iterations - i) is even, so
        // the last one lands in dst; the other buffer is scratch.
        void* scratch = nullptr;
        const long long sp = round_up((long long)rb, 128);
        if (iterations > 1) e = cudaMallocAsync(&scratch, (size_t)(sp * src->height), s);
        const void* cur = in.ptr;
        long long cur_pitch = in.pitch;
        for (int it = 1; it <= iterations && e == cudaSuccess; ++it) {
            const bool to_dst = ((iterations - it) % 2) == 0;
            a.src = cur;
            a.spitch = cur_pitch;
            a.dst = to_dst ? out.ptr : scratch;
            a.dpitch = to_dst ? out.pitch : sp;
            e = morph_launch(src->dtype, a, s);
            cur = a.dst;
            cur_pitch = a.dpitch;
        }
        if (scratch) cudaFreeAsync(scratch, s);
    }
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

int ipfc_erode(const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w, int se_h, int iterations,
               void* stream) {
    return run_morph(src, dst, se, se_w, se_h, iterations, true, (cudaStream_t)stream);
}

int ipfc_dilate(const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w, int se_h, int iterations,
                void* stream) {
    return run_morph(src, dst, se, se_w, se_h, iterations, false, (cudaStream_t)stream);
}

}  // extern "C"
