// compose.cu -- filters built on the neighbourhood kernels, each a drop-in
// for its ipf function:
//   morphologyEx       (include/ipf/morphology.hpp:140-158)
//   bilateralFilter    (include/ipf/filter.hpp:337-387)
//   integralImage      (include/ipf/filter.hpp:527-541)
//   adaptiveThreshold  (include/ipf/filter.hpp:554-567)
//   pyrDown / pyrUp    (include/ipf/geometry.hpp:504-525)
//   laplacian, gradientMagnitude, unsharpMask (include/ipf/filter.hpp:426-483)
// Intermediates live in stream-ordered device buffers; host images are staged
// once in and once out.  Wherever the reference computes in FP64 these
// kernels do too, in its operation order with separately rounded products
// and sums, so results match ipf bit for bit (bilateralFilter of float
// images excepted: its range weight calls exp per pixel, see there).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ipfc.h"
#include "api_internal.h"
#include "common.cuh"
#include "kernels.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;

// Dispatch on an element code: f(T{}) for the matching type.
template <typename F>
cudaError_t by_type(int dt, F&& f) {
    switch (dt) {
        case IPFC_U8: return f(uint8_t{});
        case IPFC_U16: return f(uint16_t{});
        case IPFC_I16: return f(int16_t{});
        case IPFC_I32: return f(int32_t{});
        case IPFC_F32: return f(float{});
        case IPFC_F64: return f(double{});
        default: return cudaErrorInvalidValue;
    }
}

// Nominal maximum of a pixel type (ipf::PixelTraits<T>::max(), core.hpp:53-66).
double pixel_max(int dt) {
    switch (dt) {
        case IPFC_U8: return 255.0;
        case IPFC_U16: return 65535.0;
        case IPFC_I16: return 32767.0;
        case IPFC_I32: return 255.0;
        default: return 1.0;
    }
}

// A stream-ordered device image, freed on the stream when it goes out of scope.
struct DevBuf {
    void* p = nullptr;
    long long pitch = 0;
    cudaStream_t s = nullptr;
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
    cudaError_t alloc(long long row_bytes, int rows, cudaStream_t st) {
        s = st;
        pitch = round_up(row_bytes > 0 ? row_bytes : 1, 128);
        return cudaMallocAsync(&p, (size_t)(pitch * (rows > 0 ? rows : 1)), st);
    }
};

// ---------------------------------------------------------------------------
// Elementwise kernels
// ---------------------------------------------------------------------------

// out = saturate_cast<T>(double(a) - double(b)) (morphology.hpp:142-147).
template <typename T>
__global__ void __launch_bounds__(kThreads) sub_sat_kernel(const void* a, long long ap, const void* b, long long bp,
                                                           void* o, long long op, int rowlen, int H) {
    const int y = blockIdx.y;
    const T* ra = row_ptr<T>(a, ap, y);
    const T* rb = row_ptr<T>(b, bp, y);
    T* ro = row_ptr_mut<T>(o, op, y);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x)
        ro[q] = sat_from_d<T>((double)ra[q] - (double)rb[q]);
}

cudaError_t launch_sub_sat(int dt, const void* a, long long ap, const void* b, long long bp, void* o, long long op,
                           int rowlen, int H, cudaStream_t s) {
    const int bx = (rowlen + kThreads - 1) / kThreads;
    dim3 grid(bx < 16 ? bx : 16, H);
    return by_type(dt, [&](auto t) {
        using T = decltype(t);
        sub_sat_kernel<T><<<grid, kThreads, 0, s>>>(a, ap, b, bp, o, op, rowlen, H);
        return cudaGetLastError();
    });
}

}  // namespace

}  // namespace ipfc

using namespace ipfc;

// ---------------------------------------------------------------------------
// morphologyEx
// ---------------------------------------------------------------------------
extern "C" int ipfc_morphology_ex(const ipfc_image* src, ipfc_image* dst, int op, const uint8_t* se, int se_w,
                                  int se_h, int iterations, void* stream) {
    const char* fn = "morphologyEx";
    if (op < IPFC_MORPH_ERODE || op > IPFC_MORPH_BLACKHAT)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid operation", fn);
    if (!se || se_w <= 0 || se_h <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: morphology: structuring element must be a non-empty single-channel mask");
    int rc = check_pair(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (op == IPFC_MORPH_ERODE) return ipfc_erode(src, dst, se, se_w, se_h, iterations, stream);
    if (op == IPFC_MORPH_DILATE) return ipfc_dilate(src, dst, se, se_w, se_h, iterations, stream);
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height, C = src->channels, dt = src->dtype;
    const long long rb = row_bytes(src);
    DevBuf t1, t2;
    cudaError_t e = t1.alloc(rb, H, s);
    if (e == cudaSuccess && op != IPFC_MORPH_OPEN && op != IPFC_MORPH_CLOSE) e = t2.alloc(rb, H, s);
    if (e != cudaSuccess) {
        finish(dst, &in, &out, s, fn);
        return cuda_status(e, fn);
    }
    const ipfc_image vin = dev_image(in.ptr, W, H, C, dt, in.pitch);
    ipfc_image vout = dev_image(out.ptr, W, H, C, dt, out.pitch);
    ipfc_image v1 = dev_image(t1.p, W, H, C, dt, t1.pitch);
    ipfc_image v2 = dev_image(t2.p, W, H, C, dt, t2.pitch);
    auto ero = [&](const ipfc_image* a, ipfc_image* b) { return ipfc_erode(a, b, se, se_w, se_h, iterations, stream); };
    auto dil = [&](const ipfc_image* a, ipfc_image* b) { return ipfc_dilate(a, b, se, se_w, se_h, iterations, stream); };
    switch (op) {
        case IPFC_MORPH_OPEN:  // dilate(erode(x))
            if (!(rc = ero(&vin, &v1))) rc = dil(&v1, &vout);
            break;
        case IPFC_MORPH_CLOSE:  // erode(dilate(x))
            if (!(rc = dil(&vin, &v1))) rc = ero(&v1, &vout);
            break;
        case IPFC_MORPH_GRADIENT:  // dilate(x) - erode(x)
            if (!(rc = dil(&vin, &v1)) && !(rc = ero(&vin, &v2)))
                e = launch_sub_sat(dt, v1.data, v1.pitch, v2.data, v2.pitch, out.ptr, out.pitch, W * C, H, s);
            break;
        case IPFC_MORPH_TOPHAT:  // x - open(x)
            if (!(rc = ero(&vin, &v1)) && !(rc = dil(&v1, &v2)))
                e = launch_sub_sat(dt, in.ptr, in.pitch, v2.data, v2.pitch, out.ptr, out.pitch, W * C, H, s);
            break;
        default:  // BlackHat: close(x) - x
            if (!(rc = dil(&vin, &v1)) && !(rc = ero(&v1, &v2)))
                e = launch_sub_sat(dt, v2.data, v2.pitch, in.ptr, in.pitch, out.ptr, out.pitch, W * C, H, s);
            break;
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

// ---------------------------------------------------------------------------
// bilateralFilter
// ---------------------------------------------------------------------------
namespace ipfc {
namespace {

struct BilatTap {
    int dx, dy;
    double w;  // spatial weight exp(-(dx^2 + dy^2) / (2 sigmaSpace^2)), FP64 on the host
};

struct BilatArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, C, border;
    int ntaps;
    const BilatTap* taps;  // row-major, i^2 + j^2 <= r^2
    const double* lut;     // range weights by integer L1 distance (integer images), or null
    int lut_n;
    double cc;             // -1 / (2 sigmaColor^2)
};

// One output pixel (all channels) per thread.  The reference's sequence
// per tap: skip a Constant-border position, L1 distance summed over channels
// in order, w = spatial * range, wsum += w, acc[c] += w * p[c]; then
// saturate_cast(acc[c] / wsum).  Products, sums and the quotient are rounded
// one at a time as there.
template <typename T, int CN>
__global__ void __launch_bounds__(kThreads) bilateral_kernel(const BilatArgs a) {
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * (kThreads / 32) + (threadIdx.x >> 5);
    if (x >= a.W || y >= a.H) return;
    const T* c0 = row_ptr<T>(a.src, a.spitch, y) + (size_t)x * CN;
    double p0[CN], acc[CN];
#pragma unroll
    for (int c = 0; c < CN; ++c) {
        p0[c] = (double)c0[c];
        acc[c] = 0.0;
    }
    double wsum = 0.0;
    for (int k = 0; k < a.ntaps; ++k) {
        const BilatTap t = a.taps[k];
        const int sx = border_index(x + t.dx, a.W, a.border), sy = border_index(y + t.dy, a.H, a.border);
        if (sx < 0 || sy < 0) continue;  // Constant border: outside pixels are skipped
        const T* p = row_ptr<T>(a.src, a.spitch, sy) + (size_t)sx * CN;
        double v[CN];
        double dist = 0.0;
#pragma unroll
        for (int c = 0; c < CN; ++c) {
            v[c] = (double)p[c];
            dist = __dadd_rn(dist, fabs(__dsub_rn(v[c], p0[c])));
        }
        double range;
        if (a.lut && dist < (double)a.lut_n) range = a.lut[(int)dist];
        else range = exp(__dmul_rn(__dmul_rn(dist, dist), a.cc));
        const double w = __dmul_rn(t.w, range);
        wsum = __dadd_rn(wsum, w);
#pragma unroll
        for (int c = 0; c < CN; ++c) acc[c] = __dadd_rn(acc[c], __dmul_rn(w, v[c]));
    }
    T* o = row_ptr_mut<T>(a.dst, a.dpitch, y) + (size_t)x * CN;
#pragma unroll
    for (int c = 0; c < CN; ++c) o[c] = sat_from_d<T>(__ddiv_rn(acc[c], wsum));
}

template <typename T>
cudaError_t launch_bilateral(const BilatArgs& a, cudaStream_t s) {
    dim3 grid((a.W + 31) / 32, (a.H + kThreads / 32 - 1) / (kThreads / 32));
    switch (a.C) {
        case 1: bilateral_kernel<T, 1><<<grid, kThreads, 0, s>>>(a); break;
        case 2: bilateral_kernel<T, 2><<<grid, kThreads, 0, s>>>(a); break;
        case 3: bilateral_kernel<T, 3><<<grid, kThreads, 0, s>>>(a); break;
        case 4: bilateral_kernel<T, 4><<<grid, kThreads, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace
}  // namespace ipfc

extern "C" int ipfc_bilateral_filter(const ipfc_image* src, ipfc_image* dst, int d, double sigma_color,
                                     double sigma_space, int border, void* stream) {
    const char* fn = "bilateralFilter";
    if (!(sigma_color > 0 && sigma_space > 0))
        return set_error(IPFC_ERR_INVALID, "ipf: bilateralFilter: sigmas must be positive");
    if (border < IPFC_BORDER_CONSTANT || border > IPFC_BORDER_WRAP)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid border mode", fn);
    int rc = check_pair(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    if (src->channels > 4)
        return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: at most 4 channels in this build", fn);
    const int r = d <= 0 ? (int)std::lround(sigma_space * 1.5) : d / 2;
    if (r > 64) return set_error(IPFC_ERR_UNSUPPORTED, "ipf: %s: window radius %d above this build's 64", fn, r);
    std::vector<BilatTap> taps;
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i)
            if (i * i + j * j <= r * r)
                taps.push_back({i, j, std::exp(-(i * i + j * j) / (2 * sigma_space * sigma_space))});
    const double cc = -1.0 / (2 * sigma_color * sigma_color);
    std::vector<double> lut;
    const int dt = src->dtype;
    if (dt != IPFC_F32 && dt != IPFC_F64) {  // integer images: range weights by integer distance
        const double max_dist = pixel_max(dt) * src->channels;
        if (max_dist <= (1 << 20)) {
            lut.resize((size_t)max_dist + 1);
            for (size_t k = 0; k < lut.size(); ++k) lut[k] = std::exp(static_cast<double>(k * k) * cc);
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    BilatTap* dtaps = nullptr;
    double* dlut = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dtaps, sizeof(BilatTap) * taps.size(), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtaps, taps.data(), sizeof(BilatTap) * taps.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !lut.empty()) {
        e = cudaMallocAsync((void**)&dlut, sizeof(double) * lut.size(), s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dlut, lut.data(), sizeof(double) * lut.size(), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) {
        BilatArgs a{in.ptr, in.pitch, out.ptr, out.pitch, src->width, src->height, src->channels, border,
                    (int)taps.size(), dtaps, dlut, (int)lut.size(), cc};
        e = by_type(dt, [&](auto t) { return launch_bilateral<decltype(t)>(a, s); });
    }
    if (dtaps) cudaFreeAsync(dtaps, s);
    if (dlut) cudaFreeAsync(dlut, s);
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

// ---------------------------------------------------------------------------
// integralImage
// ---------------------------------------------------------------------------
namespace ipfc {
namespace {

// Row pass: for each (row y, channel c) the running row sum R(y, x) in the
// reference's left-to-right order, written to I(x + 1, y + 1, c); row 0 and
// column 0 of I are zero.
template <typename T>
__global__ void __launch_bounds__(kThreads) integral_rows_kernel(const void* src, long long sp, double* I, long long ip,
                                                                 int W, int H, int C, int squared) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= (H + 1) * C) return;
    const int y = it / C, c = it - y * C;  // y: output row (0 = the zero row)
    double* orow = reinterpret_cast<double*>(reinterpret_cast<char*>(I) + (long long)y * ip);
    orow[c] = 0.0;
    if (y == 0) {
        for (int x = 1; x <= W; ++x) orow[(size_t)x * C + c] = 0.0;
        return;
    }
    const T* srow = row_ptr<T>(src, sp, y - 1);
    double run = 0.0;
    for (int x = 0; x < W; ++x) {
        const double v = (double)srow[(size_t)x * C + c];
        run = __dadd_rn(run, squared ? __dmul_rn(v, v) : v);
        orow[(size_t)(x + 1) * C + c] = run;
    }
}

// Column pass: I(x, y + 1) = I(x, y) + R(y, x - 1), top to bottom.
__global__ void __launch_bounds__(kThreads) integral_cols_kernel(double* I, long long ip, int W, int H, int C) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x + C;  // column 0 stays zero
    if (q >= (W + 1) * C) return;
    double acc = 0.0;
    for (int y = 1; y <= H; ++y) {
        double* p = reinterpret_cast<double*>(reinterpret_cast<char*>(I) + (long long)y * ip) + q;
        acc = __dadd_rn(acc, *p);
        *p = acc;
    }
}

}  // namespace
}  // namespace ipfc

extern "C" int ipfc_integral_image(const ipfc_image* src, ipfc_image* dst, int squared, void* stream) {
    const char* fn = "integralImage";
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (dst->dtype != IPFC_F64)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: the integral image is double (ImageD)", fn);
    if (dst->width != src->width + 1 || dst->height != src->height + 1 || dst->channels != src->channels)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: destination must be (W+1) x (H+1) with the source's channels", fn);
    int rc = check_pair_resized(src, dst, fn, false);
    if (rc == -1) {
        // empty source: I is a single zero row / column
        if (dst->width <= 0 || dst->height <= 0) return IPFC_OK;
    } else if (rc) {
        return rc;
    }
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if (src->width > 0 && src->height > 0 && (rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height, C = src->channels;
    cudaError_t e = by_type(src->dtype, [&](auto t) {
        using T = decltype(t);
        const int n = (H + 1) * C;
        integral_rows_kernel<T><<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(
            in.ptr, in.pitch, static_cast<double*>(out.ptr), out.pitch, W, H, C, squared ? 1 : 0);
        return cudaGetLastError();
    });
    if (e == cudaSuccess && W > 0 && H > 0) {
        const int n = W * C;
        integral_cols_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(static_cast<double*>(out.ptr),
                                                                               out.pitch, W, H, C);
        e = cudaGetLastError();
    }
    rc = finish(dst, &in, &out, s, fn);
    if (e != cudaSuccess) return cuda_status(e, fn);
    return rc;
}

// ---------------------------------------------------------------------------
// adaptiveThreshold
// ---------------------------------------------------------------------------
namespace ipfc {
namespace {

// out = saturate_cast<T>((double(src) - double(mean) > -C) == binary ? maxval : 0)
template <typename T>
__global__ void __launch_bounds__(kThreads) adaptive_kernel(const void* src, long long sp, const void* mean,
                                                            long long mp, void* dst, long long dp, int W, int H,
                                                            double maxval, double negc, int binary) {
    const int y = blockIdx.y;
    const T* rs = row_ptr<T>(src, sp, y);
    const T* rm = row_ptr<T>(mean, mp, y);
    T* ro = row_ptr_mut<T>(dst, dp, y);
    const T hi = sat_from_d<T>(maxval), lo = sat_from_d<T>(0.0);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const bool above = __dsub_rn((double)rs[x], (double)rm[x]) > negc;
        ro[x] = (above == (binary != 0)) ? hi : lo;
    }
}

}  // namespace
}  // namespace ipfc

extern "C" int ipfc_adaptive_threshold(const ipfc_image* src, ipfc_image* dst, double maxval, int method, int type,
                                       int block_size, double c, void* stream) {
    const char* fn = "adaptiveThreshold";
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (src->channels != 1) return set_error(IPFC_ERR_INVALID, "ipf: adaptiveThreshold: expected a single-channel image");
    if (!(block_size >= 3 && block_size % 2 == 1))
        return set_error(IPFC_ERR_INVALID, "ipf: adaptiveThreshold: blockSize must be odd and >= 3");
    if (type != IPFC_THRESH_BINARY && type != IPFC_THRESH_BINARY_INV)
        return set_error(IPFC_ERR_INVALID, "ipf: adaptiveThreshold: type must be Binary or BinaryInv");
    if (method != IPFC_ADAPTIVE_MEAN && method != IPFC_ADAPTIVE_GAUSSIAN)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: invalid method", fn);
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
    const int W = src->width, H = src->height, dt = src->dtype;
    DevBuf mean;
    cudaError_t e = mean.alloc(row_bytes(src), H, s);
    if (e == cudaSuccess) {
        const ipfc_image vin = dev_image(in.ptr, W, H, 1, dt, in.pitch);
        ipfc_image vm = dev_image(mean.p, W, H, 1, dt, mean.pitch);
        // the local mean in the source's type, as the reference forms it
        // (boxFilter / gaussianBlur with Replicate); the Gaussian in FP64 so
        // the rounded mean is the reference's own
        if (method == IPFC_ADAPTIVE_MEAN) {
            rc = run_box(&vin, &vm, block_size, block_size, 1, IPFC_BORDER_REPLICATE, 0.0, s, true);
        } else {
            std::vector<double> k;
            gaussian_taps(0.0, block_size, k);
            rc = run_sep(&vin, &vm, k.data(), (int)k.size(), k.data(), (int)k.size(), -1, -1, IPFC_BORDER_REPLICATE,
                         0.0, 0.0, s, fn, true);
        }
        if (!rc) {
            const int bx = (W + kThreads - 1) / kThreads;
            dim3 grid(bx < 16 ? bx : 16, H);
            e = by_type(dt, [&](auto t) {
                adaptive_kernel<decltype(t)><<<grid, kThreads, 0, s>>>(in.ptr, in.pitch, mean.p, mean.pitch, out.ptr,
                                                                      out.pitch, W, H, maxval, -c,
                                                                      type == IPFC_THRESH_BINARY ? 1 : 0);
                return cudaGetLastError();
            });
        }
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

// ---------------------------------------------------------------------------
// pyrDown / pyrUp
// ---------------------------------------------------------------------------
namespace ipfc {
namespace {

// out(x, y, c) = saturate_cast<T>(blurred(2x, 2y, c))
template <typename T>
__global__ void __launch_bounds__(kThreads) decimate_kernel(const double* b, long long bp, void* o, long long op, int W2,
                                                            int H2, int C) {
    const int y = blockIdx.y;
    const double* rb = reinterpret_cast<const double*>(reinterpret_cast<const char*>(b) + (long long)(2 * y) * bp);
    T* ro = row_ptr_mut<T>(o, op, y);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < W2 * C; q += gridDim.x * blockDim.x) {
        const int x = q / C, c = q - x * C;
        ro[q] = sat_from_d<T>(rb[(size_t)(2 * x) * C + c]);
    }
}

// up(2x, 2y, c) = src(x, y, c), zero elsewhere (a double image of 2W x 2H)
template <typename T>
__global__ void __launch_bounds__(kThreads) upsample_kernel(const void* s, long long sp, double* u, long long up, int W,
                                                            int H, int C) {
    const int y2 = blockIdx.y;
    double* ru = reinterpret_cast<double*>(reinterpret_cast<char*>(u) + (long long)y2 * up);
    const T* rs = (y2 & 1) ? nullptr : row_ptr<T>(s, sp, y2 >> 1);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < 2 * W * C; q += gridDim.x * blockDim.x) {
        const int x2 = q / C, c = q - x2 * C;
        ru[q] = (rs && !(x2 & 1)) ? (double)rs[(size_t)(x2 >> 1) * C + c] : 0.0;
    }
}

}  // namespace
}  // namespace ipfc

extern "C" int ipfc_pyr_down(const ipfc_image* src, ipfc_image* dst, void* stream) {
    const char* fn = "pyrDown";
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    const int W2 = (src->width + 1) / 2, H2 = (src->height + 1) / 2;
    if (dst->width != W2 || dst->height != H2 || dst->channels != src->channels || dst->dtype != src->dtype)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: destination must be ((W+1)/2) x ((H+1)/2), same type", fn);
    int rc = check_pair_resized(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height, C = src->channels;
    DevBuf blurred;
    cudaError_t e = blurred.alloc((long long)W * C * 8, H, s);
    if (e == cudaSuccess) {
        // sepFilter2D<double>(src, k, k, Reflect101), k the 5-tap binomial / 16
        const double k[5] = {1 / 16.0, 4 / 16.0, 6 / 16.0, 4 / 16.0, 1 / 16.0};
        const ipfc_image vin = dev_image(in.ptr, W, H, C, src->dtype, in.pitch);
        ipfc_image vb = dev_image(blurred.p, W, H, C, IPFC_F64, blurred.pitch);
        rc = run_sep(&vin, &vb, k, 5, k, 5, -1, -1, IPFC_BORDER_REFLECT101, 0.0, 0.0, s, fn, true);
        if (!rc) {
            const int bx = (W2 * C + kThreads - 1) / kThreads;
            dim3 grid(bx < 16 ? bx : 16, H2);
            e = by_type(src->dtype, [&](auto t) {
                decimate_kernel<decltype(t)><<<grid, kThreads, 0, s>>>(static_cast<const double*>(blurred.p),
                                                                      blurred.pitch, out.ptr, out.pitch, W2, H2, C);
                return cudaGetLastError();
            });
        }
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

extern "C" int ipfc_pyr_up(const ipfc_image* src, ipfc_image* dst, void* stream) {
    const char* fn = "pyrUp";
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (dst->width != 2 * src->width || dst->height != 2 * src->height || dst->channels != src->channels ||
        dst->dtype != src->dtype)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: destination must be 2W x 2H, same type", fn);
    int rc = check_pair_resized(src, dst, fn, true);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height, C = src->channels;
    DevBuf up;
    cudaError_t e = up.alloc((long long)2 * W * C * 8, 2 * H, s);
    if (e == cudaSuccess) {
        const int bx = (2 * W * C + kThreads - 1) / kThreads;
        dim3 grid(bx < 16 ? bx : 16, 2 * H);
        e = by_type(src->dtype, [&](auto t) {
            upsample_kernel<decltype(t)><<<grid, kThreads, 0, s>>>(in.ptr, in.pitch, static_cast<double*>(up.p),
                                                                  up.pitch, W, H, C);
            return cudaGetLastError();
        });
    }
    if (e == cudaSuccess) {
        // sepFilter2D<T>(up, k, k, Reflect101), k the 5-tap binomial / 8
        const double k[5] = {1 / 8.0, 4 / 8.0, 6 / 8.0, 4 / 8.0, 1 / 8.0};
        const ipfc_image vu = dev_image(up.p, 2 * W, 2 * H, C, IPFC_F64, up.pitch);
        ipfc_image vo = dev_image(out.ptr, 2 * W, 2 * H, C, src->dtype, out.pitch);
        rc = run_sep(&vu, &vo, k, 5, k, 5, -1, -1, IPFC_BORDER_REFLECT101, 0.0, 0.0, s, fn, true);
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

// ---------------------------------------------------------------------------
// laplacian, gradientMagnitude, unsharpMask (include/ipf/filter.hpp:426-483)
// ---------------------------------------------------------------------------
namespace ipfc {
namespace {

// out += b, float (laplacian's sum of the two second derivatives)
__global__ void __launch_bounds__(kThreads) add_f32_kernel(float* o, long long op, const float* b, long long bp,
                                                           int rowlen) {
    const int y = blockIdx.y;
    float* ro = row_ptr_mut<float>(o, op, y);
    const float* rb = reinterpret_cast<const float*>(reinterpret_cast<const char*>(b) + (long long)y * bp);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) ro[q] = ro[q] + rb[q];
}

// out = hypot(out, b) in float, rounded as the C library's hypotf rounds it:
// sqrt(x^2 + y^2) evaluated in double (both squares exact) and rounded once
// to float; an infinite operand gives +inf, a NaN propagates.
__global__ void __launch_bounds__(kThreads) hypot_f32_kernel(float* o, long long op, const float* b, long long bp,
                                                             int rowlen) {
    const int y = blockIdx.y;
    float* ro = row_ptr_mut<float>(o, op, y);
    const float* rb = reinterpret_cast<const float*>(reinterpret_cast<const char*>(b) + (long long)y * bp);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) {
        const float gx = ro[q], gy = rb[q];
        float r;
        if (isinf(gx) || isinf(gy)) {
            r = INFINITY;
        } else if (isnan(gx) || isnan(gy)) {
            r = gx + gy;
        } else {
            const double dx = gx, dy = gy;
            r = __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy))));
        }
        ro[q] = r;
    }
}

// out = saturate_cast<T>(|v - b| > threshold ? v + amount (v - b) : v), double
template <typename T>
__global__ void __launch_bounds__(kThreads) unsharp_kernel(const void* s, long long sp, const double* b, long long bp,
                                                           void* o, long long op, int rowlen, double amount,
                                                           double threshold) {
    const int y = blockIdx.y;
    const T* rs = row_ptr<T>(s, sp, y);
    const double* rb = reinterpret_cast<const double*>(reinterpret_cast<const char*>(b) + (long long)y * bp);
    T* ro = row_ptr_mut<T>(o, op, y);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) {
        const double v = (double)rs[q], diff = __dsub_rn(v, rb[q]);
        ro[q] = sat_from_d<T>(fabs(diff) > threshold ? __dadd_rn(v, __dmul_rn(amount, diff)) : v);
    }
}

dim3 rows_grid(int rowlen, int H) {
    const int bx = (rowlen + kThreads - 1) / kThreads;
    return dim3(bx < 16 ? bx : 16, H);
}

// A float destination of the source's shape (laplacian, gradientMagnitude).
int check_f32_dst(const ipfc_image* src, const ipfc_image* dst, const char* fn) {
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (dst->dtype != IPFC_F32)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: the result is float (ImageF)", fn);
    return check_pair(src, dst, fn, false);
}

// Two derivative images of the staged source: into the result view and into
// a float buffer, then a per-sample kernel joins them into the result.
template <typename Join>
int two_sobels(const ipfc_image* src, ipfc_image* dst, int dx0, int dy0, int dx1, int dy1, int ksize, double scale,
               int border, void* stream, const char* fn, Join join) {
    int rc = check_f32_dst(src, dst, fn);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height, C = src->channels;
    cudaError_t e = cudaSuccess;
    {
        DevBuf b;
        e = b.alloc((long long)W * C * 4, H, s);
        if (e == cudaSuccess) {
            const ipfc_image vin = dev_image(in.ptr, W, H, C, src->dtype, in.pitch);
            ipfc_image vo = dev_image(out.ptr, W, H, C, IPFC_F32, out.pitch);
            ipfc_image vb = dev_image(b.p, W, H, C, IPFC_F32, b.pitch);
            rc = ipfc_sobel(&vin, &vo, dx0, dy0, ksize, scale, border, s);
            if (!rc) rc = ipfc_sobel(&vin, &vb, dx1, dy1, ksize, scale, border, s);
            if (!rc) {
                join(static_cast<float*>(out.ptr), out.pitch, static_cast<const float*>(b.p), b.pitch, W * C, H, s);
                e = cudaGetLastError();
            }
        }
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

}  // namespace
}  // namespace ipfc

extern "C" int ipfc_laplacian(const ipfc_image* src, ipfc_image* dst, int ksize, double scale, int border,
                              void* stream) {
    const char* fn = "laplacian";
    if (ksize == 1) {
        // filter2D<float> with {0,1,0, 1,-4,1, 0,1,0}, each tap (float)(tap * scale)
        if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
        if (dst->dtype != IPFC_F32) return set_error(IPFC_ERR_INVALID, "ipf: %s: the result is float (ImageF)", fn);
        const float base[9] = {0, 1, 0, 1, -4, 1, 0, 1, 0};
        float k[9];
        for (int i = 0; i < 9; ++i) k[i] = (float)((double)base[i] * scale);
        return ipfc_filter2d(src, dst, k, 3, 3, -1, -1, border, 0.0, 0.0, stream);
    }
    return two_sobels(src, dst, 2, 0, 0, 2, ksize, scale, border, stream, fn,
                      [](float* o, long long op, const float* b, long long bp, int rowlen, int H, cudaStream_t s) {
                          add_f32_kernel<<<rows_grid(rowlen, H), kThreads, 0, s>>>(o, op, b, bp, rowlen);
                      });
}

extern "C" int ipfc_gradient_magnitude(const ipfc_image* src, ipfc_image* dst, int ksize, void* stream) {
    return two_sobels(src, dst, 1, 0, 0, 1, ksize, 1.0, IPFC_BORDER_REFLECT101, stream, "gradientMagnitude",
                      [](float* o, long long op, const float* b, long long bp, int rowlen, int H, cudaStream_t s) {
                          hypot_f32_kernel<<<rows_grid(rowlen, H), kThreads, 0, s>>>(o, op, b, bp, rowlen);
                      });
}

extern "C" int ipfc_unsharp_mask(const ipfc_image* src, ipfc_image* dst, double sigma, double amount, double threshold,
                                 void* stream) {
    const char* fn = "unsharpMask";
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
    const int W = src->width, H = src->height, C = src->channels;
    cudaError_t e = cudaSuccess;
    {
        DevBuf blurred;
        e = blurred.alloc((long long)W * C * 8, H, s);
        if (e == cudaSuccess) {
            // gaussianBlur<double>(src, sigma): FP64 in the reference's order
            const ipfc_image vin = dev_image(in.ptr, W, H, C, src->dtype, in.pitch);
            ipfc_image vb = dev_image(blurred.p, W, H, C, IPFC_F64, blurred.pitch);
            rc = ipfc_gaussian_blur(&vin, &vb, sigma, 0.0, 0, IPFC_BORDER_REFLECT101, s);
            if (!rc) {
                e = by_type(src->dtype, [&](auto t) {
                    unsharp_kernel<decltype(t)><<<rows_grid(W * C, H), kThreads, 0, s>>>(
                        in.ptr, in.pitch, static_cast<const double*>(blurred.p), blurred.pitch, out.ptr, out.pitch,
                        W * C, amount, threshold);
                    return cudaGetLastError();
                });
            }
        }
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}
