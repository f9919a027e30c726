// features.cu -- the reference's callers of the neighbourhood filters, on the
// GPU: ssim (include/ipf/metrics.hpp:51-78), cornerHarris / cornerMinEigenVal
// over detail::structureTensor (include/ipf/features.hpp:111-142) and canny
// (include/ipf/features.hpp:27-88).
//
// The filter steps run the separable and box kernels with FP64 accumulation
// in the reference's operation order (bit-identical intermediates); the
// per-pixel arithmetic repeats the reference's float / double expressions
// with every product, sum and quotient rounded on its own (no fused
// multiply-add), so per-pixel results match ipf bit for bit.  Two places
// differ in the last bits, by construction: the unnormalised box sums of the
// corner detectors are FP64 window sums where the reference keeps FP64
// running sums, and the SSIM mean is a parallel FP64 sum.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/ipfc.h"
#include "api_internal.h"
#include "common.cuh"

namespace ipfc {

namespace {

constexpr int kThreads = 256;

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

double pixel_max(int dt) {
    switch (dt) {
        case IPFC_U8: return 255.0;
        case IPFC_U16: return 65535.0;
        case IPFC_I16: return 32767.0;
        case IPFC_I32: return 255.0;
        default: return 1.0;
    }
}

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

dim3 row_grid(int rowlen, int H) {
    const int bx = (rowlen + kThreads - 1) / kThreads;
    return dim3(bx < 16 ? bx : 16, H);
}

// Sobel of order (dx, dy) with `scale` folded into the horizontal taps
// (filter.hpp:395-407), FP64 accumulation, into dst.
int sobel_fp64(const ipfc_image* src, ipfc_image* dst, int dx, int dy, int ksize, double scale, int border,
               cudaStream_t s, const char* fn) {
    std::vector<double> kx, ky;
    if (deriv_taps(dx, ksize, kx)) return IPFC_ERR_INVALID;
    if (deriv_taps(dy, ksize, ky)) return IPFC_ERR_INVALID;
    if (ksize == 1) {
        if (kx.size() == 1) kx = {0.0, 1.0, 0.0};
        if (ky.size() == 1) ky = {0.0, 1.0, 0.0};
    }
    for (double& v : kx) v *= scale;
    return run_sep(src, dst, kx.data(), (int)kx.size(), ky.data(), (int)ky.size(), -1, -1, border, 0.0, 0.0, s, fn,
                   true);
}

// ---------------------------------------------------------------------------
// ssim
// ---------------------------------------------------------------------------

// xx = x*x, yy = y*y, xy = x*y in FP64 (metrics.hpp:56-60)
template <typename T>
__global__ void __launch_bounds__(kThreads) ssim_products_kernel(const void* a, long long ap, const void* b, long long bp,
                                                                 double* xx, double* yy, double* xy, long long dp,
                                                                 int rowlen) {
    const int y = blockIdx.y;
    const T* ra = row_ptr<T>(a, ap, y);
    const T* rb = row_ptr<T>(b, bp, y);
    double* r0 = row_ptr_mut<double>(xx, dp, y);
    double* r1 = row_ptr_mut<double>(yy, dp, y);
    double* r2 = row_ptr_mut<double>(xy, dp, y);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < rowlen; q += gridDim.x * blockDim.x) {
        const double u = (double)ra[q], v = (double)rb[q];
        r0[q] = __dmul_rn(u, u);
        r1[q] = __dmul_rn(v, v);
        r2[q] = __dmul_rn(u, v);
    }
}

struct SsimMaps {
    const double *mx, *my, *sxx, *syy, *sxy;
    long long dp;
    float* map;
    long long mp;
    int rowlen;
    double c1, c2;
};

// the SSIM map (metrics.hpp:62-66), every operation rounded as written
__global__ void __launch_bounds__(kThreads) ssim_map_kernel(const SsimMaps m) {
    const int y = blockIdx.y;
    const double* pmx = row_ptr<double>(m.mx, m.dp, y);
    const double* pmy = row_ptr<double>(m.my, m.dp, y);
    const double* pxx = row_ptr<double>(m.sxx, m.dp, y);
    const double* pyy = row_ptr<double>(m.syy, m.dp, y);
    const double* pxy = row_ptr<double>(m.sxy, m.dp, y);
    float* out = row_ptr_mut<float>(m.map, m.mp, y);
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < m.rowlen; q += gridDim.x * blockDim.x) {
        const double ux = pmx[q], uy = pmy[q];
        const double vx = __dsub_rn(pxx[q], __dmul_rn(ux, ux));
        const double vy = __dsub_rn(pyy[q], __dmul_rn(uy, uy));
        const double cxy = __dsub_rn(pxy[q], __dmul_rn(ux, uy));
        const double num = __dmul_rn(__dadd_rn(__dmul_rn(__dmul_rn(2.0, ux), uy), m.c1),
                                     __dadd_rn(__dmul_rn(2.0, cxy), m.c2));
        const double den = __dmul_rn(__dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), m.c1),
                                     __dadd_rn(__dadd_rn(vx, vy), m.c2));
        out[q] = __double2float_rn(__ddiv_rn(num, den));
    }
}

// Sum of the map over rows [y0, y1) and samples [q0, q1): one FP64 partial
// per block (fixed order within the block), summed by one block after.
__global__ void __launch_bounds__(kThreads) ssim_partial_kernel(const float* map, long long mp, int q0, int q1, int y0,
                                                                int y1, double* partial) {
    __shared__ double red[kThreads];
    double s = 0.0;
    const int n = (q1 - q0);
    const long long total = (long long)n * (y1 - y0);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const int y = y0 + (int)(i / n), q = q0 + (int)(i % n);
        s = __dadd_rn(s, (double)row_ptr<float>(map, mp, y)[q]);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void ssim_final_kernel(const double* partial, int n, double denom, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = __dadd_rn(s, partial[i]);
    *out = __ddiv_rn(s, denom);
}

// ---------------------------------------------------------------------------
// corners
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) tensor_products_kernel(const float* dx, const float* dy, long long gp,
                                                                   float* xx, float* xy, float* yy, long long tp,
                                                                   int W) {
    const int y = blockIdx.y;
    const float* a = row_ptr<float>(dx, gp, y);
    const float* b = row_ptr<float>(dy, gp, y);
    float* o0 = row_ptr_mut<float>(xx, tp, y);
    float* o1 = row_ptr_mut<float>(xy, tp, y);
    float* o2 = row_ptr_mut<float>(yy, tp, y);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        o0[x] = __fmul_rn(a[x], a[x]);
        o1[x] = __fmul_rn(a[x], b[x]);
        o2[x] = __fmul_rn(b[x], b[x]);
    }
}

// Harris R = A C - B^2 - k (A + C)^2, or (min_eig) the smaller eigenvalue
// (A + C) - sqrt((A - C)^2 + B^2) with A, C halved (features.hpp:128-142).
__global__ void __launch_bounds__(kThreads) corner_response_kernel(const float* ga, const float* gb, const float* gc,
                                                                   long long tp, float* out, long long op, int W,
                                                                   double k, int min_eig) {
    const int y = blockIdx.y;
    const float* pa = row_ptr<float>(ga, tp, y);
    const float* pb = row_ptr<float>(gb, tp, y);
    const float* pc = row_ptr<float>(gc, tp, y);
    float* o = row_ptr_mut<float>(out, op, y);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        if (min_eig) {
            const double A = __dmul_rn((double)pa[x], 0.5), B = (double)pb[x], C = __dmul_rn((double)pc[x], 0.5);
            const double d = __dsub_rn(A, C);
            o[x] = __double2float_rn(__dsub_rn(__dadd_rn(A, C), __dsqrt_rn(__dadd_rn(__dmul_rn(d, d), __dmul_rn(B, B)))));
        } else {
            const double A = pa[x], B = pb[x], C = pc[x];
            const double t = __dadd_rn(A, C);
            o[x] = __double2float_rn(
                __dsub_rn(__dsub_rn(__dmul_rn(A, C), __dmul_rn(B, B)), __dmul_rn(__dmul_rn(k, t), t)));
        }
    }
}

// ---------------------------------------------------------------------------
// canny
// ---------------------------------------------------------------------------

// Strongest channel per pixel (features.hpp:32-48): the first channel with
// the largest magnitude (L1 |a|+|b|, or L2 sqrt(a a + b b), in float).
__global__ void __launch_bounds__(kThreads) canny_grad_kernel(const float* gx, const float* gy, long long gp, int W,
                                                              int C, int l2, float* mag, float* dxo, float* dyo,
                                                              long long fp) {
    const int y = blockIdx.y;
    const float* a = row_ptr<float>(gx, gp, y);
    const float* b = row_ptr<float>(gy, gp, y);
    float* pm = row_ptr_mut<float>(mag, fp, y);
    float* px = row_ptr_mut<float>(dxo, fp, y);
    float* py = row_ptr_mut<float>(dyo, fp, y);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        float best = -1.f, bx = 0.f, by = 0.f;
        for (int c = 0; c < C; ++c) {
            const float u = a[(size_t)x * C + c], v = b[(size_t)x * C + c];
            const float m = l2 ? __fsqrt_rn(__fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v))) : __fadd_rn(fabsf(u), fabsf(v));
            if (m > best) {
                best = m;
                bx = u;
                by = v;
            }
        }
        pm[x] = best;
        px[x] = bx;
        py[x] = by;
    }
}

// Non-maximum suppression (features.hpp:52-69): state 2 strong, 1 weak, 0 not.
__global__ void __launch_bounds__(kThreads) canny_nms_kernel(const float* mag, const float* gdx, const float* gdy,
                                                             long long fp, int W, int H, double low, double high,
                                                             unsigned char* state, long long sp) {
    const int y = blockIdx.y;
    auto M = [&](int x, int yy) -> float {
        return (x < 0 || yy < 0 || x >= W || yy >= H) ? 0.f : row_ptr<float>(mag, fp, yy)[x];
    };
    const float tan22 = 0.41421356f;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const float m = row_ptr<float>(mag, fp, y)[x];
        unsigned char st = 0;
        if ((double)m > low) {
            const float dxv = row_ptr<float>(gdx, fp, y)[x], dyv = row_ptr<float>(gdy, fp, y)[x];
            const float ax = fabsf(dxv), ay = fabsf(dyv);
            bool is_max;
            if (ay <= __fmul_rn(ax, tan22)) {
                is_max = m > M(x - 1, y) && m >= M(x + 1, y);
            } else if (__fmul_rn(ay, tan22) >= ax) {
                is_max = m > M(x, y - 1) && m >= M(x, y + 1);
            } else {
                const int sg = (dxv < 0) != (dyv < 0) ? -1 : 1;
                is_max = m > M(x - sg, y - 1) && m > M(x + sg, y + 1);
            }
            if (is_max) st = (double)m > high ? 2 : 1;
        }
        row_ptr_mut<unsigned char>(state, sp, y)[x] = st;
    }
}

// Hysteresis: weak pixels 8-connected to a strong one become strong.  Each
// CTA takes a 32 x 8 tile with a one-pixel apron in shared memory and grows
// the strong set inside it until nothing changes (at most the tile's pixel
// count of rounds), then writes back; the host relaunches until no pixel
// changed anywhere.  The fixpoint is the reference's result whatever the
// visiting order.
constexpr int kHystTX = 32, kHystTY = 8;

__global__ void __launch_bounds__(kHystTX* kHystTY) canny_hyst_kernel(unsigned char* state, long long sp, int W, int H,
                                                                      unsigned* changed) {
    __shared__ unsigned char t[kHystTY + 2][kHystTX + 2];
    __shared__ int any;
    const int tx = threadIdx.x % kHystTX, ty = threadIdx.x / kHystTX;
    const int x0 = blockIdx.x * kHystTX, y0 = blockIdx.y * kHystTY;
    for (int i = threadIdx.x; i < (kHystTY + 2) * (kHystTX + 2); i += blockDim.x) {
        const int r = i / (kHystTX + 2), c = i % (kHystTX + 2);
        const int gx = x0 + c - 1, gy = y0 + r - 1;
        t[r][c] = (gx < 0 || gy < 0 || gx >= W || gy >= H) ? 0 : row_ptr<unsigned char>(state, sp, gy)[gx];
    }
    __syncthreads();
    const int gx = x0 + tx, gy = y0 + ty;
    const bool inside = gx < W && gy < H;
    bool mine = false;  // this pixel turned strong in this launch
    for (int round = 0; round < kHystTX * kHystTY; ++round) {
        if (threadIdx.x == 0) any = 0;
        __syncthreads();
        if (inside && t[ty + 1][tx + 1] == 1) {
            bool near = false;
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) near = near || t[ty + j][tx + i] == 2;
            if (near) {
                t[ty + 1][tx + 1] = 2;
                mine = true;
                any = 1;
            }
        }
        __syncthreads();
        const int go_on = any;
        __syncthreads();  // every thread has read `any` before thread 0 resets it
        if (!go_on) break;
    }
    if (mine) {
        row_ptr_mut<unsigned char>(state, sp, gy)[gx] = 2;
        *changed = 1u;
    }
}

__global__ void __launch_bounds__(kThreads) canny_out_kernel(const unsigned char* state, long long sp, unsigned char* o,
                                                             long long op, int W) {
    const int y = blockIdx.y;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x)
        row_ptr_mut<unsigned char>(o, op, y)[x] = row_ptr<unsigned char>(state, sp, y)[x] == 2 ? 255 : 0;
}

}  // namespace

}  // namespace ipfc

using namespace ipfc;

extern "C" int ipfc_ssim(const ipfc_image* a, const ipfc_image* b, double* result, ipfc_image* ssim_map,
                         void* stream) {
    const char* fn = "ssim";
    if (!a || !b || !result) return set_error(IPFC_ERR_INVALID, "ipf: %s: null argument", fn);
    if (a->width != b->width || a->height != b->height || a->channels != b->channels || a->dtype != b->dtype ||
        a->width <= 0 || a->height <= 0)
        return set_error(IPFC_ERR_INVALID, "ipf: ssim: images must be non-empty and have the same shape");
    if (ssim_map && (ssim_map->width != a->width || ssim_map->height != a->height ||
                     ssim_map->channels != a->channels || ssim_map->dtype != IPFC_F32))
        return set_error(IPFC_ERR_INVALID, "ipf: %s: the map is float with the images' shape", fn);
    // the two images may be one buffer: check each as the source of a pair
    // with a stand-in destination
    ipfc_image stand_in = *a;
    stand_in.mem = IPFC_MEM_DEVICE;
    stand_in.pitch = 0;
    stand_in.data = reinterpret_cast<char*>(const_cast<void*>(a->data)) + 1;
    int rc = check_pair(a, &stand_in, fn, true);
    if (!rc) {
        stand_in.data = reinterpret_cast<char*>(const_cast<void*>(b->data)) + 1;
        rc = check_pair(b, &stand_in, fn, true);
    }
    if (rc) return rc == -1 ? set_error(IPFC_ERR_INVALID, "ipf: ssim: images must be non-empty and have the same shape")
                            : rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int W = a->width, H = a->height, C = a->channels, rowlen = W * C;
    const double L = pixel_max(a->dtype), C1 = (0.01 * L) * (0.01 * L), C2 = (0.03 * L) * (0.03 * L);
    DevView va, vb, vm;
    if ((rc = view_in(a, s, &va, fn))) return rc;
    if ((rc = view_in(b, s, &vb, fn))) {
        if (va.owned) cudaFreeAsync(va.ptr, s);
        return rc;
    }
    DevBuf map;
    DevBuf d[8];  // xx yy xy, then blurred x y xx yy xy
    cudaError_t e = map.alloc((long long)rowlen * 4, H, s);
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) e = d[i].alloc((long long)rowlen * 8, H, s);
    double* dres = nullptr;
    double* partial = nullptr;
    constexpr int kParts = 512;
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dres, sizeof(double), s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&partial, sizeof(double) * kParts, s);
    if (e == cudaSuccess) {
        e = by_type(a->dtype, [&](auto t) {
            ssim_products_kernel<decltype(t)><<<row_grid(rowlen, H), kThreads, 0, s>>>(
                va.ptr, va.pitch, vb.ptr, vb.pitch, static_cast<double*>(d[0].p), static_cast<double*>(d[1].p),
                static_cast<double*>(d[2].p), d[0].pitch, rowlen);
            return cudaGetLastError();
        });
    }
    // gaussianBlur(., 1.5, 1.5, 11, Reflect101) of x, y, xx, yy, xy in FP64
    std::vector<double> g;
    gaussian_taps(1.5, 11, g);
    const ipfc_image ia = dev_image(va.ptr, W, H, C, a->dtype, va.pitch);
    const ipfc_image ib = dev_image(vb.ptr, W, H, C, b->dtype, vb.pitch);
    const ipfc_image srcs[5] = {ia, ib, dev_image(d[0].p, W, H, C, IPFC_F64, d[0].pitch),
                                dev_image(d[1].p, W, H, C, IPFC_F64, d[1].pitch),
                                dev_image(d[2].p, W, H, C, IPFC_F64, d[2].pitch)};
    for (int i = 0; i < 5 && e == cudaSuccess && !rc; ++i) {
        ipfc_image o = dev_image(d[3 + i].p, W, H, C, IPFC_F64, d[3 + i].pitch);
        rc = run_sep(&srcs[i], &o, g.data(), (int)g.size(), g.data(), (int)g.size(), -1, -1,
                     IPFC_BORDER_REFLECT101, 0.0, 0.0, s, fn, true);
    }
    if (e == cudaSuccess && !rc) {
        SsimMaps m{static_cast<double*>(d[3].p), static_cast<double*>(d[4].p), static_cast<double*>(d[5].p),
                   static_cast<double*>(d[6].p), static_cast<double*>(d[7].p), d[3].pitch,
                   static_cast<float*>(map.p), map.pitch, rowlen, C1, C2};
        ssim_map_kernel<<<row_grid(rowlen, H), kThreads, 0, s>>>(m);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !rc) {
        const int r = 5;
        const bool valid = W > 2 * r && H > 2 * r;
        const int rx = valid ? r : 0, ry = valid ? r : 0, rw = valid ? W - 2 * r : W, rh = valid ? H - 2 * r : H;
        ssim_partial_kernel<<<kParts, kThreads, 0, s>>>(static_cast<float*>(map.p), map.pitch, rx * C, (rx + rw) * C,
                                                        ry, ry + rh, partial);
        ssim_final_kernel<<<1, 32, 0, s>>>(partial, kParts, (double)rw * rh * C, dres);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(result, dres, sizeof(double), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess && !rc && ssim_map) {
        if ((rc = view_out(ssim_map, s, &vm, fn)) == 0)
            e = cudaMemcpy2DAsync(vm.ptr, (size_t)vm.pitch, map.p, (size_t)map.pitch, (size_t)rowlen * 4, (size_t)H,
                                  cudaMemcpyDeviceToDevice, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // *result is read by the caller on return
    if (dres) cudaFreeAsync(dres, s);
    if (partial) cudaFreeAsync(partial, s);
    int frc = IPFC_OK;
    if (ssim_map && vm.ptr) frc = finish(ssim_map, nullptr, &vm, s, fn);
    if (vb.owned) cudaFreeAsync(vb.ptr, s);
    if (va.owned) cudaFreeAsync(va.ptr, s);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    if (frc) return frc;
    return take_device_error(s, fn);
}

namespace {

int run_corners(const ipfc_image* src, ipfc_image* dst, int block_size, int ksize, double k, bool min_eig,
                void* stream) {
    const char* fn = min_eig ? "cornerMinEigenVal" : "cornerHarris";
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (src->channels != 1)
        return set_error(IPFC_ERR_INVALID, "ipf: corner detection: expected a single-channel image");
    if (dst->dtype != IPFC_F32) return set_error(IPFC_ERR_INVALID, "ipf: %s: the response is float (ImageF)", fn);
    if (block_size <= 0) return set_error(IPFC_ERR_INVALID, "ipf: boxFilter: kernel size must be positive");
    int rc = check_pair(src, dst, fn, false);
    if (rc == -1) return IPFC_OK;
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    double scale = (double)(1 << ((ksize > 0 ? ksize : 3) - 1)) * block_size;
    if (src->dtype != IPFC_F32 && src->dtype != IPFC_F64) scale *= pixel_max(src->dtype);
    scale = 1.0 / scale;
    DevView in, out;
    if ((rc = view_in(src, s, &in, fn))) return rc;
    if ((rc = view_out(dst, s, &out, fn))) {
        finish(dst, &in, &out, s, fn);
        return rc;
    }
    const int W = src->width, H = src->height;
    DevBuf g[2], t[3], r[3];
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = g[i].alloc((long long)W * 4, H, s);
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = t[i].alloc((long long)W * 4, H, s);
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = r[i].alloc((long long)W * 4, H, s);
    const ipfc_image vin = dev_image(in.ptr, W, H, 1, src->dtype, in.pitch);
    if (e == cudaSuccess) {
        ipfc_image gx = dev_image(g[0].p, W, H, 1, IPFC_F32, g[0].pitch);
        ipfc_image gy = dev_image(g[1].p, W, H, 1, IPFC_F32, g[1].pitch);
        rc = sobel_fp64(&vin, &gx, 1, 0, ksize, scale, IPFC_BORDER_REFLECT101, s, fn);
        if (!rc) rc = sobel_fp64(&vin, &gy, 0, 1, ksize, scale, IPFC_BORDER_REFLECT101, s, fn);
    }
    if (e == cudaSuccess && !rc) {
        tensor_products_kernel<<<row_grid(W, H), kThreads, 0, s>>>(
            static_cast<float*>(g[0].p), static_cast<float*>(g[1].p), g[0].pitch, static_cast<float*>(t[0].p),
            static_cast<float*>(t[1].p), static_cast<float*>(t[2].p), t[0].pitch, W);
        e = cudaGetLastError();
    }
    for (int i = 0; i < 3 && e == cudaSuccess && !rc; ++i) {
        const ipfc_image ti = dev_image(t[i].p, W, H, 1, IPFC_F32, t[i].pitch);
        ipfc_image ri = dev_image(r[i].p, W, H, 1, IPFC_F32, r[i].pitch);
        rc = run_box(&ti, &ri, block_size, block_size, 0, IPFC_BORDER_REFLECT101, 0.0, s, true);
    }
    if (e == cudaSuccess && !rc) {
        corner_response_kernel<<<row_grid(W, H), kThreads, 0, s>>>(
            static_cast<float*>(r[0].p), static_cast<float*>(r[1].p), static_cast<float*>(r[2].p), r[0].pitch,
            static_cast<float*>(out.ptr), out.pitch, W, k, min_eig ? 1 : 0);
        e = cudaGetLastError();
    }
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}

}  // namespace

extern "C" int ipfc_corner_harris(const ipfc_image* src, ipfc_image* dst, int block_size, int ksize, double k,
                                  void* stream) {
    return run_corners(src, dst, block_size, ksize, k, false, stream);
}

extern "C" int ipfc_corner_min_eigen_val(const ipfc_image* src, ipfc_image* dst, int block_size, int ksize,
                                         void* stream) {
    return run_corners(src, dst, block_size, ksize, 0.0, true, stream);
}

extern "C" int ipfc_canny(const ipfc_image* src, ipfc_image* dst, double low_threshold, double high_threshold,
                          int ksize, int l2_gradient, void* stream) {
    const char* fn = "canny";
    if (!(low_threshold <= high_threshold))
        return set_error(IPFC_ERR_INVALID, "ipf: canny: lowThreshold must be <= highThreshold");
    if (!src || !dst) return set_error(IPFC_ERR_INVALID, "ipf: %s: null image", fn);
    if (dst->dtype != IPFC_U8 || dst->channels != 1 || dst->width != src->width || dst->height != src->height)
        return set_error(IPFC_ERR_INVALID, "ipf: %s: the edge map is uint8, single channel, the source's size", fn);
    int rc = check_pair_resized(src, dst, fn, false);
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
    DevBuf gx, gy, mag, gdx, gdy, state;
    unsigned* changed = nullptr;
    cudaError_t e = gx.alloc((long long)W * C * 4, H, s);
    if (e == cudaSuccess) e = gy.alloc((long long)W * C * 4, H, s);
    if (e == cudaSuccess) e = mag.alloc((long long)W * 4, H, s);
    if (e == cudaSuccess) e = gdx.alloc((long long)W * 4, H, s);
    if (e == cudaSuccess) e = gdy.alloc((long long)W * 4, H, s);
    if (e == cudaSuccess) e = state.alloc(W, H, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&changed, sizeof(unsigned), s);
    if (e == cudaSuccess) {
        const ipfc_image vin = dev_image(in.ptr, W, H, C, src->dtype, in.pitch);
        ipfc_image ix = dev_image(gx.p, W, H, C, IPFC_F32, gx.pitch);
        ipfc_image iy = dev_image(gy.p, W, H, C, IPFC_F32, gy.pitch);
        rc = sobel_fp64(&vin, &ix, 1, 0, ksize, 1.0, IPFC_BORDER_REPLICATE, s, fn);
        if (!rc) rc = sobel_fp64(&vin, &iy, 0, 1, ksize, 1.0, IPFC_BORDER_REPLICATE, s, fn);
    }
    if (e == cudaSuccess && !rc) {
        canny_grad_kernel<<<row_grid(W, H), kThreads, 0, s>>>(
            static_cast<float*>(gx.p), static_cast<float*>(gy.p), gx.pitch, W, C, l2_gradient ? 1 : 0,
            static_cast<float*>(mag.p), static_cast<float*>(gdx.p), static_cast<float*>(gdy.p), mag.pitch);
        canny_nms_kernel<<<row_grid(W, H), kThreads, 0, s>>>(
            static_cast<float*>(mag.p), static_cast<float*>(gdx.p), static_cast<float*>(gdy.p), mag.pitch, W, H,
            low_threshold, high_threshold, static_cast<unsigned char*>(state.p), state.pitch);
        e = cudaGetLastError();
    }
    // hysteresis: relaunch until a pass changes nothing (each pass turns at
    // least one weak pixel strong, so W*H passes bound the loop)
    dim3 hgrid((W + kHystTX - 1) / kHystTX, (H + kHystTY - 1) / kHystTY);
    for (long long pass = 0; e == cudaSuccess && !rc && pass < (long long)W * H + 1; ++pass) {
        unsigned h = 0;
        e = cudaMemsetAsync(changed, 0, sizeof(unsigned), s);
        if (e != cudaSuccess) break;
        canny_hyst_kernel<<<hgrid, kHystTX * kHystTY, 0, s>>>(static_cast<unsigned char*>(state.p), state.pitch, W, H,
                                                              changed);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, changed, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (h == 0) break;
    }
    if (e == cudaSuccess && !rc) {
        canny_out_kernel<<<row_grid(W, H), kThreads, 0, s>>>(static_cast<unsigned char*>(state.p), state.pitch,
                                                             static_cast<unsigned char*>(out.ptr), out.pitch, W);
        e = cudaGetLastError();
    }
    if (changed) cudaFreeAsync(changed, s);
    const int frc = finish(dst, &in, &out, s, fn);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, fn);
    return frc;
}
