/*
 * oracle.c -- CPU restatement of ipf's neighbourhood-filter arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it is
 * linked by the test suite, by __graft_entry__.smoke() and by the CPU-baseline
 * leg of bench.py, and by nothing that ships.  The product library never calls
 * it and has no CPU fallback.
 *
 * Every routine restates the reference algorithm in plain C with the same
 * floating-point operation order (FP64 accumulation, same summation order, no
 * FMA contraction: build with -ffp-contract=off), so that its results are
 * bit-identical to the reference's for the same inputs.  Parity is pinned two
 * ways (tests/test_oracle.py): against the reference's own known-answer
 * tests (tests/test_filter.cpp, tests/test_morphology.cpp) and against the
 * reference headers compiled into oracle/_ref/ on many seeded inputs.
 *
 * Image buffers are dense, interleaved row-major (HWC), as ipf::Image<T>
 * stores them (include/ipf/core.hpp:220-222, 389-391).
 *
 * Element type codes (shared with the C-ABI in include/ipfc.h):
 *   0 u8, 1 u16, 2 i16, 3 i32, 4 f32, 5 f64.
 * Border codes follow ipf::BorderMode's declaration order (core.hpp:183):
 *   0 Constant, 1 Replicate, 2 Reflect, 3 Reflect101, 4 Wrap.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_U8 0
#define ORC_U16 1
#define ORC_I16 2
#define ORC_I32 3
#define ORC_F32 4
#define ORC_F64 5

#define ORC_CONSTANT 0
#define ORC_REPLICATE 1
#define ORC_REFLECT 2
#define ORC_REFLECT101 3
#define ORC_WRAP 4

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

/* ---------------------------------------------------------------------------
 * Border index: include/ipf/core.hpp:187-214 (borderIndex).
 * Maps p into [0, len) by the border rule; -1 means "use the border value".
 * ------------------------------------------------------------------------- */
int orc_border_index(int p, int len, int mode) {
    if (p >= 0 && p < len) return p;
    if (len <= 0) return -1;
    if (mode == ORC_CONSTANT) return -1;
    if (mode == ORC_REPLICATE) return p < 0 ? 0 : len - 1;
    if (mode == ORC_REFLECT) {
        long long per = 2LL * len, q = p % per;
        if (q < 0) q += per;
        return (int)(q < len ? q : per - 1 - q);
    }
    if (mode == ORC_REFLECT101) {
        if (len == 1) return 0;
        long long per = 2LL * len - 2, q = p % per;
        if (q < 0) q += per;
        return (int)(q < len ? q : per - q);
    }
    if (mode == ORC_WRAP) {
        int q = p % len;
        return q < 0 ? q + len : q;
    }
    return -1;
}

/* filter.hpp:28-32 (detail::borderTable): index of every padded position. */
static int* border_table(int len, int before, int after, int mode) {
    int n = len + before + after;
    int* t = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!t) return NULL;
    for (int p = 0; p < n; ++p) t[p] = orc_border_index(p - before, len, mode);
    return t;
}

/* ---------------------------------------------------------------------------
 * Element access and saturate_cast (core.hpp:69-103).
 * Float -> integer: NaN -> 0, d += (d < 0 ? -0.5 : 0.5) in double, saturate
 * at the type's limits, then truncate.  Float -> float: plain conversion.
 * ------------------------------------------------------------------------- */
static double load_elem(const void* p, int dt, size_t i) {
    switch (dt) {
        case ORC_U8: return (double)((const uint8_t*)p)[i];
        case ORC_U16: return (double)((const uint16_t*)p)[i];
        case ORC_I16: return (double)((const int16_t*)p)[i];
        case ORC_I32: return (double)((const int32_t*)p)[i];
        case ORC_F32: return (double)((const float*)p)[i];
        default: return ((const double*)p)[i];
    }
}

static void range_of(int dt, double* lo, double* hi) {
    switch (dt) {
        case ORC_U8: *lo = 0; *hi = 255; break;
        case ORC_U16: *lo = 0; *hi = 65535; break;
        case ORC_I16: *lo = -32768; *hi = 32767; break;
        default: *lo = -2147483648.0; *hi = 2147483647.0; break;
    }
}

static void store_sat(void* p, int dt, size_t i, double v) {
    if (dt == ORC_F32) { ((float*)p)[i] = (float)v; return; }
    if (dt == ORC_F64) { ((double*)p)[i] = v; return; }
    double lo, hi;
    range_of(dt, &lo, &hi);
    long long r;
    if (!(v == v)) {
        r = 0;
    } else {
        double d = v < 0 ? v - 0.5 : v + 0.5;
        if (d <= lo) r = (long long)lo;
        else if (d >= hi) r = (long long)hi;
        else r = (long long)d; /* truncation toward zero */
    }
    switch (dt) {
        case ORC_U8: ((uint8_t*)p)[i] = (uint8_t)r; break;
        case ORC_U16: ((uint16_t*)p)[i] = (uint16_t)r; break;
        case ORC_I16: ((int16_t*)p)[i] = (int16_t)r; break;
        default: ((int32_t*)p)[i] = (int32_t)r; break;
    }
}

/* Same-type copy used where the reference returns the source unchanged. */
static size_t elem_size(int dt) {
    static const size_t sz[] = {1, 2, 2, 4, 4, 8};
    return (dt >= 0 && dt <= 5) ? sz[dt] : 0;
}

double orc_saturate(double v, int dt) {
    /* Scalar probe of the cast above, for the tests. */
    union { uint8_t u8; uint16_t u16; int16_t i16; int32_t i32; float f; double d; } u;
    store_sat(&u, dt, 0, v);
    return load_elem(&u, dt, 0);
}

/* ---------------------------------------------------------------------------
 * Tap generators.
 * ------------------------------------------------------------------------- */

/* filter.hpp:129-145 (gaussianKernel1D).  Writes up to cap taps; returns the
 * kernel length, or -1 for invalid arguments. */
int orc_gaussian_kernel_1d(double sigma, int ksize, double* out, int cap) {
    if (ksize <= 0) {
        if (!(sigma > 0)) return -1;
        int r = (int)(3.0 * sigma + 0.5);
        ksize = 2 * (r > 1 ? r : 1) + 1;
    }
    if (ksize % 2 != 1) return -1;
    if (sigma <= 0) sigma = 0.3 * ((ksize - 1) * 0.5 - 1) + 0.8;
    if (ksize > cap) return ksize; /* caller retries with room */
    const int c = ksize / 2;
    double sum = 0;
    for (int i = 0; i < ksize; ++i) {
        out[i] = exp(-0.5 * (i - c) * (i - c) / (sigma * sigma));
        sum += out[i];
    }
    for (int i = 0; i < ksize; ++i) out[i] /= sum;
    return ksize;
}

/* filter.hpp:93-114 (detail::derivKernel): binomial smoothing convolved with
 * (-1, 1) `order` times.  Returns the length or -1. */
int orc_deriv_kernel(int order, int ksize, double* out, int cap) {
    if (ksize == 1) {
        if (cap < 3) return -1;
        if (order == 0) { out[0] = 1; return 1; }
        if (order == 1) { out[0] = -1; out[1] = 0; out[2] = 1; return 3; }
        if (order == 2) { out[0] = 1; out[1] = -2; out[2] = 1; return 3; }
        return -1;
    }
    if (ksize % 2 != 1 || ksize < 3 || ksize > 31) return -1;
    if (order < 0 || order >= ksize || cap < ksize) return -1;
    double k[32], r[32];
    int n = 1;
    k[0] = 1.0;
    for (int step = 0; step < ksize - 1; ++step) {
        const double a = step < ksize - 1 - order ? 1.0 : -1.0, b = 1.0;
        for (int i = 0; i <= n; ++i) r[i] = 0.0;
        for (int i = 0; i < n; ++i) {
            r[i] += k[i] * a;
            r[i + 1] += k[i] * b;
        }
        ++n;
        for (int i = 0; i < n; ++i) k[i] = r[i];
    }
    for (int i = 0; i < n; ++i) out[i] = k[i];
    return n;
}

/* morphology.hpp:24-49 (getStructuringElement): 0 Rect, 1 Cross, 2 Ellipse. */
int orc_structuring_element(int shape, int width, int height, uint8_t* out) {
    if (height <= 0) height = width;
    if (width <= 0 || height <= 0) return ORC_EINVAL;
    memset(out, 0, (size_t)width * height);
    const int r = height / 2, c = width / 2;
    const double inv_r2 = r ? 1.0 / ((double)r * r) : 0.0;
    for (int i = 0; i < height; ++i) {
        int j1 = 0, j2 = 0;
        if (shape == 0 || (shape == 1 && i == r)) {
            j1 = 0;
            j2 = width;
        } else if (shape == 1) {
            j1 = c;
            j2 = c + 1;
        } else {
            const int dy = i - r;
            if (abs(dy) <= r) {
                /* saturate_cast<int>(double): round half away from zero */
                const double v = c * sqrt((r * r - dy * dy) * inv_r2);
                const int dx = (int)(v + 0.5);
                j1 = c - dx > 0 ? c - dx : 0;
                j2 = c + dx + 1 < width ? c + dx + 1 : width;
            }
        }
        for (int j = j1; j < j2; ++j) out[(size_t)i * width + j] = 1;
    }
    return ORC_OK;
}

/* ---------------------------------------------------------------------------
 * Separable correlation: filter.hpp:37-90 (detail::sepFilterImpl).
 * Pass 1 fills an FP64 intermediate of (H + kh - 1) padded rows, each the
 * horizontal correlation of a border-extended source row, accumulated tap by
 * tap from 0.0.  Pass 2 starts every output at delta, adds the vertical taps
 * in order, and saturates to the output type.
 * ------------------------------------------------------------------------- */
int orc_sep_filter(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const double* kx, int kw,
                   const double* ky, int kh, int ax, int ay, int border, double delta, double border_value) {
    if (kw <= 0 || kh <= 0) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    int* xt = border_table(W, ax, kw - 1 - ax, border);
    int* yt = border_table(H, ay, kh - 1 - ay, border);
    const int PH = H + kh - 1, PW = W + kw - 1;
    const size_t row = (size_t)W * C;
    double* tmp = (double*)malloc(sizeof(double) * (size_t)PH * row);
    double* pad = (double*)malloc(sizeof(double) * (size_t)PW * C);
    double* acc = (double*)malloc(sizeof(double) * row);
    if (!xt || !yt || !tmp || !pad || !acc) {
        free(xt); free(yt); free(tmp); free(pad); free(acc);
        return ORC_ENOMEM;
    }
    for (int py = 0; py < PH; ++py) {
        const int sy = yt[py];
        for (int px = 0; px < PW; ++px)
            for (int c = 0; c < C; ++c)
                pad[(size_t)px * C + c] = (sy < 0 || xt[px] < 0)
                                              ? border_value
                                              : load_elem(src, sdt, ((size_t)sy * W + xt[px]) * C + c);
        double* t = tmp + (size_t)py * row;
        for (size_t q = 0; q < row; ++q) t[q] = 0.0;
        for (int i = 0; i < kw; ++i) {
            const double k = kx[i];
            const double* b = pad + (size_t)i * C;
            for (size_t q = 0; q < row; ++q) t[q] += k * b[q];
        }
    }
    for (int y = 0; y < H; ++y) {
        for (size_t q = 0; q < row; ++q) acc[q] = delta;
        for (int j = 0; j < kh; ++j) {
            const double k = ky[j];
            const double* r = tmp + (size_t)(y + j) * row;
            for (size_t q = 0; q < row; ++q) acc[q] += k * r[q];
        }
        for (size_t q = 0; q < row; ++q) store_sat(dst, ddt, (size_t)y * row + q, acc[q]);
    }
    free(xt); free(yt); free(tmp); free(pad); free(acc);
    return ORC_OK;
}

/* ---------------------------------------------------------------------------
 * Dense correlation: filter.hpp:159-194 (filter2D).  Taps are float32; zero
 * taps are dropped; each sample starts at delta and adds the remaining taps in
 * row-major order in FP64, then saturates.
 * ------------------------------------------------------------------------- */
/* Output rows [y0, y1) of filter2D over the whole image; dst holds only those
 * rows (y1 - y0 rows of W*C samples).  Lets a test check full-width bands of
 * a large image -- its top, bottom and interior -- without the whole image. */
int orc_filter2d_rows(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const float* kernel, int kw,
                      int kh, int ax, int ay, int border, double delta, double border_value, int y0, int y1);

int orc_filter2d(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const float* kernel, int kw, int kh,
                 int ax, int ay, int border, double delta, double border_value) {
    return orc_filter2d_rows(src, sdt, W, H, C, dst, ddt, kernel, kw, kh, ax, ay, border, delta, border_value, 0, H);
}

int orc_filter2d_rows(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const float* kernel, int kw,
                      int kh, int ax, int ay, int border, double delta, double border_value, int y0, int y1) {
    if (kw <= 0 || kh <= 0) return ORC_EINVAL;
    if (y0 < 0) y0 = 0;
    if (y1 > H) y1 = H;
    if (ax < 0) ax = kw / 2;
    if (ay < 0) ay = kh / 2;
    if (ax >= kw || ay >= kh) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    int ntap = 0;
    int* tdx = (int*)malloc(sizeof(int) * (size_t)kw * kh);
    int* tdy = (int*)malloc(sizeof(int) * (size_t)kw * kh);
    double* tw = (double*)malloc(sizeof(double) * (size_t)kw * kh);
    int* xt = border_table(W, ax, kw - 1 - ax, border);
    int* yt = border_table(H, ay, kh - 1 - ay, border);
    if (!tdx || !tdy || !tw || !xt || !yt) {
        free(tdx); free(tdy); free(tw); free(xt); free(yt);
        return ORC_ENOMEM;
    }
    for (int j = 0; j < kh; ++j)
        for (int i = 0; i < kw; ++i) {
            const float w = kernel[(size_t)j * kw + i];
            if (w != 0.f) {
                tdx[ntap] = i;
                tdy[ntap] = j;
                tw[ntap] = (double)w;
                ++ntap;
            }
        }
    for (int y = y0; y < y1; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < C; ++c) {
                double s = delta;
                for (int t = 0; t < ntap; ++t) {
                    const int sx = xt[x + tdx[t]], sy = yt[y + tdy[t]];
                    s += tw[t] * ((sx < 0 || sy < 0) ? border_value
                                                     : load_elem(src, sdt, ((size_t)sy * W + sx) * C + c));
                }
                store_sat(dst, ddt, ((size_t)(y - y0) * W + x) * C + c, s);
            }
    free(tdx); free(tdy); free(tw); free(xt); free(yt);
    return ORC_OK;
}

/* ---------------------------------------------------------------------------
 * Box filter: filter.hpp:206-253 (boxFilter).  Horizontal window sums by a
 * running add/subtract per padded row, then vertical running column sums,
 * each output = column sum * (normalize ? 1/(kw*kh) : 1), saturated.
 * Anchor at (kw/2, kh/2), also for even sizes.
 * ------------------------------------------------------------------------- */
int orc_box_filter(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, int kw, int kh, int normalize,
                   int border, double border_value) {
    if (kw <= 0 || kh <= 0) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    const int ax = kw / 2, ay = kh / 2;
    int* xt = border_table(W, ax, kw - 1 - ax, border);
    int* yt = border_table(H, ay, kh - 1 - ay, border);
    const int PH = H + kh - 1;
    const size_t row = (size_t)W * C;
    double* rows = (double*)malloc(sizeof(double) * (size_t)PH * row);
    double* col = (double*)malloc(sizeof(double) * row);
    if (!xt || !yt || !rows || !col) {
        free(xt); free(yt); free(rows); free(col);
        return ORC_ENOMEM;
    }
    for (int py = 0; py < PH; ++py) {
        const int sy = yt[py];
        double* r = rows + (size_t)py * row;
        for (int c = 0; c < C; ++c) {
#define BOXVAL(px) ((sy < 0 || xt[(px)] < 0) ? border_value : load_elem(src, sdt, ((size_t)sy * W + xt[(px)]) * C + c))
            double s = 0;
            for (int i = 0; i < kw; ++i) s += BOXVAL(i);
            r[c] = s;
            for (int x = 1; x < W; ++x) {
                s += BOXVAL(x + kw - 1) - BOXVAL(x - 1);
                r[(size_t)x * C + c] = s;
            }
#undef BOXVAL
        }
    }
    const double scale = normalize ? 1.0 / ((double)kw * kh) : 1.0;
    for (size_t q = 0; q < row; ++q) {
        double s = 0.0;
        for (int j = 0; j < kh; ++j) s += rows[(size_t)j * row + q];
        col[q] = s;
    }
    for (int y = 0; y < H; ++y) {
        for (size_t q = 0; q < row; ++q) store_sat(dst, ddt, (size_t)y * row + q, col[q] * scale);
        if (y + 1 < H)
            for (size_t q = 0; q < row; ++q)
                col[q] += rows[(size_t)(y + kh) * row + q] - rows[(size_t)y * row + q];
    }
    free(xt); free(yt); free(rows); free(col);
    return ORC_OK;
}

/* ---------------------------------------------------------------------------
 * Median: filter.hpp:302-332 (medianBlur) and 271-297 (Huang histogram path).
 * Both reference paths return the value of rank k*k/2 of the window, so one
 * selection routine restates both.  Constant border is an error; ksize 1 and
 * empty images return the source.
 * ------------------------------------------------------------------------- */
static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

int orc_median_blur(const void* src, int dt, int W, int H, int C, void* dst, int ksize, int border) {
    if (ksize < 1 || ksize % 2 != 1) return ORC_EINVAL;
    if (border == ORC_CONSTANT) return ORC_EINVAL;
    const size_t total = (size_t)W * H * C;
    if (W <= 0 || H <= 0) return ORC_OK;
    if (ksize == 1) {
        memcpy(dst, src, total * elem_size(dt));
        return ORC_OK;
    }
    const int r = ksize / 2;
    int* xt = border_table(W, r, r, border);
    int* yt = border_table(H, r, r, border);
    const size_t n = (size_t)ksize * ksize;
    double* win = (double*)malloc(sizeof(double) * n);
    if (!xt || !yt || !win) {
        free(xt); free(yt); free(win);
        return ORC_ENOMEM;
    }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < C; ++c) {
                size_t k = 0;
                for (int j = 0; j < ksize; ++j)
                    for (int i = 0; i < ksize; ++i)
                        win[k++] = load_elem(src, dt, ((size_t)yt[y + j] * W + xt[x + i]) * C + c);
                qsort(win, n, sizeof(double), cmp_double);
                store_sat(dst, dt, ((size_t)y * W + x) * C + c, win[n / 2]);
            }
    free(xt); free(yt); free(win);
    return ORC_OK;
}

/* ---------------------------------------------------------------------------
 * Erosion / dilation: morphology.hpp:53-107 (detail::morphOnce), 112-127.
 * An all-ones element runs as a row pass then a column pass over windows
 * clipped to the image; any other element visits its offsets, skipping those
 * outside the image, starting from the centre sample and replacing it with
 * the first in-image value.  No border mode: outside pixels never count.
 * ------------------------------------------------------------------------- */
static void morph_once(const double* s, double* d, double* tmp, int W, int H, int C, const uint8_t* se, int sw,
                       int sh, int is_min) {
    const int ax = sw / 2, ay = sh / 2;
    int is_rect = 1;
    for (int i = 0; i < sw * sh; ++i)
        if (!se[i]) is_rect = 0;
#define BETTER(a, b) (is_min ? ((a) < (b)) : ((b) < (a)))
#define AT(buf, x, y, c) (buf)[((size_t)(y) * W + (x)) * C + (c)]
    if (is_rect) {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                for (int c = 0; c < C; ++c) {
                    double v = AT(s, x, y, c);
                    const int i0 = x - ax > 0 ? x - ax : 0, i1 = x - ax + sw - 1 < W - 1 ? x - ax + sw - 1 : W - 1;
                    for (int i = i0; i <= i1; ++i)
                        if (BETTER(AT(s, i, y, c), v)) v = AT(s, i, y, c);
                    AT(tmp, x, y, c) = v;
                }
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                for (int c = 0; c < C; ++c) {
                    double v = AT(tmp, x, y, c);
                    const int j0 = y - ay > 0 ? y - ay : 0, j1 = y - ay + sh - 1 < H - 1 ? y - ay + sh - 1 : H - 1;
                    for (int j = j0; j <= j1; ++j)
                        if (BETTER(AT(tmp, x, j, c), v)) v = AT(tmp, x, j, c);
                    AT(d, x, y, c) = v;
                }
        return;
    }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < C; ++c) {
                int any = 0;
                double v = AT(s, x, y, c);
                for (int j = 0; j < sh; ++j)
                    for (int i = 0; i < sw; ++i) {
                        if (!se[(size_t)j * sw + i]) continue;
                        const int sx = x + i - ax, sy = y + j - ay;
                        if (sx < 0 || sy < 0 || sx >= W || sy >= H) continue;
                        const double sv = AT(s, sx, sy, c);
                        if (!any || BETTER(sv, v)) v = sv;
                        any = 1;
                    }
                AT(d, x, y, c) = v;
            }
#undef AT
#undef BETTER
}

int orc_morph(const void* src, int dt, int W, int H, int C, void* dst, const uint8_t* se, int sw, int sh, int is_erode,
              int iterations) {
    if (sw <= 0 || sh <= 0) return ORC_EINVAL;
    const size_t total = (size_t)W * H * C;
    if (total == 0) return ORC_OK;
    double* a = (double*)malloc(sizeof(double) * total);
    double* b = (double*)malloc(sizeof(double) * total);
    double* t = (double*)malloc(sizeof(double) * total);
    if (!a || !b || !t) {
        free(a); free(b); free(t);
        return ORC_ENOMEM;
    }
    for (size_t i = 0; i < total; ++i) a[i] = load_elem(src, dt, i);
    for (int it = 0; it < iterations; ++it) {
        morph_once(a, b, t, W, H, C, se, sw, sh, is_erode);
        double* sw_ = a;
        a = b;
        b = sw_;
    }
    for (size_t i = 0; i < total; ++i) store_sat(dst, dt, i, a[i]);
    free(a); free(b); free(t);
    return ORC_OK;
}

/* ===========================================================================
 * The reference's other filters and the callers of the filters.
 * ======================================================================== */

/* ipf::PixelTraits<T>::max() (core.hpp:53-66). */
static double pixel_max(int dt) {
    switch (dt) {
        case ORC_U8: return 255.0;
        case ORC_U16: return 65535.0;
        case ORC_I16: return 32767.0;
        case ORC_I32: return 255.0;
        default: return 1.0;
    }
}

/* morphology.hpp:140-158 (morphologyEx): op 0 Erode, 1 Dilate, 2 Open,
 * 3 Close, 4 Gradient, 5 TopHat, 6 BlackHat; differences are
 * saturate_cast<T>(double(a) - double(b)). */
int orc_morphology_ex(const void* src, int dt, int W, int H, int C, void* dst, int op, const uint8_t* se, int sw,
                      int sh, int iterations) {
    if (op < 0 || op > 6) return ORC_EINVAL;
    if (op == 0) return orc_morph(src, dt, W, H, C, dst, se, sw, sh, 1, iterations);
    if (op == 1) return orc_morph(src, dt, W, H, C, dst, se, sw, sh, 0, iterations);
    const size_t n = (size_t)W * H * C, es = elem_size(dt);
    void* t1 = malloc(n * es + 1);
    void* t2 = malloc(n * es + 1);
    if (!t1 || !t2) {
        free(t1); free(t2);
        return ORC_ENOMEM;
    }
    int rc = ORC_OK;
    const void *a = NULL, *b = NULL;
    switch (op) {
        case 2:  /* dilate(erode(x)) */
            rc = orc_morph(src, dt, W, H, C, t1, se, sw, sh, 1, iterations);
            if (!rc) rc = orc_morph(t1, dt, W, H, C, dst, se, sw, sh, 0, iterations);
            break;
        case 3:  /* erode(dilate(x)) */
            rc = orc_morph(src, dt, W, H, C, t1, se, sw, sh, 0, iterations);
            if (!rc) rc = orc_morph(t1, dt, W, H, C, dst, se, sw, sh, 1, iterations);
            break;
        case 4:  /* dilate(x) - erode(x) */
            rc = orc_morph(src, dt, W, H, C, t1, se, sw, sh, 0, iterations);
            if (!rc) rc = orc_morph(src, dt, W, H, C, t2, se, sw, sh, 1, iterations);
            a = t1; b = t2;
            break;
        case 5:  /* x - open(x) */
            rc = orc_morph(src, dt, W, H, C, t1, se, sw, sh, 1, iterations);
            if (!rc) rc = orc_morph(t1, dt, W, H, C, t2, se, sw, sh, 0, iterations);
            a = src; b = t2;
            break;
        default: /* close(x) - x */
            rc = orc_morph(src, dt, W, H, C, t1, se, sw, sh, 0, iterations);
            if (!rc) rc = orc_morph(t1, dt, W, H, C, t2, se, sw, sh, 1, iterations);
            a = t2; b = src;
            break;
    }
    if (!rc && a)
        for (size_t i = 0; i < n; ++i) store_sat(dst, dt, i, load_elem(a, dt, i) - load_elem(b, dt, i));
    free(t1); free(t2);
    return rc;
}

/* filter.hpp:337-387 (bilateralFilter): circular window of radius d/2 (or
 * lround(1.5 sigmaSpace)), spatial Gaussian, range Gaussian of the L1 colour
 * distance (table by integer distance for integer images), Constant-border
 * positions skipped, FP64 throughout. */
int orc_bilateral(const void* src, int dt, int W, int H, int C, void* dst, int d, double sigma_color,
                  double sigma_space, int border) {
    if (!(sigma_color > 0 && sigma_space > 0)) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    const int r = d <= 0 ? (int)lround(sigma_space * 1.5) : d / 2;
    int nt = 0;
    int* tdx = (int*)malloc(sizeof(int) * (size_t)(2 * r + 1) * (2 * r + 1));
    int* tdy = (int*)malloc(sizeof(int) * (size_t)(2 * r + 1) * (2 * r + 1));
    double* tw = (double*)malloc(sizeof(double) * (size_t)(2 * r + 1) * (2 * r + 1));
    int* xt = border_table(W, r, r, border);
    int* yt = border_table(H, r, r, border);
    double* lut = NULL;
    size_t nlut = 0;
    const double cc = -1.0 / (2 * sigma_color * sigma_color);
    if (dt != ORC_F32 && dt != ORC_F64) {
        const double max_dist = pixel_max(dt) * C;
        if (max_dist <= (1 << 20)) {
            nlut = (size_t)max_dist + 1;
            lut = (double*)malloc(sizeof(double) * nlut);
            if (lut)
                for (size_t k = 0; k < nlut; ++k) lut[k] = exp((double)(k * k) * cc);
        }
    }
    double* acc = (double*)malloc(sizeof(double) * (size_t)C);
    if (!tdx || !tdy || !tw || !xt || !yt || !acc || (nlut && !lut)) {
        free(tdx); free(tdy); free(tw); free(xt); free(yt); free(lut); free(acc);
        return ORC_ENOMEM;
    }
    for (int j = -r; j <= r; ++j)
        for (int i = -r; i <= r; ++i)
            if (i * i + j * j <= r * r) {
                tdx[nt] = i;
                tdy[nt] = j;
                tw[nt] = exp(-(i * i + j * j) / (2 * sigma_space * sigma_space));
                ++nt;
            }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t p0 = ((size_t)y * W + x) * C;
            for (int c = 0; c < C; ++c) acc[c] = 0.0;
            double wsum = 0;
            for (int t = 0; t < nt; ++t) {
                const int sx = xt[x + r + tdx[t]], sy = yt[y + r + tdy[t]];
                if (sx < 0 || sy < 0) continue;
                const size_t p = ((size_t)sy * W + sx) * C;
                double dist = 0;
                for (int c = 0; c < C; ++c) dist += fabs(load_elem(src, dt, p + c) - load_elem(src, dt, p0 + c));
                const double w = tw[t] * (lut ? lut[(size_t)dist] : exp(dist * dist * cc));
                wsum += w;
                for (int c = 0; c < C; ++c) acc[c] += w * load_elem(src, dt, p + c);
            }
            for (int c = 0; c < C; ++c) store_sat(dst, dt, p0 + c, acc[c] / wsum);
        }
    free(tdx); free(tdy); free(tw); free(xt); free(yt); free(lut); free(acc);
    return ORC_OK;
}

/* filter.hpp:527-541 (integralImage): I is (W+1) x (H+1) x C doubles,
 * I(x+1, y+1) = I(x+1, y) + (running row sum of row y up to x). */
int orc_integral(const void* src, int dt, int W, int H, int C, double* I, int squared) {
    const size_t iw = (size_t)(W + 1) * C;
    for (size_t i = 0; i < iw * (size_t)(H + 1); ++i) I[i] = 0.0;
    double* rs = (double*)malloc(sizeof(double) * (size_t)(C > 0 ? C : 1));
    if (!rs) return ORC_ENOMEM;
    for (int y = 0; y < H; ++y) {
        for (int c = 0; c < C; ++c) rs[c] = 0.0;
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < C; ++c) {
                const double v = load_elem(src, dt, ((size_t)y * W + x) * C + c);
                rs[c] += squared ? v * v : v;
                I[(size_t)(y + 1) * iw + (size_t)(x + 1) * C + c] = I[(size_t)y * iw + (size_t)(x + 1) * C + c] + rs[c];
            }
    }
    free(rs);
    return ORC_OK;
}

/* filter.hpp:554-567 (adaptiveThreshold), single channel: the local mean by
 * boxFilter (method 0) or gaussianBlur (method 1) with Replicate, in the
 * source's type; type 0 Binary, 1 BinaryInv. */
int orc_adaptive_threshold(const void* src, int dt, int W, int H, void* dst, double maxval, int method, int type,
                           int bs, double c) {
    if (bs < 3 || bs % 2 != 1 || (type != 0 && type != 1)) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    const size_t n = (size_t)W * H;
    void* mean = malloc(n * elem_size(dt) + 1);
    if (!mean) return ORC_ENOMEM;
    int rc;
    if (method == 0) {
        rc = orc_box_filter(src, dt, W, H, 1, mean, dt, bs, bs, 1, ORC_REPLICATE, 0.0);
    } else {
        double k[64];
        const int kl = orc_gaussian_kernel_1d(0.0, bs, k, 64);
        rc = kl < 0 || kl > 64 ? ORC_EINVAL
                                : orc_sep_filter(src, dt, W, H, 1, mean, dt, k, kl, k, kl, kl / 2, kl / 2,
                                                 ORC_REPLICATE, 0.0, 0.0);
    }
    if (!rc)
        for (size_t i = 0; i < n; ++i) {
            const int above = load_elem(src, dt, i) - load_elem(mean, dt, i) > -c;
            store_sat(dst, dt, i, (above == (type == 0)) ? maxval : 0.0);
        }
    free(mean);
    return rc;
}

/* geometry.hpp:504-513 (pyrDown): sepFilter2D<double> with the 5-tap binomial
 * / 16 (Reflect101), every other row and column, saturate_cast. */
int orc_pyr_down(const void* src, int dt, int W, int H, int C, void* dst) {
    if (W <= 0 || H <= 0) return ORC_OK;
    const double k[5] = {1 / 16.0, 4 / 16.0, 6 / 16.0, 4 / 16.0, 1 / 16.0};
    double* b = (double*)malloc(sizeof(double) * (size_t)W * H * C);
    if (!b) return ORC_ENOMEM;
    int rc = orc_sep_filter(src, dt, W, H, C, b, ORC_F64, k, 5, k, 5, 2, 2, ORC_REFLECT101, 0.0, 0.0);
    const int W2 = (W + 1) / 2, H2 = (H + 1) / 2;
    if (!rc)
        for (int y = 0; y < H2; ++y)
            for (int x = 0; x < W2; ++x)
                for (int c = 0; c < C; ++c)
                    store_sat(dst, dt, ((size_t)y * W2 + x) * C + c, b[((size_t)(2 * y) * W + 2 * x) * C + c]);
    free(b);
    return rc;
}

/* geometry.hpp:516-525 (pyrUp): zero insertion into a double image of twice
 * the size, then sepFilter2D<T> with the binomial / 8 (Reflect101). */
int orc_pyr_up(const void* src, int dt, int W, int H, int C, void* dst) {
    if (W <= 0 || H <= 0) return ORC_OK;
    const int W2 = 2 * W, H2 = 2 * H;
    double* up = (double*)calloc((size_t)W2 * H2 * C, sizeof(double));
    if (!up) return ORC_ENOMEM;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            for (int c = 0; c < C; ++c)
                up[((size_t)(2 * y) * W2 + 2 * x) * C + c] = load_elem(src, dt, ((size_t)y * W + x) * C + c);
    const double k[5] = {1 / 8.0, 4 / 8.0, 6 / 8.0, 4 / 8.0, 1 / 8.0};
    const int rc = orc_sep_filter(up, ORC_F64, W2, H2, C, dst, dt, k, 5, k, 5, 2, 2, ORC_REFLECT101, 0.0, 0.0);
    free(up);
    return rc;
}

/* metrics.hpp:51-78 (ssim): 11-tap Gaussian (sigma 1.5, Reflect101) means of
 * x, y, x^2, y^2, xy in FP64; the map in float; the mean over the valid
 * region (5-pixel margin when the image is larger than 10 x 10). */
int orc_ssim(const void* a, const void* b, int dt, int W, int H, int C, double* result, float* map) {
    if (W <= 0 || H <= 0) return ORC_EINVAL;
    const size_t n = (size_t)W * H * C;
    const double L = pixel_max(dt), C1 = (0.01 * L) * (0.01 * L), C2 = (0.03 * L) * (0.03 * L);
    double* buf = (double*)malloc(sizeof(double) * n * 10);
    float* mp = map ? map : (float*)malloc(sizeof(float) * n);
    if (!buf || !mp) {
        free(buf);
        if (!map) free(mp);
        return ORC_ENOMEM;
    }
    double *x = buf, *y = buf + n, *xx = buf + 2 * n, *yy = buf + 3 * n, *xy = buf + 4 * n;
    double *mx = buf + 5 * n, *my = buf + 6 * n, *sxx = buf + 7 * n, *syy = buf + 8 * n, *sxy = buf + 9 * n;
    for (size_t i = 0; i < n; ++i) {
        x[i] = load_elem(a, dt, i);
        y[i] = load_elem(b, dt, i);
        xx[i] = x[i] * x[i];
        yy[i] = y[i] * y[i];
        xy[i] = x[i] * y[i];
    }
    double g[16];
    const int gl = orc_gaussian_kernel_1d(1.5, 11, g, 16);
    double* ins[5] = {x, y, xx, yy, xy};
    double* outs[5] = {mx, my, sxx, syy, sxy};
    int rc = ORC_OK;
    for (int i = 0; i < 5 && !rc; ++i)
        rc = orc_sep_filter(ins[i], ORC_F64, W, H, C, outs[i], ORC_F64, g, gl, g, gl, gl / 2, gl / 2, ORC_REFLECT101,
                            0.0, 0.0);
    if (!rc) {
        for (size_t i = 0; i < n; ++i) {
            const double ux = mx[i], uy = my[i];
            const double vx = sxx[i] - ux * ux, vy = syy[i] - uy * uy, cxy = sxy[i] - ux * uy;
            mp[i] = (float)(((2 * ux * uy + C1) * (2 * cxy + C2)) / ((ux * ux + uy * uy + C1) * (vx + vy + C2)));
        }
        const int r = 5;
        const int valid = W > 2 * r && H > 2 * r;
        const int rx = valid ? r : 0, ry = valid ? r : 0, rw = valid ? W - 2 * r : W, rh = valid ? H - 2 * r : H;
        double s = 0;
        for (int yy0 = ry; yy0 < ry + rh; ++yy0)
            for (int xx0 = rx; xx0 < rx + rw; ++xx0)
                for (int c = 0; c < C; ++c) s += mp[((size_t)yy0 * W + xx0) * C + c];
        *result = s / ((double)rw * rh * C);
    }
    free(buf);
    if (!map) free(mp);
    return rc;
}

/* Sobel of order (dx, dy) into float (filter.hpp:395-407): derivKernel taps,
 * ksize 1 kept 3 long, `scale` folded into the horizontal taps. */
static int sobel_f32(const void* src, int dt, int W, int H, int C, float* out, int dx, int dy, int ksize,
                     double scale, int border) {
    double kx[32], ky[32];
    int nx = orc_deriv_kernel(dx, ksize, kx, 32), ny = orc_deriv_kernel(dy, ksize, ky, 32);
    if (nx < 0 || ny < 0) return ORC_EINVAL;
    if (ksize == 1) {
        if (nx == 1) { kx[0] = 0; kx[1] = 1; kx[2] = 0; nx = 3; }
        if (ny == 1) { ky[0] = 0; ky[1] = 1; ky[2] = 0; ny = 3; }
    }
    for (int i = 0; i < nx; ++i) kx[i] *= scale;
    return orc_sep_filter(src, dt, W, H, C, out, ORC_F32, kx, nx, ky, ny, nx / 2, ny / 2, border, 0.0, 0.0);
}

/* features.hpp:111-142 (detail::structureTensor, cornerHarris,
 * cornerMinEigenVal): single channel, float response. */
int orc_corner(const void* src, int dt, int W, int H, float* dst, int bs, int ksize, double k, int min_eig) {
    if (W <= 0 || H <= 0) return ORC_OK;
    double scale = (double)(1 << ((ksize > 0 ? ksize : 3) - 1)) * bs;
    if (dt != ORC_F32 && dt != ORC_F64) scale *= pixel_max(dt);
    scale = 1.0 / scale;
    const size_t n = (size_t)W * H;
    float* f = (float*)malloc(sizeof(float) * n * 8);
    if (!f) return ORC_ENOMEM;
    float *gx = f, *gy = f + n, *xx = f + 2 * n, *xy = f + 3 * n, *yy = f + 4 * n, *ra = f + 5 * n, *rb = f + 6 * n,
          *rc_ = f + 7 * n;
    int rc = sobel_f32(src, dt, W, H, 1, gx, 1, 0, ksize, scale, ORC_REFLECT101);
    if (!rc) rc = sobel_f32(src, dt, W, H, 1, gy, 0, 1, ksize, scale, ORC_REFLECT101);
    if (!rc) {
        for (size_t i = 0; i < n; ++i) {
            xx[i] = gx[i] * gx[i];
            xy[i] = gx[i] * gy[i];
            yy[i] = gy[i] * gy[i];
        }
        rc = orc_box_filter(xx, ORC_F32, W, H, 1, ra, ORC_F32, bs, bs, 0, ORC_REFLECT101, 0.0);
        if (!rc) rc = orc_box_filter(xy, ORC_F32, W, H, 1, rb, ORC_F32, bs, bs, 0, ORC_REFLECT101, 0.0);
        if (!rc) rc = orc_box_filter(yy, ORC_F32, W, H, 1, rc_, ORC_F32, bs, bs, 0, ORC_REFLECT101, 0.0);
    }
    if (!rc)
        for (size_t i = 0; i < n; ++i) {
            if (min_eig) {
                const double A = ra[i] * 0.5, B = rb[i], C = rc_[i] * 0.5;
                dst[i] = (float)((A + C) - sqrt((A - C) * (A - C) + B * B));
            } else {
                const double A = ra[i], B = rb[i], C = rc_[i];
                dst[i] = (float)(A * C - B * B - k * (A + C) * (A + C));
            }
        }
    free(f);
    return rc;
}

/* features.hpp:27-88 (canny): Sobel gradients (Replicate), the strongest
 * channel per pixel, non-maximum suppression, hysteresis by a worklist. */
int orc_canny(const void* src, int dt, int W, int H, int C, uint8_t* dst, double low, double high, int ksize, int l2) {
    if (!(low <= high)) return ORC_EINVAL;
    if (W <= 0 || H <= 0) return ORC_OK;
    const size_t n = (size_t)W * H;
    float* f = (float*)malloc(sizeof(float) * n * (2 * (size_t)C + 3));
    int* q = (int*)malloc(sizeof(int) * n);
    if (!f || !q) {
        free(f); free(q);
        return ORC_ENOMEM;
    }
    float *gx = f, *gy = f + n * C, *mag = f + 2 * n * C, *dx = mag + n, *dy = dx + n;
    int rc = sobel_f32(src, dt, W, H, C, gx, 1, 0, ksize, 1.0, ORC_REPLICATE);
    if (!rc) rc = sobel_f32(src, dt, W, H, C, gy, 0, 1, ksize, 1.0, ORC_REPLICATE);
    if (rc) {
        free(f); free(q);
        return rc;
    }
    for (size_t i = 0; i < n; ++i) {
        float best = -1;
        for (int c = 0; c < C; ++c) {
            const float a = gx[i * C + c], b = gy[i * C + c];
            const float m = l2 ? sqrtf(a * a + b * b) : fabsf(a) + fabsf(b);
            if (m > best) {
                best = m;
                dx[i] = a;
                dy[i] = b;
            }
        }
        mag[i] = best;
    }
    memset(dst, 0, n);
    const float tan22 = 0.41421356f;
#define ORC_M(X, Y) (((X) < 0 || (Y) < 0 || (X) >= W || (Y) >= H) ? 0.f : mag[(size_t)(Y) * W + (X)])
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            const float m = mag[i];
            if (m <= low) continue;
            const float ax = fabsf(dx[i]), ay = fabsf(dy[i]);
            int is_max;
            if (ay <= ax * tan22) {
                is_max = m > ORC_M(x - 1, y) && m >= ORC_M(x + 1, y);
            } else if (ay * tan22 >= ax) {
                is_max = m > ORC_M(x, y - 1) && m >= ORC_M(x, y + 1);
            } else {
                const int s = (dx[i] < 0) != (dy[i] < 0) ? -1 : 1;
                is_max = m > ORC_M(x - s, y - 1) && m > ORC_M(x + s, y + 1);
            }
            if (is_max) dst[i] = m > high ? 2 : 1;
        }
#undef ORC_M
    size_t head = 0, tail = 0;
    for (size_t i = 0; i < n; ++i)
        if (dst[i] == 2) q[tail++] = (int)i;
    while (head < tail) {
        const int p = q[head++], px = p % W, py = p / W;
        for (int j = -1; j <= 1; ++j)
            for (int i = -1; i <= 1; ++i) {
                const int nx = px + i, ny = py + j;
                if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
                uint8_t* s = &dst[(size_t)ny * W + nx];
                if (*s != 1) continue;
                *s = 2;
                q[tail++] = ny * W + nx;
            }
    }
    for (size_t i = 0; i < n; ++i) dst[i] = dst[i] == 2 ? 255 : 0;
    free(f); free(q);
    return ORC_OK;
}

/* filter.hpp:426-438 (laplacian): ksize 1 is filter2D<float> with the 3x3
 * kernel {0,1,0, 1,-4,1, 0,1,0}, each tap (float)(tap * scale), default
 * anchor, no delta; a larger ksize sums sobel(2, 0) and sobel(0, 2) in float. */
int orc_laplacian(const void* src, int dt, int W, int H, int C, float* dst, int ksize, double scale, int border) {
    if (W <= 0 || H <= 0) return ORC_OK;
    if (ksize == 1) {
        const float base[9] = {0, 1, 0, 1, -4, 1, 0, 1, 0};
        float k[9];
        for (int i = 0; i < 9; ++i) k[i] = (float)((double)base[i] * scale);
        return orc_filter2d(src, dt, W, H, C, dst, ORC_F32, k, 3, 3, -1, -1, border, 0.0, 0.0);
    }
    const size_t n = (size_t)W * H * C;
    float* b = (float*)malloc(n * sizeof(float));
    if (!b) return ORC_ENOMEM;
    int rc = sobel_f32(src, dt, W, H, C, dst, 2, 0, ksize, scale, border);
    if (!rc) rc = sobel_f32(src, dt, W, H, C, b, 0, 2, ksize, scale, border);
    if (!rc)
        for (size_t i = 0; i < n; ++i) dst[i] += b[i];
    free(b);
    return rc;
}

/* filter.hpp:462-467 (gradientMagnitude) over magnitude (filter.hpp:440-446):
 * hypot of sobel(1, 0) and sobel(0, 1) (Reflect101), in float. */
int orc_gradient_magnitude(const void* src, int dt, int W, int H, int C, float* dst, int ksize) {
    if (W <= 0 || H <= 0) return ORC_OK;
    const size_t n = (size_t)W * H * C;
    float* gy = (float*)malloc(n * sizeof(float));
    if (!gy) return ORC_ENOMEM;
    int rc = sobel_f32(src, dt, W, H, C, dst, 1, 0, ksize, 1.0, ORC_REFLECT101);
    if (!rc) rc = sobel_f32(src, dt, W, H, C, gy, 0, 1, ksize, 1.0, ORC_REFLECT101);
    if (!rc)
        for (size_t i = 0; i < n; ++i) dst[i] = hypotf(dst[i], gy[i]);
    free(gy);
    return rc;
}

/* filter.hpp:473-483 (unsharpMask): blurred = gaussianBlur<double>(src,
 * sigma) (Reflect101); out = saturate_cast<T>(|v - b| > threshold
 * ? v + amount * (v - b) : v), every operation in double. */
int orc_unsharp_mask(const void* src, int dt, int W, int H, int C, void* dst, double sigma, double amount,
                     double threshold) {
    if (W <= 0 || H <= 0) return ORC_OK;
    const int nk = orc_gaussian_kernel_1d(sigma, 0, NULL, 0);  /* the length only */
    if (nk < 0) return ORC_EINVAL;
    double* k = (double*)malloc((size_t)nk * sizeof(double));
    const size_t n = (size_t)W * H * C;
    double* b = (double*)malloc(n * sizeof(double));
    if (!k || !b) {
        free(k);
        free(b);
        return ORC_ENOMEM;
    }
    orc_gaussian_kernel_1d(sigma, 0, k, nk);
    int rc = orc_sep_filter(src, dt, W, H, C, b, ORC_F64, k, nk, k, nk, nk / 2, nk / 2, ORC_REFLECT101, 0.0, 0.0);
    free(k);
    if (!rc)
        for (size_t i = 0; i < n; ++i) {
            const double v = load_elem(src, dt, i), diff = v - b[i];
            store_sat(dst, dt, i, fabs(diff) > threshold ? v + amount * diff : v);
        }
    free(b);
    return rc;
}
