// ref_shim.cpp -- C entry points over the reference's own headers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference
// headers where they lie (include/ipf/*.hpp of ImageProcessingFlex) into
// oracle/_ref/libipfref.so.  It is used to pin the C restatement in
// oracle/oracle.c against the reference itself, to generate the golden
// fixtures under tests/golden/, and as the timed CPU baseline (the reference's
// threaded CPU path, ipf::setNumThreads(0)).  Nothing that ships links it.
//
// Signatures mirror oracle.c's orc_* functions with a ref_ prefix; element and
// border codes are the same.
#include <ipf/features.hpp>
#include <ipf/filter.hpp>
#include <ipf/geometry.hpp>
#include <ipf/metrics.hpp>
#include <ipf/morphology.hpp>

#include <cstdint>
#include <cstring>
#include <vector>

namespace {

using namespace ipf;

template <class T>
Image<T> wrap(const void* p, int W, int H, int C) {
    return Image<T>::fromData(W, H, C, static_cast<const T*>(p));
}

template <class T>
void unwrap(const Image<T>& img, void* out) {
    if (!img.empty()) std::memcpy(out, img.data(), img.sampleCount() * sizeof(T));
}

// Calls fn.template operator()<T>() with T the element type of code dt.
template <class Fn>
int dispatch(int dt, Fn&& fn) {
    switch (dt) {
        case 0: fn(std::uint8_t{}); return 0;
        case 1: fn(std::uint16_t{}); return 0;
        case 2: fn(std::int16_t{}); return 0;
        case 3: fn(std::int32_t{}); return 0;
        case 4: fn(float{}); return 0;
        case 5: fn(double{}); return 0;
        default: return 1;
    }
}

int guard(const std::function<int()>& f) {
    try {
        return f();
    } catch (const ipf::Error&) {
        return 1;
    } catch (...) {
        return 2;
    }
}

BorderMode bm(int b) { return static_cast<BorderMode>(b); }

}  // namespace

extern "C" {

void ref_set_threads(int n) { ipf::setNumThreads(n); }
int ref_get_threads(void) { return ipf::getNumThreads(); }

int ref_gaussian_kernel_1d(double sigma, int ksize, double* out, int cap) {
    try {
        const std::vector<double> k = ipf::gaussianKernel1D(sigma, ksize);
        if (static_cast<int>(k.size()) <= cap) std::memcpy(out, k.data(), k.size() * sizeof(double));
        return static_cast<int>(k.size());
    } catch (...) {
        return -1;
    }
}

int ref_deriv_kernel(int order, int ksize, double* out, int cap) {
    try {
        const std::vector<double> k = ipf::detail::derivKernel(order, ksize);
        if (static_cast<int>(k.size()) > cap) return -1;
        std::memcpy(out, k.data(), k.size() * sizeof(double));
        return static_cast<int>(k.size());
    } catch (...) {
        return -1;
    }
}

int ref_structuring_element(int shape, int w, int h, std::uint8_t* out) {
    return guard([&] {
        const auto se = ipf::getStructuringElement(static_cast<MorphShape>(shape), w, h);
        std::memcpy(out, se.data(), se.sampleCount());
        return 0;
    });
}

int ref_sep_filter(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const double* kx, int kw,
                   const double* ky, int kh, int ax, int ay, int border, double delta, double bv) {
    return guard([&] {
        std::vector<double> vx(kx, kx + kw), vy(ky, ky + kh);
        int rc = 0;
        dispatch(sdt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, C);
            rc = dispatch(ddt, [&](auto d) {
                using D = decltype(d);
                unwrap(detail::sepFilterImpl<D>(in, vx, vy, ax, ay, bm(border), delta, bv), dst);
            });
        });
        return rc;
    });
}

int ref_gaussian_blur(const void* src, int dt, int W, int H, int C, void* dst, int ddt, double sx, double sy,
                      int ksize, int border) {
    return guard([&] {
        int rc = 0;
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, C);
            rc = dispatch(ddt, [&](auto d) {
                using D = decltype(d);
                unwrap(ipf::gaussianBlur<D>(in, sx, sy, ksize, bm(border)), dst);
            });
        });
        return rc;
    });
}

int ref_filter2d(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, const float* k, int kw, int kh,
                 int ax, int ay, int border, double delta, double bv) {
    return guard([&] {
        const Kernel kern = Kernel::fromData(kw, kh, 1, k);
        int rc = 0;
        dispatch(sdt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, C);
            rc = dispatch(ddt, [&](auto d) {
                using D = decltype(d);
                unwrap(ipf::filter2D<D>(in, kern, bm(border), delta, Point(ax, ay), bv), dst);
            });
        });
        return rc;
    });
}

int ref_box_filter(const void* src, int sdt, int W, int H, int C, void* dst, int ddt, int kw, int kh, int normalize,
                   int border, double bv) {
    return guard([&] {
        int rc = 0;
        dispatch(sdt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, C);
            rc = dispatch(ddt, [&](auto d) {
                using D = decltype(d);
                unwrap(ipf::boxFilter<D>(in, kw, kh, normalize != 0, bm(border), bv), dst);
            });
        });
        return rc;
    });
}

int ref_sobel(const void* src, int sdt, int W, int H, int C, float* dst, int dx, int dy, int ksize, double scale,
              int border) {
    return guard([&] {
        dispatch(sdt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::sobel(wrap<S>(src, W, H, C), dx, dy, ksize, scale, bm(border)), dst);
        });
        return 0;
    });
}

int ref_median_blur(const void* src, int dt, int W, int H, int C, void* dst, int ksize, int border) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::medianBlur(wrap<S>(src, W, H, C), ksize, bm(border)), dst);
        });
        return 0;
    });
}

int ref_morph(const void* src, int dt, int W, int H, int C, void* dst, const std::uint8_t* se, int sw, int sh,
              int is_erode, int iterations) {
    return guard([&] {
        const StructuringElement el = StructuringElement::fromData(sw, sh, 1, se);
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, C);
            unwrap(is_erode ? ipf::erode(in, el, iterations) : ipf::dilate(in, el, iterations), dst);
        });
        return 0;
    });
}

int ref_morphology_ex(const void* src, int dt, int W, int H, int C, void* dst, int op, const std::uint8_t* se, int sw,
                      int sh, int iterations) {
    return guard([&] {
        const StructuringElement el = StructuringElement::fromData(sw, sh, 1, se);
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::morphologyEx(wrap<S>(src, W, H, C), static_cast<MorphOp>(op), el, iterations), dst);
        });
        return 0;
    });
}

int ref_bilateral(const void* src, int dt, int W, int H, int C, void* dst, int d, double sc, double ss, int border) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::bilateralFilter(wrap<S>(src, W, H, C), d, sc, ss, bm(border)), dst);
        });
        return 0;
    });
}

int ref_integral(const void* src, int dt, int W, int H, int C, double* dst, int squared) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::integralImage(wrap<S>(src, W, H, C), squared != 0), dst);
        });
        return 0;
    });
}

int ref_adaptive_threshold(const void* src, int dt, int W, int H, void* dst, double maxval, int method, int type,
                           int bs, double c) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::adaptiveThreshold(wrap<S>(src, W, H, 1), maxval, static_cast<AdaptiveMethod>(method),
                                          static_cast<ThresholdType>(type), bs, c),
                   dst);
        });
        return 0;
    });
}

int ref_pyr_down(const void* src, int dt, int W, int H, int C, void* dst) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::pyrDown(wrap<S>(src, W, H, C)), dst);
        });
        return 0;
    });
}

int ref_pyr_up(const void* src, int dt, int W, int H, int C, void* dst) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::pyrUp(wrap<S>(src, W, H, C)), dst);
        });
        return 0;
    });
}

int ref_ssim(const void* a, const void* b, int dt, int W, int H, int C, double* result, float* map) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            ImageF m;
            *result = ipf::ssim(wrap<S>(a, W, H, C), wrap<S>(b, W, H, C), map ? &m : nullptr);
            if (map) unwrap(m, map);
        });
        return 0;
    });
}

int ref_corner(const void* src, int dt, int W, int H, float* dst, int bs, int ksize, double k, int min_eig) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            const Image<S> in = wrap<S>(src, W, H, 1);
            unwrap(min_eig ? ipf::cornerMinEigenVal(in, bs, ksize) : ipf::cornerHarris(in, bs, ksize, k), dst);
        });
        return 0;
    });
}

int ref_canny(const void* src, int dt, int W, int H, int C, std::uint8_t* dst, double low, double high, int ksize,
              int l2) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::canny(wrap<S>(src, W, H, C), low, high, ksize, l2 != 0), dst);
        });
        return 0;
    });
}

int ref_laplacian(const void* src, int dt, int W, int H, int C, float* dst, int ksize, double scale, int border) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::laplacian(wrap<S>(src, W, H, C), ksize, scale, static_cast<BorderMode>(border)), dst);
        });
        return 0;
    });
}

int ref_gradient_magnitude(const void* src, int dt, int W, int H, int C, float* dst, int ksize) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::gradientMagnitude(wrap<S>(src, W, H, C), ksize), dst);
        });
        return 0;
    });
}

int ref_unsharp_mask(const void* src, int dt, int W, int H, int C, void* dst, double sigma, double amount,
                     double threshold) {
    return guard([&] {
        dispatch(dt, [&](auto s) {
            using S = decltype(s);
            unwrap(ipf::unsharpMask(wrap<S>(src, W, H, C), sigma, amount, threshold), dst);
        });
        return 0;
    });
}

}  // extern "C"
