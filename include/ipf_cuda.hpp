// ipf_cuda.hpp -- ipf::cuda: the neighbourhood-filter functions of
// ImageProcessingFlex with the reference's own signatures, computed on a B200.
//
//   #include <ipf/ipf.hpp>        // the reference library (Image<T>, BorderMode, ...)
//   #include <ipf_cuda.hpp>       // this header; link libipfcuda.so
//
//   ipf::ImageU8 out = ipf::cuda::gaussianBlur(img, 2.0);   // was ipf::gaussianBlur
//
// Each function takes and returns ipf::Image<T> by value exactly like its
// ipf:: counterpart (same template parameters, defaults and error type); the
// call copies the image to the device, runs the CUDA kernel and copies the
// result back through the C ABI of ipfc.h.  Argument errors throw
// ipf::Error with the reference's "ipf: <function>: <reason>" text.  There
// is no CPU fallback: without a usable GPU the calls throw.
//
// Element types: all six of the reference (ImageU8, ImageU16, ImageI16,
// ImageI32, ImageF, ImageD).  Calls with an int32 or double image on either
// side accumulate in FP64 in the reference's own operation order, so their
// results match ipf's bit for bit; the others accumulate in FP32.
#pragma once

#include <ipf/filter.hpp>
#include <ipf/morphology.hpp>

#include <cstdint>
#include <type_traits>
#include <vector>

#include "ipfc.h"

namespace ipf {
namespace cuda {

namespace detail {

template <class TOut, class T>
using OutT = std::conditional_t<std::is_void<TOut>::value, T, TOut>;

template <class T>
constexpr int dtype_of() {
    if constexpr (std::is_same<T, std::uint8_t>::value) return IPFC_U8;
    else if constexpr (std::is_same<T, std::uint16_t>::value) return IPFC_U16;
    else if constexpr (std::is_same<T, std::int16_t>::value) return IPFC_I16;
    else if constexpr (std::is_same<T, std::int32_t>::value) return IPFC_I32;
    else if constexpr (std::is_same<T, float>::value) return IPFC_F32;
    else return IPFC_F64;
}

template <class T>
ipfc_image view(const Image<T>& im) {
    ipfc_image v;
    v.data = const_cast<T*>(im.data());
    v.width = im.width();
    v.height = im.height();
    v.channels = im.channels();
    v.dtype = dtype_of<T>();
    v.pitch = 0;
    v.mem = IPFC_MEM_HOST;
    return v;
}

inline void check(int rc) {
    if (rc != IPFC_OK) throw ipf::Error(ipfc_last_error());
}

}  // namespace detail

/// sepFilter2D (include/ipf/filter.hpp:197-203).
template <class TOut = void, class T>
Image<detail::OutT<TOut, T>> sepFilter2D(const Image<T>& src, const std::vector<double>& kx,
                                         const std::vector<double>& ky, BorderMode border = BorderMode::Reflect101,
                                         double delta = 0.0, double borderValue = 0.0) {
    Image<detail::OutT<TOut, T>> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_sep_filter2d(&s, &d, kx.data(), static_cast<int>(kx.size()), ky.data(),
                                    static_cast<int>(ky.size()), -1, -1, static_cast<int>(border), delta, borderValue,
                                    nullptr));
    return out;
}

/// gaussianBlur (include/ipf/filter.hpp:262-267).
template <class TOut = void, class T>
Image<detail::OutT<TOut, T>> gaussianBlur(const Image<T>& src, double sigmaX, double sigmaY = 0.0, int ksize = 0,
                                          BorderMode border = BorderMode::Reflect101) {
    Image<detail::OutT<TOut, T>> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_gaussian_blur(&s, &d, sigmaX, sigmaY, ksize, static_cast<int>(border), nullptr));
    return out;
}

/// boxFilter (include/ipf/filter.hpp:206-253).
template <class TOut = void, class T>
Image<detail::OutT<TOut, T>> boxFilter(const Image<T>& src, int kw, int kh, bool normalize = true,
                                       BorderMode border = BorderMode::Reflect101, double borderValue = 0.0) {
    Image<detail::OutT<TOut, T>> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_box_filter(&s, &d, kw, kh, normalize ? 1 : 0, static_cast<int>(border), borderValue, nullptr));
    return out;
}

/// blur (include/ipf/filter.hpp:256-259).
template <class TOut = void, class T>
Image<detail::OutT<TOut, T>> blur(const Image<T>& src, int ksize, BorderMode border = BorderMode::Reflect101) {
    return boxFilter<TOut>(src, ksize, ksize, true, border);
}

/// sobel (include/ipf/filter.hpp:395-407): float output like the reference.
template <class T>
ImageF sobel(const Image<T>& src, int dx, int dy, int ksize = 3, double scale = 1.0,
             BorderMode border = BorderMode::Reflect101) {
    ImageF out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_sobel(&s, &d, dx, dy, ksize, scale, static_cast<int>(border), nullptr));
    return out;
}

/// filter2D (include/ipf/filter.hpp:159-194).
template <class TOut = void, class T>
Image<detail::OutT<TOut, T>> filter2D(const Image<T>& src, const Kernel& kernel,
                                      BorderMode border = BorderMode::Reflect101, double delta = 0.0,
                                      Point anchor = Point(-1, -1), double borderValue = 0.0) {
    if (kernel.channels() != 1 || kernel.empty())
        throw ipf::Error("ipf: filter2D: kernel must be a non-empty single-channel image");
    Image<detail::OutT<TOut, T>> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_filter2d(&s, &d, kernel.data(), kernel.width(), kernel.height(), anchor.x, anchor.y,
                                static_cast<int>(border), delta, borderValue, nullptr));
    return out;
}

/// medianBlur (include/ipf/filter.hpp:302-332).
template <class T>
Image<T> medianBlur(const Image<T>& src, int ksize, BorderMode border = BorderMode::Replicate) {
    if (!(ksize >= 1 && ksize % 2 == 1)) throw ipf::Error("ipf: medianBlur: ksize must be odd and positive");
    if (border == BorderMode::Constant) throw ipf::Error("ipf: medianBlur: Constant border is not supported");
    if (src.empty() || ksize == 1) return src;
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_median_blur(&s, &d, ksize, static_cast<int>(border), nullptr));
    return out;
}

/// erode (include/ipf/morphology.hpp:112-118).
template <class T>
Image<T> erode(const Image<T>& src, const StructuringElement& se = getStructuringElement(MorphShape::Rect, 3),
               int iterations = 1) {
    if (se.channels() != 1 || se.empty())
        throw ipf::Error("ipf: morphology: structuring element must be a non-empty single-channel mask");
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_erode(&s, &d, se.data(), se.width(), se.height(), iterations, nullptr));
    return out;
}

/// dilate (include/ipf/morphology.hpp:121-127).
template <class T>
Image<T> dilate(const Image<T>& src, const StructuringElement& se = getStructuringElement(MorphShape::Rect, 3),
                int iterations = 1) {
    if (se.channels() != 1 || se.empty())
        throw ipf::Error("ipf: morphology: structuring element must be a non-empty single-channel mask");
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_dilate(&s, &d, se.data(), se.width(), se.height(), iterations, nullptr));
    return out;
}

/// morphologyEx (include/ipf/morphology.hpp:140-158).
template <class T>
Image<T> morphologyEx(const Image<T>& src, MorphOp op,
                      const StructuringElement& se = getStructuringElement(MorphShape::Rect, 3), int iterations = 1) {
    if (se.channels() != 1 || se.empty())
        throw ipf::Error("ipf: morphology: structuring element must be a non-empty single-channel mask");
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_morphology_ex(&s, &d, static_cast<int>(op), se.data(), se.width(), se.height(), iterations,
                                     nullptr));
    return out;
}

/// bilateralFilter (include/ipf/filter.hpp:337-387).
template <class T>
Image<T> bilateralFilter(const Image<T>& src, int d, double sigmaColor, double sigmaSpace,
                         BorderMode border = BorderMode::Reflect101) {
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), o = detail::view(out);
    detail::check(ipfc_bilateral_filter(&s, &o, d, sigmaColor, sigmaSpace, static_cast<int>(border), nullptr));
    return out;
}

/// integralImage (include/ipf/filter.hpp:527-541).
template <class T>
ImageD integralImage(const Image<T>& src, bool squared = false) {
    ImageD out(src.width() + 1, src.height() + 1, src.channels(), 0.0);
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_integral_image(&s, &d, squared ? 1 : 0, nullptr));
    return out;
}

/// adaptiveThreshold (include/ipf/filter.hpp:554-567).
template <class T>
Image<T> adaptiveThreshold(const Image<T>& src, double maxval, AdaptiveMethod method, ThresholdType type,
                           int blockSize, double C) {
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_adaptive_threshold(&s, &d, maxval, static_cast<int>(method), static_cast<int>(type), blockSize,
                                          C, nullptr));
    return out;
}

/// pyrDown (include/ipf/geometry.hpp:504-513).
template <class T>
Image<T> pyrDown(const Image<T>& src) {
    Image<T> out((src.width() + 1) / 2, (src.height() + 1) / 2, src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_pyr_down(&s, &d, nullptr));
    return out;
}

/// pyrUp (include/ipf/geometry.hpp:516-525).
template <class T>
Image<T> pyrUp(const Image<T>& src) {
    Image<T> out(src.width() * 2, src.height() * 2, src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_pyr_up(&s, &d, nullptr));
    return out;
}

/// scharr (include/ipf/filter.hpp:411-414): sepFilter2D<float> with
/// {-scale, 0, scale} along the derivative axis and {3, 10, 3} across it.
template <class T>
ImageF scharr(const Image<T>& src, int dx, int dy, double scale = 1.0, BorderMode border = BorderMode::Reflect101) {
    if (!((dx == 1 && dy == 0) || (dx == 0 && dy == 1))) throw Error("ipf: scharr: (dx, dy) must be (1,0) or (0,1)");
    const std::vector<double> d = {-scale, 0.0, scale}, s = {3.0, 10.0, 3.0};
    return dx ? ipf::cuda::sepFilter2D<float>(src, d, s, border) : ipf::cuda::sepFilter2D<float>(src, s, d, border);
}

/// prewitt (include/ipf/filter.hpp:419-422).
template <class T>
ImageF prewitt(const Image<T>& src, int dx, int dy, BorderMode border = BorderMode::Reflect101) {
    if (!((dx == 1 && dy == 0) || (dx == 0 && dy == 1))) throw Error("ipf: prewitt: (dx, dy) must be (1,0) or (0,1)");
    const std::vector<double> d = {-1.0, 0.0, 1.0}, s = {1.0, 1.0, 1.0};
    return dx ? ipf::cuda::sepFilter2D<float>(src, d, s, border) : ipf::cuda::sepFilter2D<float>(src, s, d, border);
}

/// sharpen (include/ipf/filter.hpp:487-490): filter2D with the 3x3 Laplacian sharpening kernel.
template <class T>
Image<T> sharpen(const Image<T>& src, double strength = 1.0) {
    const float s = static_cast<float>(strength);
    return ipf::cuda::filter2D(src, makeKernel(3, 3, {0, -s, 0, -s, 1 + 4 * s, -s, 0, -s, 0}));
}

/// emboss (include/ipf/filter.hpp:494-496).
template <class T>
Image<T> emboss(const Image<T>& src) {
    return ipf::cuda::filter2D(src, makeKernel(3, 3, {-2, -1, 0, -1, 1, 1, 0, 1, 2}));
}

/// laplacian (include/ipf/filter.hpp:426-438).
template <class T>
ImageF laplacian(const Image<T>& src, int ksize = 1, double scale = 1.0, BorderMode border = BorderMode::Reflect101) {
    ImageF out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_laplacian(&s, &d, ksize, scale, static_cast<int>(border), nullptr));
    return out;
}

/// gradientMagnitude (include/ipf/filter.hpp:462-467).
template <class T>
ImageF gradientMagnitude(const Image<T>& src, int ksize = 3) {
    ImageF out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_gradient_magnitude(&s, &d, ksize, nullptr));
    return out;
}

/// unsharpMask (include/ipf/filter.hpp:473-483).
template <class T>
Image<T> unsharpMask(const Image<T>& src, double sigma = 1.0, double amount = 1.0, double threshold = 0.0) {
    Image<T> out(src.width(), src.height(), src.channels());
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_unsharp_mask(&s, &d, sigma, amount, threshold, nullptr));
    return out;
}

/// ssim (include/ipf/metrics.hpp:51-78).
template <class T>
double ssim(const Image<T>& a, const Image<T>& b, ImageF* ssimMap = nullptr) {
    ipfc_image va = detail::view(a), vb = detail::view(b);
    ImageF map;
    ipfc_image vm;
    if (ssimMap) {
        map = ImageF(a.width(), a.height(), a.channels());
        vm = detail::view(map);
    }
    double r = 0;
    detail::check(ipfc_ssim(&va, &vb, &r, ssimMap ? &vm : nullptr, nullptr));
    if (ssimMap) *ssimMap = std::move(map);
    return r;
}

/// cornerHarris (include/ipf/features.hpp:128-136).
template <class T>
ImageF cornerHarris(const Image<T>& src, int blockSize = 3, int ksize = 3, double k = 0.04) {
    ImageF out(src.width(), src.height(), 1);
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_corner_harris(&s, &d, blockSize, ksize, k, nullptr));
    return out;
}

/// cornerMinEigenVal (include/ipf/features.hpp:138-146).
template <class T>
ImageF cornerMinEigenVal(const Image<T>& src, int blockSize = 3, int ksize = 3) {
    ImageF out(src.width(), src.height(), 1);
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_corner_min_eigen_val(&s, &d, blockSize, ksize, nullptr));
    return out;
}

/// canny (include/ipf/features.hpp:27-88).
template <class T>
ImageU8 canny(const Image<T>& src, double lowThreshold, double highThreshold, int ksize = 3, bool l2Gradient = false) {
    ImageU8 out(src.width(), src.height(), 1);
    ipfc_image s = detail::view(src), d = detail::view(out);
    detail::check(ipfc_canny(&s, &d, lowThreshold, highThreshold, ksize, l2Gradient ? 1 : 0, nullptr));
    return out;
}

}  // namespace cuda
}  // namespace ipf
