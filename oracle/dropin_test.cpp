// dropin_test.cpp -- the drop-in check in the reference's own language.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile against the reference
// headers (include/ipf/*.hpp) into oracle/_ref/dropin_test and linked with
// libipfcuda.so; run on a GPU by tests/test_gpu_dropin.py.  For seeded images
// it calls ipf::X and ipf::cuda::X with identical arguments and compares the
// ipf::Image results: exact for median, morphology, box on uint8 and
// integer-tap (Sobel) filters; within 1 LSB for FP32-accumulated uint8
// outputs (mismatch rate printed); 1e-5 relative for float outputs.  It also
// checks that argument errors throw ipf::Error with the reference's text.
#include <ipf/features.hpp>
#include <ipf/filter.hpp>
#include <ipf/geometry.hpp>
#include <ipf/metrics.hpp>
#include <ipf/morphology.hpp>
#include <ipf_cuda.hpp>

#include <cmath>
#include <cstdio>
#include <random>
#include <string>

using namespace ipf;

namespace {

int g_fail = 0;

template <class T>
Image<T> seeded(int w, int h, int c, unsigned seed) {
    std::mt19937 rng(seed);
    Image<T> img(w, h, c);
    for (auto& v : img) {
        if constexpr (std::is_floating_point<T>::value)
            v = static_cast<T>(std::uniform_real_distribution<double>(0.0, 1.0)(rng));
        else
            v = static_cast<T>(std::uniform_int_distribution<long long>(0, 255)(rng));
    }
    return img;
}

template <class T>
void compare(const char* what, const Image<T>& got, const Image<T>& want, double lsb, double rel) {
    if (!got.sameShape(want)) {
        std::printf("FAIL %s: shape\n", what);
        ++g_fail;
        return;
    }
    double maxd = 0;
    std::size_t mism = 0, bad = 0;
    for (std::size_t i = 0; i < want.sampleCount(); ++i) {
        const double a = static_cast<double>(got.data()[i]), b = static_cast<double>(want.data()[i]);
        const double d = std::fabs(a - b);
        maxd = std::fmax(maxd, d);
        mism += d > 0;
        const double lim = std::is_floating_point<T>::value ? rel * std::fmax(1.0, std::fabs(b)) : lsb;
        bad += d > lim;
    }
    std::printf("%s %-52s max|diff| %-10.3g mismatches %zu / %zu\n", bad ? "FAIL" : "ok  ", what, maxd, mism,
                want.sampleCount());
    g_fail += bad != 0;
}

template <class Fn>
void expect_error(const char* what, const std::string& msg, Fn fn) {
    try {
        fn();
        std::printf("FAIL %s: no ipf::Error\n", what);
        ++g_fail;
    } catch (const ipf::Error& e) {
        const bool ok = msg == e.what();
        std::printf("%s %-52s \"%s\"\n", ok ? "ok  " : "FAIL", what, e.what());
        g_fail += !ok;
    }
}

}  // namespace

int main() {
    const BorderMode modes[] = {BorderMode::Constant, BorderMode::Replicate, BorderMode::Reflect,
                                BorderMode::Reflect101, BorderMode::Wrap};
    const char* names[] = {"Constant", "Replicate", "Reflect", "Reflect101", "Wrap"};
    const ImageU8 rgb = seeded<std::uint8_t>(1920, 1080, 3, 1);
    const ImageU8 gray = seeded<std::uint8_t>(997, 601, 1, 2);
    const ImageF grayf = seeded<float>(640, 480, 1, 3);
    char buf[160];
    // gaussianBlur sigma 2 on 1080p RGB (the reference's published benchmark shape)
    compare("gaussianBlur sigma=2 1920x1080x3 u8 Reflect101", cuda::gaussianBlur(rgb, 2.0), gaussianBlur(rgb, 2.0), 1, 0);
    for (int m = 0; m < 5; ++m) {
        std::snprintf(buf, sizeof buf, "gaussianBlur sigma=(2.3,0.8) gray u8 %s", names[m]);
        compare(buf, cuda::gaussianBlur(gray, 2.3, 0.8, 0, modes[m]), gaussianBlur(gray, 2.3, 0.8, 0, modes[m]), 1, 0);
        std::snprintf(buf, sizeof buf, "gaussianBlur<float> sigma=1.5 f32 %s", names[m]);
        compare(buf, cuda::gaussianBlur<float>(grayf, 1.5, 0.0, 0, modes[m]),
                gaussianBlur<float>(grayf, 1.5, 0.0, 0, modes[m]), 0, 1e-5);
        std::snprintf(buf, sizeof buf, "boxFilter 5x3 borderValue=3 u8 %s", names[m]);
        compare(buf, cuda::boxFilter(gray, 5, 3, true, modes[m], 3.0), boxFilter(gray, 5, 3, true, modes[m], 3.0), 0, 0);
        std::snprintf(buf, sizeof buf, "sobel dx=1 ksize=3 -> float %s", names[m]);
        compare(buf, cuda::sobel(gray, 1, 0, 3, 1.0, modes[m]), sobel(gray, 1, 0, 3, 1.0, modes[m]), 0, 0);
        const auto kx = ipf::detail::derivKernel(0, 5), ky = ipf::detail::derivKernel(1, 5);
        std::snprintf(buf, sizeof buf, "sepFilter2D<int16_t> Sobel dy ksize=5 %s", names[m]);
        compare(buf, cuda::sepFilter2D<std::int16_t>(gray, kx, ky, modes[m]),
                sepFilter2D<std::int16_t>(gray, kx, ky, modes[m]), 0, 0);
        Kernel k(5, 3, 1);
        std::mt19937 rng(7 + m);
        for (float& v : k) v = static_cast<float>(std::normal_distribution<double>(0.0, 1.0)(rng));
        std::snprintf(buf, sizeof buf, "filter2D 5x3 delta=0.5 borderValue=7 u8 %s", names[m]);
        compare(buf, cuda::filter2D(gray, k, modes[m], 0.5, Point(-1, -1), 7.0),
                filter2D(gray, k, modes[m], 0.5, Point(-1, -1), 7.0), 1, 0);
        if (m != 0)
            for (int ks : {3, 5, 7}) {
                std::snprintf(buf, sizeof buf, "medianBlur %d u8 %s", ks, names[m]);
                compare(buf, cuda::medianBlur(gray, ks, modes[m]), medianBlur(gray, ks, modes[m]), 0, 0);
            }
    }
    for (MorphShape sh : {MorphShape::Rect, MorphShape::Cross, MorphShape::Ellipse}) {
        const auto se = getStructuringElement(sh, 5, 7);
        std::snprintf(buf, sizeof buf, "erode 5x7 shape %d x2 RGB", static_cast<int>(sh));
        compare(buf, cuda::erode(rgb, se, 2), erode(rgb, se, 2), 0, 0);
        std::snprintf(buf, sizeof buf, "dilate 5x7 shape %d RGB", static_cast<int>(sh));
        compare(buf, cuda::dilate(rgb, se), dilate(rgb, se), 0, 0);
    }
    compare("erode default 3x3 rect gray", cuda::erode(gray), erode(gray), 0, 0);
    // int32 / double images and TOut = double: FP64 in the reference's order, exact
    const ImageD grayd = seeded<double>(331, 217, 1, 11);
    const ImageI32 grayi = seeded<std::int32_t>(331, 217, 3, 12);
    compare("gaussianBlur ImageD sigma 1.5", cuda::gaussianBlur(grayd, 1.5), gaussianBlur(grayd, 1.5), 0, 0);
    compare("gaussianBlur<double> of uint8 RGB", cuda::gaussianBlur<double>(rgb, 2.0), gaussianBlur<double>(rgb, 2.0),
            0, 0);
    compare("filter2D ImageI32", cuda::filter2D(grayi, makeKernel(3, 3, {1, -2, 1, 2, 0, -2, 1, 2, 1})),
            filter2D(grayi, makeKernel(3, 3, {1, -2, 1, 2, 0, -2, 1, 2, 1})), 0, 0);
    compare("medianBlur 5 ImageD", cuda::medianBlur(grayd, 5), medianBlur(grayd, 5), 0, 0);
    // the reference's other filters and its callers of the filters
    compare("morphologyEx Gradient 5x5 ellipse RGB",
            cuda::morphologyEx(rgb, MorphOp::Gradient, getStructuringElement(MorphShape::Ellipse, 5)),
            morphologyEx(rgb, MorphOp::Gradient, getStructuringElement(MorphShape::Ellipse, 5)), 0, 0);
    compare("morphologyEx TopHat 15x15 rect gray",
            cuda::morphologyEx(gray, MorphOp::TopHat, getStructuringElement(MorphShape::Rect, 15)),
            morphologyEx(gray, MorphOp::TopHat, getStructuringElement(MorphShape::Rect, 15)), 0, 0);
    compare("bilateralFilter d 9 RGB", cuda::bilateralFilter(rgb, 9, 50.0, 3.0), bilateralFilter(rgb, 9, 50.0, 3.0), 0,
            0);
    compare("integralImage RGB", cuda::integralImage(rgb), integralImage(rgb), 0, 0);
    compare("adaptiveThreshold Gaussian 11", cuda::adaptiveThreshold(gray, 255.0, AdaptiveMethod::Gaussian,
                                                                   ThresholdType::Binary, 11, 2.0),
            adaptiveThreshold(gray, 255.0, AdaptiveMethod::Gaussian, ThresholdType::Binary, 11, 2.0), 0, 0);
    compare("pyrDown RGB", cuda::pyrDown(rgb), pyrDown(rgb), 0, 0);
    compare("pyrUp gray", cuda::pyrUp(gray), pyrUp(gray), 0, 0);
    compare("canny RGB 50 150", cuda::canny(rgb, 50.0, 150.0), canny(rgb, 50.0, 150.0), 0, 0);
    compare("cornerHarris gray", cuda::cornerHarris(gray), cornerHarris(gray), 0, 1e-5);
    compare("scharr dx RGB", cuda::scharr(rgb, 1, 0), scharr(rgb, 1, 0), 0, 0);
    compare("prewitt dy gray", cuda::prewitt(gray, 0, 1), prewitt(gray, 0, 1), 0, 0);
    compare("sharpen 0.7 RGB", cuda::sharpen(rgb, 0.7), sharpen(rgb, 0.7), 1, 0);
    compare("emboss gray", cuda::emboss(gray), emboss(gray), 0, 0);
    compare("laplacian ksize 1 RGB", cuda::laplacian(rgb), laplacian(rgb), 0, 1e-5);
    compare("laplacian ksize 3 gray", cuda::laplacian(gray, 3), laplacian(gray, 3), 0, 0);
    compare("gradientMagnitude RGB", cuda::gradientMagnitude(rgb), gradientMagnitude(rgb), 0, 0);
    compare("unsharpMask RGB sigma 1.5 amount 0.8 threshold 3", cuda::unsharpMask(rgb, 1.5, 0.8, 3.0),
            unsharpMask(rgb, 1.5, 0.8, 3.0), 0, 0);
    {
        ImageF mg, mr;
        const ImageU8 other = seeded<std::uint8_t>(1920, 1080, 3, 2);
        const double g = cuda::ssim(rgb, other, &mg), r = ssim(rgb, other, &mr);
        compare("ssim map RGB", mg, mr, 0, 0);
        const bool ok = std::fabs(g - r) <= 1e-12 * std::fmax(1.0, std::fabs(r));
        std::printf("%s %-52s %.17g vs %.17g\n", ok ? "ok  " : "FAIL", "ssim mean RGB", g, r);
        g_fail += !ok;
    }
    expect_error("medianBlur even ksize throws", "ipf: medianBlur: ksize must be odd and positive",
                 [&] { (void)cuda::medianBlur(gray, 4); });
    expect_error("medianBlur Constant throws", "ipf: medianBlur: Constant border is not supported",
                 [&] { (void)cuda::medianBlur(gray, 3, BorderMode::Constant); });
    expect_error("boxFilter zero size throws", "ipf: boxFilter: kernel size must be positive",
                 [&] { (void)cuda::boxFilter(gray, 0, 3); });
    expect_error("sepFilter2D empty kernel throws", "ipf: separable filter: empty kernel",
                 [&] { (void)cuda::sepFilter2D(gray, {}, {1.0}); });
    std::printf(g_fail ? "dropin: %d FAILED\n" : "dropin: all ok\n", g_fail);
    return g_fail ? 1 : 0;
}
