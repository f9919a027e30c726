"""B200-native (sm_100a) neighbourhood-filter path of ImageProcessingFlex.

``from imageprocessingflex_b200 import gaussianBlur, BorderMode`` mirrors the
reference's ``ipf::gaussianBlur`` etc. on numpy arrays (host) and CUDA torch
tensors (device).  The C++ form is ``include/ipf_cuda.hpp``; the C ABI is
``include/ipfc.h``; the kernels live in ``csrc/``.
"""
from .filters import (  # noqa: F401
    AdaptiveMethod,
    BorderMode,
    Error,
    MorphOp,
    MorphShape,
    ThresholdType,
    adaptiveThreshold,
    bilateralFilter,
    blur,
    boxFilter,
    canny,
    cornerHarris,
    cornerMinEigenVal,
    derivKernel,
    dilate,
    emboss,
    erode,
    filter2D,
    gaussianBlur,
    gaussianKernel1D,
    getStructuringElement,
    gradientMagnitude,
    integralImage,
    laplacian,
    medianBlur,
    morphologyEx,
    prewitt,
    pyrDown,
    pyrUp,
    scharr,
    sepFilter2D,
    sharpen,
    sobel,
    ssim,
    unsharpMask,
)

__version__ = "1.0.0"
