// api_internal.h -- helpers of the C ABI layer (api.cu) shared with the
// composite entry points (compose.cu): error reporting, argument checks,
// staging of host images, separable filters with a chosen accumulator.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/ipfc.h"

namespace ipfc {

int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* fn);
size_t elem_bytes(int dt);
long long row_bytes(const ipfc_image* im);
long long pitch_of(const ipfc_image* im);
long long round_up(long long v, long long m);
cudaError_t prepare_device();
unsigned* device_error_word();
int take_device_error(cudaStream_t s, const char* fn);

// Checks a source/destination pair: IPFC_OK, an error, or -1 for an empty
// image (nothing to do).
int check_pair(const ipfc_image* src, const ipfc_image* dst, const char* fn, bool same_type);
// Per thread: calls from this thread run on kernels that leave SMs to other
// streams (the request server sets it around its requests).
void set_shared_gpu(bool on);
int check_pair_resized(const ipfc_image* src, const ipfc_image* dst, const char* fn, bool same_type);

// A device view of an image: the caller's memory, or a staged copy.
struct DevView {
    void* ptr = nullptr;
    long long pitch = 0;
    bool owned = false;
};
int view_in(const ipfc_image* im, cudaStream_t s, DevView* v, const char* fn);
int view_out(const ipfc_image* im, cudaStream_t s, DevView* v, const char* fn);
// Copies a staged result back, releases staging memory and waits for the
// stream when a side lives in host memory.
int finish(const ipfc_image* dst, DevView* in, DevView* out, cudaStream_t s, const char* fn);

int gaussian_taps(double sigma, int ksize, std::vector<double>& k);
int deriv_taps(int order, int ksize, std::vector<double>& k);

// The separable path of sepFilter2D / gaussianBlur / sobel; force_fp64 makes
// it accumulate in FP64 in the reference's operation order (bit-identical to
// ipf) whatever the element types.
int run_sep(const ipfc_image* src, ipfc_image* dst, const double* kx, int kw, const double* ky, int kh, int ax, int ay,
            int border, double delta, double bv, cudaStream_t s, const char* fn, bool force_fp64);

// boxFilter; force_fp64 sums every source type in FP64.
int run_box(const ipfc_image* src, ipfc_image* dst, int kw, int kh, int normalize, int border, double border_value,
            cudaStream_t s, bool force_fp64);

// An ipfc_image describing device memory.
inline ipfc_image dev_image(void* p, int w, int h, int c, int dt, long long pitch) {
    ipfc_image im;
    im.data = p;
    im.width = w;
    im.height = h;
    im.channels = c;
    im.dtype = dt;
    im.pitch = pitch;
    im.mem = IPFC_MEM_DEVICE;
    return im;
}

}  // namespace ipfc
