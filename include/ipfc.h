/*
 * ipfc.h -- C ABI of the B200 (sm_100a) neighbourhood-filter library.
 *
 * Drop-in boundary for the hot path of ImageProcessingFlex (ipf): separable
 * correlation (sepFilter2D / gaussianBlur / boxFilter / sobel), dense
 * filter2D, medianBlur and erode / dilate, with ipf's five BorderModes and
 * its saturate_cast rounding.  ipf itself is header-only C++ whose "operator
 * API" is the set of free template functions in namespace ipf; each entry
 * point below replaces one of them and cites it as
 * include/ipf/<file>.hpp:<line>.  The C++ wrapper include/ipf_cuda.hpp gives
 * the same functions back as ipf::cuda::* over ipf::Image<T>.
 *
 * Conventions
 *  - Images are interleaved row-major (pixel (x, y) channel c at
 *    row(y)[x*channels + c]), like ipf::Image<T> (core.hpp:220-222).  `pitch`
 *    is bytes between rows; 0 means dense rows.
 *  - `mem` says where `data` lives.  IPFC_MEM_DEVICE: device pointer on the
 *    current device; the call is asynchronous on `stream` (a cudaStream_t,
 *    NULL = legacy default stream).  IPFC_MEM_HOST: host memory (pinned or
 *    pageable); the call stages through device memory owned by the library
 *    and returns after the result is back in host memory.
 *  - dst must already have src's width, height and channel count (the
 *    reference allocates it; here the caller does).  Its dtype selects the
 *    output type, the TOut template argument of the reference.
 *  - Every function returns an ipfc_status.  On failure ipfc_last_error()
 *    returns a thread-local message; argument errors carry the reference's
 *    own "ipf: <function>: <reason>" text (core.hpp:41-44).
 *  - Nothing here falls back to the CPU.  With no usable CUDA device the
 *    compute entry points fail with IPFC_ERR_CUDA.
 */
#ifndef IPFC_H
#define IPFC_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define IPFC_API __attribute__((visibility("default")))
#else
#define IPFC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Element types: the reference's ImageU8 / U16 / I16 / I32 / F / D
 * (core.hpp:403-408). */
typedef enum ipfc_dtype {
    IPFC_U8 = 0,
    IPFC_U16 = 1,
    IPFC_I16 = 2,
    IPFC_I32 = 3,
    IPFC_F32 = 4,
    IPFC_F64 = 5
} ipfc_dtype;

/* Border modes, in the order of ipf::BorderMode (core.hpp:183). */
typedef enum ipfc_border {
    IPFC_BORDER_CONSTANT = 0,
    IPFC_BORDER_REPLICATE = 1,
    IPFC_BORDER_REFLECT = 2,
    IPFC_BORDER_REFLECT101 = 3,
    IPFC_BORDER_WRAP = 4
} ipfc_border;

/* Structuring-element shapes, in the order of ipf::MorphShape
 * (morphology.hpp:21). */
typedef enum ipfc_morph_shape { IPFC_MORPH_RECT = 0, IPFC_MORPH_CROSS = 1, IPFC_MORPH_ELLIPSE = 2 } ipfc_morph_shape;

typedef enum ipfc_mem { IPFC_MEM_HOST = 0, IPFC_MEM_DEVICE = 1 } ipfc_mem;

typedef enum ipfc_status {
    IPFC_OK = 0,
    IPFC_ERR_INVALID = 1,     /* invalid argument: the reference throws ipf::Error here */
    IPFC_ERR_NOMEM = 2,       /* device or pinned allocation failed */
    IPFC_ERR_CUDA = 3,        /* CUDA runtime error (no device, launch failure, ...) */
    IPFC_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    IPFC_ERR_UNSUPPORTED = 5  /* valid for the reference, not provided by this build (dtype) */
} ipfc_status;

/* An image view.  Plain data: the library never takes ownership. */
typedef struct ipfc_image {
    void* data;
    int width;
    int height;
    int channels;
    int dtype;       /* ipfc_dtype */
    long long pitch; /* bytes between row starts; 0 = width * channels * sizeof(element) */
    int mem;         /* ipfc_mem */
} ipfc_image;

/* ---- library ------------------------------------------------------------- */

/* Thread-local text of the last failure on this thread ("" when none).
 * Replaces the message of ipf::Error (include/ipf/core.hpp:35-41): argument
 * errors carry the same "ipf: <function>: <reason>" text. */
IPFC_API const char* ipfc_last_error(void);

/* (major << 16) | (minor << 8) | patch of this library (its own numbering,
 * not IPF_VERSION_* of include/ipf/core.hpp:24-26). */
IPFC_API int ipfc_version(void);

/* Waits for `stream`, then reports whether any kernel since the last check
 * gave up a bounded device-side wait (IPFC_ERR_TIMEOUT; the word is then
 * cleared).  Calls with host images check this themselves.  No counterpart
 * in the reference, whose CPU code has no device waits. */
IPFC_API int ipfc_check_device(void* stream);

/* ---- tap and element generators (host, FP64) ----------------------------- */

/* gaussianKernel1D (filter.hpp:129-145).  Writes min(len, cap) taps to out and
 * returns the kernel length, or -1 with ipfc_last_error() set. */
IPFC_API int ipfc_gaussian_kernel_1d(double sigma, int ksize, double* out, int cap);

/* detail::derivKernel (filter.hpp:93-114).  Returns the length or -1. */
IPFC_API int ipfc_deriv_kernel(int order, int ksize, double* out, int cap);

/* getStructuringElement (morphology.hpp:24-49).  out holds width*height
 * bytes (height <= 0 means height = width). */
IPFC_API int ipfc_structuring_element(int shape, int width, int height, uint8_t* out);

/* ---- separable correlation --------------------------------------------- */

/* detail::sepFilterImpl (filter.hpp:37-90), reached from sepFilter2D
 * (filter.hpp:197-203) with anchors kw/2, kh/2.  ax/ay < 0 select those
 * defaults.  Accumulates in FP32 on the device (FP64 on the reference). */
IPFC_API int ipfc_sep_filter2d(const ipfc_image* src, ipfc_image* dst, const double* kx, int kw, const double* ky, int kh,
                      int ax, int ay, int border, double delta, double border_value, void* stream);

/* gaussianBlur (filter.hpp:262-267): FP64 taps from gaussianKernel1D on the
 * host, then the separable path. */
IPFC_API int ipfc_gaussian_blur(const ipfc_image* src, ipfc_image* dst, double sigma_x, double sigma_y, int ksize, int border,
                       void* stream);

/* boxFilter (filter.hpp:206-253) and blur (filter.hpp:256-259, normalize = 1,
 * kw = kh = ksize).  Integer sources are summed exactly. */
IPFC_API int ipfc_box_filter(const ipfc_image* src, ipfc_image* dst, int kw, int kh, int normalize, int border,
                    double border_value, void* stream);

/* sobel (filter.hpp:395-407).  The reference returns ImageF; any dst dtype is
 * accepted here (IPFC_I16 gives sepFilter2D<int16_t> with the same taps). */
IPFC_API int ipfc_sobel(const ipfc_image* src, ipfc_image* dst, int dx, int dy, int ksize, double scale, int border,
               void* stream);

/* ---- dense correlation -------------------------------------------------- */

/* filter2D (filter.hpp:159-194).  kernel: kw*kh float32 taps, row-major (the
 * reference's Kernel = ImageF).  ax/ay < 0 select kw/2, kh/2.  FP32 CUDA-core
 * accumulation. */
IPFC_API int ipfc_filter2d(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax, int ay,
                  int border, double delta, double border_value, void* stream);

/* The two forms of filter2D behind ipfc_filter2d, for callers that choose:
 *  ipfc_filter2d_fp32  -- CUDA cores, FP32 accumulation, every channel count
 *                         and element type;
 *  ipfc_filter2d_split -- tcgen05 tensor cores: uint8 pixels exact in FP16 or
 *                         float pixels split into FP16 hi + lo (with a per-tile
 *                         power-of-two scale), taps split into FP16 hi + lo,
 *                         FP32 accumulation.  Single-channel images, uint8 to
 *                         uint8 / uint16 / int16 / float or float to float,
 *                         kernels up to 32 x 33; otherwise
 *                         IPFC_ERR_UNSUPPORTED.  Non-finite float pixels give
 *                         NaN where the reference's skipped zero taps would not.
 * Same arguments and checks as ipfc_filter2d (filter.hpp:159-194). */
IPFC_API int ipfc_filter2d_fp32(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax,
                                int ay, int border, double delta, double border_value, void* stream);
IPFC_API int ipfc_filter2d_split(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax,
                                 int ay, int border, double delta, double border_value, void* stream);

/* filter2D for callers that cannot allocate device memory (inside a custom
 * allocator, under a framework that reserved the device's memory, in a
 * pipeline that forbids allocation after start-up).  It always runs the FP32
 * CUDA-core form, the same kernel and result as ipfc_filter2d_fp32 (not
 * necessarily ipfc_filter2d's, which may pick the tensor-core form), on
 * device images only.  The non-zero taps are staged in a fixed 64 KB device
 * array that the library holds on every GPU it runs on, so at most 4096
 * non-zero taps (larger kernels are rejected with IPFC_ERR_INVALID).  The
 * first call on a device looks up that array's address.  A call on a
 * capturing stream is rejected with IPFC_ERR_UNSUPPORTED: the taps are
 * copied from a per-thread host buffer.  Calls share the array: any two calls
 * whose streams the caller has not ordered (same stream, an event or a
 * synchronisation) race on it.  No counterpart in the reference, whose CPU
 * code allocates freely. */
IPFC_API int ipfc_filter2d_noalloc(const ipfc_image* src, ipfc_image* dst, const float* kernel, int kw, int kh, int ax,
                                   int ay, int border, double delta, double border_value, void* stream);

/* Bound of every device-side wait of the tensor-core kernels (a stage of a
 * pipeline that never completes), in nanoseconds; 0 restores the default
 * (250 ms).  A wait that runs out makes the call report IPFC_ERR_TIMEOUT
 * (ipfc_check_device for device images) and the kernel ends; the final wait
 * for issued MMAs before tensor memory is freed keeps its own bound.
 * Returns the previous bound.  No counterpart in the reference (it has no
 * device waits); tests use it to make a wait run out. */
IPFC_API unsigned long long ipfc_set_wait_limit_ns(unsigned long long ns);

/* ---- order statistics and morphology -------------------------------------- */

/* medianBlur (filter.hpp:302-332): exact; Constant border is an error. */
IPFC_API int ipfc_median_blur(const ipfc_image* src, ipfc_image* dst, int ksize, int border, void* stream);

/* erode / dilate (morphology.hpp:112-127 over detail::morphOnce, 53-107).
 * se: se_w*se_h mask bytes (non-zero = member), anchor (se_w/2, se_h/2).
 * Pixels outside the image never count; there is no border mode. */
IPFC_API int ipfc_erode(const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w, int se_h, int iterations,
               void* stream);
IPFC_API int ipfc_dilate(const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w, int se_h, int iterations,
                void* stream);

/* morphologyEx (morphology.hpp:140-158): op in ipf::MorphOp order; the
 * compound ops run the same erode / dilate kernels through device buffers,
 * and differences are saturate_cast<T>(double(a) - double(b)). */
enum {
    IPFC_MORPH_ERODE = 0,
    IPFC_MORPH_DILATE = 1,
    IPFC_MORPH_OPEN = 2,
    IPFC_MORPH_CLOSE = 3,
    IPFC_MORPH_GRADIENT = 4,
    IPFC_MORPH_TOPHAT = 5,
    IPFC_MORPH_BLACKHAT = 6
};
IPFC_API int ipfc_morphology_ex(const ipfc_image* src, ipfc_image* dst, int op, const uint8_t* se, int se_w, int se_h,
                                int iterations, void* stream);

/* ---- more filters and the reference's callers of the filters ---------------
 *
 * Each is computed on the GPU with the kernels above; where the reference
 * accumulates in FP64 these do too, in its operation order, so results are
 * bit-identical to ipf's unless noted. */

/* bilateralFilter (filter.hpp:337-387): circular window of radius d/2 (or
 * lround(1.5 sigma_space) for d <= 0, at most 64), L1 colour distance,
 * Constant-border positions skipped.  Integer images use the reference's
 * range-weight table (bit-identical); float images evaluate exp per tap on
 * the GPU (within a few units in the last place of FP64).  1 to 4 channels. */
IPFC_API int ipfc_bilateral_filter(const ipfc_image* src, ipfc_image* dst, int d, double sigma_color,
                                   double sigma_space, int border, void* stream);

/* integralImage (filter.hpp:527-541): dst is IPFC_F64 with (W+1) x (H+1)
 * pixels and the source's channels; squared != 0 sums squares. */
IPFC_API int ipfc_integral_image(const ipfc_image* src, ipfc_image* dst, int squared, void* stream);

/* adaptiveThreshold (filter.hpp:554-567): single channel; method and type in
 * ipf's AdaptiveMethod / ThresholdType order (Binary and BinaryInv only). */
enum { IPFC_ADAPTIVE_MEAN = 0, IPFC_ADAPTIVE_GAUSSIAN = 1 };
enum { IPFC_THRESH_BINARY = 0, IPFC_THRESH_BINARY_INV = 1 };
IPFC_API int ipfc_adaptive_threshold(const ipfc_image* src, ipfc_image* dst, double maxval, int method, int type,
                                     int block_size, double c, void* stream);

/* pyrDown / pyrUp (geometry.hpp:504-525): dst is ((W+1)/2) x ((H+1)/2),
 * respectively 2W x 2H, same type and channels. */
IPFC_API int ipfc_pyr_down(const ipfc_image* src, ipfc_image* dst, void* stream);
IPFC_API int ipfc_pyr_up(const ipfc_image* src, ipfc_image* dst, void* stream);

/* ssim (metrics.hpp:51-78): mean SSIM of a and b (same shape and type) over
 * the valid region into *result; ssim_map (nullable) receives the per-pixel
 * map, IPFC_F32 with a's shape.  The map is bit-identical to the reference's;
 * the mean is a parallel FP64 sum (within 1e-12 relative of its sequential
 * one). */
IPFC_API int ipfc_ssim(const ipfc_image* a, const ipfc_image* b, double* result, ipfc_image* ssim_map, void* stream);

/* cornerHarris / cornerMinEigenVal (features.hpp:111-142): single-channel
 * source, dst IPFC_F32.  The Sobel terms are bit-identical; the unnormalised
 * box sums are FP64 window sums where the reference keeps FP64 running sums,
 * so results agree to about one unit in the last place of FP32. */
IPFC_API int ipfc_corner_harris(const ipfc_image* src, ipfc_image* dst, int block_size, int ksize, double k,
                                void* stream);
IPFC_API int ipfc_corner_min_eigen_val(const ipfc_image* src, ipfc_image* dst, int block_size, int ksize,
                                       void* stream);

/* canny (features.hpp:27-88): dst is IPFC_U8, single channel, 0 / 255.  Sobel
 * gradients with Replicate, per-pixel strongest channel, non-maximum
 * suppression and hysteresis (propagated on the GPU until no edge changes;
 * the result does not depend on the visiting order). */
IPFC_API int ipfc_canny(const ipfc_image* src, ipfc_image* dst, double low_threshold, double high_threshold, int ksize,
                        int l2_gradient, void* stream);

/* laplacian (filter.hpp:426-438): dst IPFC_F32.  ksize 1 is filter2D with
 * the 3x3 kernel {0,1,0, 1,-4,1, 0,1,0} times scale; a larger ksize sums the
 * second-order Sobel derivatives sobel(2,0) + sobel(0,2). */
IPFC_API int ipfc_laplacian(const ipfc_image* src, ipfc_image* dst, int ksize, double scale, int border, void* stream);

/* gradientMagnitude (filter.hpp:462-467): dst IPFC_F32, hypot of sobel(1,0)
 * and sobel(0,1) (Reflect101), rounded as the C library's hypotf. */
IPFC_API int ipfc_gradient_magnitude(const ipfc_image* src, ipfc_image* dst, int ksize, void* stream);

/* unsharpMask (filter.hpp:473-483): dst of the source's type;
 * out = saturate_cast(|v - b| > threshold ? v + amount (v - b) : v) with
 * b = gaussianBlur<double>(src, sigma), all in FP64 as the reference. */
IPFC_API int ipfc_unsharp_mask(const ipfc_image* src, ipfc_image* dst, double sigma, double amount, double threshold,
                               void* stream);

/* ---- batches: many images, a few launches --------------------------------
 *
 * No counterpart in the reference (ipf runs one call per image).  A batch
 * collects per-image calls -- the same functions and arguments as the
 * entry points above, on device images -- and runs them together: every
 * image is cut into the per-image kernels' tiles.  Separable items with the
 * same taps and channels share one launch (up to 40 items, their arguments
 * in the kernel parameters); median and morphology tiles are walked by
 * persistent kernels, one tile queue per register class, over all images.
 * The launches are spread over parallel graph branches.  The first
 * ipfc_batch_run plans the batch (autotuned tile shapes, tile order, device
 * tables) and captures it as a CUDA graph; later runs replay the graph on
 * `stream`.  Each image's result is bit-identical to its per-image call.
 *
 * Covered: uint8 images with 1, 3 or 4 channels; separable filters and
 * gaussianBlur with equal odd tap counts 3..25 and centred anchors;
 * medianBlur with ksize 3..15; erode / dilate with an all-ones element up
 * to 31x31 and one iteration.  Other calls return IPFC_ERR_UNSUPPORTED.
 * The images must stay allocated, at the same addresses, while the batch
 * exists; a batch is re-run on new pixels by writing them into the same
 * buffers.  A batch belongs to the device current when its first image was
 * added and is not safe for concurrent use from several threads. */
typedef struct ipfc_batch ipfc_batch;

enum {
    IPFC_BATCH_AUTOTUNE = 1, /* 1 (default): tune unseen tile keys at planning; 0: built-in shapes */
    IPFC_BATCH_GRAPH = 2     /* 1 (default): capture and replay a CUDA graph; 0: launch directly */
};

enum {
    IPFC_BATCH_INFO_ITEMS = 0,
    IPFC_BATCH_INFO_PLANNED = 1,
    IPFC_BATCH_INFO_TILES_LIGHT = 2,
    IPFC_BATCH_INFO_TILES_HEAVY = 3,
    IPFC_BATCH_INFO_GRID_LIGHT = 4,
    IPFC_BATCH_INFO_GRID_HEAVY = 5,
    IPFC_BATCH_INFO_KERNELS = 6, /* kernel launches per run: queue kernels and separable group launches */
    IPFC_BATCH_INFO_GRAPH = 7,
    IPFC_BATCH_INFO_TILES_MEM = 8, /* 3x3 / 5x5 median and morphology tiles */
    IPFC_BATCH_INFO_GRID_MEM = 9
};

/* Tile keys of the autotuner: op 0 separable (k = taps), 1 median (k =
 * ksize), 2 morphology (k = element width); size class 0..3 by pixel count
 * (< 64Ki, < 512Ki, < 2Mi, larger).  Values: separable a = rows per tile;
 * median / morphology a = tile width in samples, b = tile height in rows. */
IPFC_API int ipfc_batch_create(ipfc_batch** out);
IPFC_API int ipfc_batch_destroy(ipfc_batch* b);
IPFC_API int ipfc_batch_set_option(ipfc_batch* b, int option, int value);
IPFC_API int ipfc_batch_add_sep_filter(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const double* kx, int kw,
                                       const double* ky, int kh, int border, double delta, double border_value);
IPFC_API int ipfc_batch_add_gaussian_blur(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, double sigma_x,
                                          double sigma_y, int ksize, int border);
IPFC_API int ipfc_batch_add_median_blur(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, int ksize, int border);
IPFC_API int ipfc_batch_add_erode(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w,
                                  int se_h, int iterations);
IPFC_API int ipfc_batch_add_dilate(ipfc_batch* b, const ipfc_image* src, ipfc_image* dst, const uint8_t* se, int se_w,
                                   int se_h, int iterations);
IPFC_API int ipfc_batch_run(ipfc_batch* b, void* stream);
IPFC_API int ipfc_batch_info(const ipfc_batch* b, int what, long long* value);
IPFC_API int ipfc_tune_get(int op, int k, int channels, int size_class, int* a, int* b);
IPFC_API int ipfc_tune_set(int op, int k, int channels, int size_class, int a, int b);
/* Text table, one "device op k channels size_class a b" line per entry;
 * ipfc_tune_load adds the entries it reads and stores their count. */
IPFC_API int ipfc_tune_save(const char* path);
IPFC_API int ipfc_tune_load(const char* path, int* count);
IPFC_API int ipfc_tune_clear(void);

/* ---- request server: continuous batching ----------------------------------
 *
 * No counterpart in the reference (ipf is a library of synchronous calls).
 * A server takes filter requests -- one image and one op each, with host
 * (preferably pinned) or device images -- and runs them on the current
 * device from a scheduler thread: requests are admitted in arrival order as
 * in-flight slots and device memory (a budget, from a pool the server keeps)
 * free up, spread over several streams so that their copies and kernels
 * overlap, and requests the batch kernels cover are merged into one
 * persistent launch.  Each result equals the per-image call's result.
 * Completions report the arrival, admission and completion times (seconds
 * on the server's clock, ipfc_server_now). */
typedef struct ipfc_server ipfc_server;

enum {
    IPFC_OP_GAUSSIAN = 0, /* gaussianBlur: sigma_x, sigma_y, ksize, border */
    IPFC_OP_SOBEL = 1,    /* sobel: dx, dy, ksize, scale, border (dst float or int16) */
    IPFC_OP_MEDIAN = 2,   /* medianBlur: ksize, border */
    IPFC_OP_FILTER2D = 3, /* filter2D: kernel kw x kh (copied at submit), border, delta, border_value */
    IPFC_OP_BOX = 4,      /* blur: ksize x ksize normalised, border */
    IPFC_OP_ERODE = 5,    /* erode by a ksize x ksize rect */
    IPFC_OP_DILATE = 6    /* dilate by a ksize x ksize rect */
};

typedef struct ipfc_request {
    int op;
    ipfc_image src;
    ipfc_image dst;
    double sigma_x, sigma_y;
    int ksize;
    int dx, dy;
    double scale;
    const float* kernel;
    int kw, kh;
    int border;
    double delta, border_value;
    double arrival; /* server-clock seconds; < 0: the time of submission */
} ipfc_request;

typedef struct ipfc_completion {
    unsigned long long ticket;
    int status; /* ipfc_status of the request */
    double arrival, admitted, done;
} ipfc_completion;

typedef struct ipfc_server_config {
    size_t device_budget_bytes; /* device bytes of requests in flight (default 40 GiB) */
    int max_inflight;           /* requests in flight at once (default 64) */
    int streams;                /* streams the work is spread over (default 4) */
    int batch;                  /* 1 (default): merge batchable requests admitted together */
} ipfc_server_config;

enum {
    IPFC_SERVER_STAT_GROUPS = 0,
    IPFC_SERVER_STAT_BATCHED = 1,
    IPFC_SERVER_STAT_BATCH_LAUNCHES = 2,
    IPFC_SERVER_STAT_MAX_INFLIGHT = 3,
    IPFC_SERVER_STAT_MAX_BYTES = 4,
    IPFC_SERVER_STAT_FAILED = 5
};

IPFC_API int ipfc_server_create(ipfc_server** out, const ipfc_server_config* cfg); /* cfg NULL: defaults */
IPFC_API int ipfc_server_destroy(ipfc_server* s); /* finishes queued and in-flight requests first */
IPFC_API double ipfc_server_now(const ipfc_server* s);
IPFC_API int ipfc_server_submit(ipfc_server* s, const ipfc_request* r, unsigned long long* ticket);
IPFC_API int ipfc_server_poll(ipfc_server* s, ipfc_completion* out, int max, int* n, int wait_ms);
IPFC_API int ipfc_server_drain(ipfc_server* s, int timeout_ms); /* < 0: no limit */
IPFC_API int ipfc_server_stats(const ipfc_server* s, int what, double* value);

/* Failure injection on the host, for tests of the failure path: from now on
 * the nth device-buffer allocation the server makes for a request (counted
 * from the server's creation, 1-based; 0 disables) fails as if the
 * pool were exhausted.  That request completes with IPFC_ERR_NOMEM and runs
 * no kernel; every other request completes normally.  No counterpart in the
 * reference (it has no request server). */
IPFC_API int ipfc_server_fail_allocation(ipfc_server* s, long long nth);

/* ---- device probes of the scalar rules --------------------------------- */

/* borderIndex (core.hpp:187-214) evaluated by the device code the kernels
 * use: out[i] = border index of p[i] for a row of length len.  p and out are
 * device pointers of n ints. */
IPFC_API int ipfc_probe_border_index(const int* p, int* out, int n, int len, int border, void* stream);

/* saturate_cast<To>(float) (core.hpp:69-103) evaluated by the device store
 * path: v is n device floats, out n elements of dtype `to`. */
IPFC_API int ipfc_probe_saturate(const float* v, void* out, int n, int to, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IPFC_H */
