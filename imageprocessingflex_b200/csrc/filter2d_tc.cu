// filter2d_tc.cu -- filter2D on the 5th-generation tensor cores (tcgen05):
// split-precision FP16 operands, FP32 accumulation in tensor memory.
//
// Geometry and the GEMM form are in filter2d_tc.cuh.  One persistent CTA per
// SM walks the 128 x 64 output tiles with 8 worker warps and one MMA warp:
//  1. once per CTA: B (taps hi and lo side by side, banded, in the shared
//     layout) is copied from global memory, 256 tensor-memory columns are
//     allocated (two accumulator sets) and the barriers initialised;
//  2. per tile, the workers stage the transposed source tile into one of two
//     A buffers, one tile ahead (loads issued before the previous tile's
//     read-out): 8 source rows x 4 pixels per work item, borders resolved at
//     load, pixels centred and converted to FP16 (uint8: exact, by byte
//     permutes; float: hi and lo parts under a per-tile power of two),
//     stored as 16-byte rows of K-major core matrices;
//  3. one thread of the MMA warp issues the tile's MMAs -- 4 groups x kw tap
//     columns x Kt/16 K steps, each one N = 32 MMA (hi and lo taps) plus,
//     for float sources, one N = 16 MMA (lo pixels x hi taps) -- into one of
//     two accumulator sets and commits them to a barrier;
//  4. the workers read the previous tile's accumulators with tcgen05.ld
//     (warp w reads lanes 32 (w mod 4) .. +31, half the columns each), add
//     the correction set, scale, add the offset, saturate_cast and store
//     128-pixel row runs -- while the tensor cores work on the next tile.
// Every wait is bounded; a timeout records kErrTcWait in the device error
// word and ends the loops, and the CTA frees its tensor memory only after a
// last bounded wait for every MMA it issued.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ipfc.h"
#include "common.cuh"
#include "filter2d_tc.cuh"
#include "tc_common.cuh"

namespace ipfc {

int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* fn);
unsigned* device_error_word();
unsigned long long device_wait_limit_ns();
cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

constexpr unsigned kErrTcWait = 0x201u;   // a pipeline wait gave up
constexpr unsigned kErrTcDrain = 0x202u;  // the final MMA drain gave up: tensor memory left allocated

struct F2DTcArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H, border;
    int C, rowlen;  // channels; samples per row (W * C)
    float delta, bv;
    int kw, kh, ax, ay;
    float tap_unscale;  // 2^-s
    float tap_sum;      // sum of the taps (FP64 on the host, rounded once)
    int tiles_x, ntiles;
    int byte_border;    // uint8 source whose Constant border value (if any) is a byte: packed staging
    unsigned char bvb;  // that byte
    const uint4* btab;  // B in the shared layout
    unsigned* err;
    unsigned long long wait_ns;  // bound of a pipeline wait
};

namespace {

// Tensor memory: two accumulator sets (double buffer, 256 columns apart).
// Group g of a set owns columns 64 g .. 64 g + 63: tap columns i of even
// index accumulate at +0, odd ones at +32, each as the hi x hi products
// ("main", 16 columns) followed by the small hi x lo / lo x hi correction
// products (16 columns).  Splitting the sum four ways keeps every
// accumulator small (its rounding is relative to its magnitude); the four
// are added once, in FP32, when the results are read.
constexpr int kTmemCols = 512;
constexpr int kSetCols = 256;
constexpr int kCorrCol = 16;
constexpr int kOddCol = 32;

// Source samples of one work item: 8 rows x 4 pixels starting at image
// (gy0, gx0), borders resolved (-1: the Constant border value).
template <typename Tin>
__device__ __forceinline__ void load_item(const F2DTcArgs& a, int gy0, int gx0, float (&v)[8][4]) {
    const bool cols_in = gx0 >= 0 && gx0 + 4 <= a.rowlen;
    int cx[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) cx[c] = cols_in ? gx0 + c : border_sample(gx0 + c, a.W, a.C, a.border);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int sy = border_index(gy0 + j, a.H, a.border);
        if (sy < 0) {
#pragma unroll
            for (int c = 0; c < 4; ++c) v[j][c] = a.bv;
            continue;
        }
        const Tin* row = row_ptr<Tin>(a.src, a.spitch, sy);
        if constexpr (sizeof(Tin) == 1) {
            if (cols_in && (((uintptr_t)(row + gx0)) & 3) == 0) {
                const unsigned w = __ldg(reinterpret_cast<const unsigned*>(row + gx0));
#pragma unroll
                for (int c = 0; c < 4; ++c) v[j][c] = (float)((w >> (8 * c)) & 0xffu);
                continue;
            }
        } else {
            if (cols_in && (((uintptr_t)(row + gx0)) & 15) == 0) {
                const float4 q = __ldg(reinterpret_cast<const float4*>(row + gx0));
                v[j][0] = q.x;
                v[j][1] = q.y;
                v[j][2] = q.z;
                v[j][3] = q.w;
                continue;
            }
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) v[j][c] = cx[c] < 0 ? a.bv : (float)__ldg(row + cx[c]);
    }
}


// Per-tile scaling of the staged operands and of the results.
struct TileScale {
    float escale;   // applied to centred pixels before the FP16 split
    float centre;   // subtracted from pixels
    float unscale;  // 2^-(e+s): accumulator -> result
    float offset;   // centre * sum(taps) + delta
};

// staging items per worker: XR/4 x KR/8 items per tile, at most 42 x 12 for
// one channel and 64 x 12 for up to 4 channels (uint8 only)
__host__ __device__ constexpr int tc_items_per_thread(bool float_src) { return float_src ? 2 : 3; }

// uint8 source, prefetch form: 8 rows x 4 pixels at (gy0, gx0) as one word
// (4 bytes) per row, borders resolved, Constant as the border byte.
__device__ __forceinline__ void load_item_raw(const F2DTcArgs& a, int gy0, int gx0, unsigned (&w)[8]) {
    const bool cols_in = gx0 >= 0 && gx0 + 4 <= a.rowlen;
    int cx[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) cx[c] = cols_in ? gx0 + c : border_sample(gx0 + c, a.W, a.C, a.border);
    const unsigned cfill = 0x01010101u * a.bvb;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int sy = border_index(gy0 + j, a.H, a.border);
        if (sy < 0) {
            w[j] = cfill;
            continue;
        }
        const uint8_t* row = row_ptr<uint8_t>(a.src, a.spitch, sy);
        if (cols_in && (((uintptr_t)(row + gx0)) & 3) == 0) {
            w[j] = __ldg(reinterpret_cast<const unsigned*>(row + gx0));
            continue;
        }
        unsigned x = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) x |= (cx[c] < 0 ? (unsigned)a.bvb : (unsigned)__ldg(row + cx[c])) << (8 * c);
        w[j] = x;
    }
}

// Stores one prefetched uint8 item: pixel c's 8 rows as FP16 (b - 128),
// exact -- byte b -> f16 bits 0x6400 | b (= 1024 + b) by byte permutes, minus
// 1152 (0x6480).  Lanes store their four 16-byte rows in rotated order, so
// one store instruction's rows land 80 bytes apart, on distinct bank groups.
__device__ __forceinline__ void store_item_raw(unsigned char* A, const TcGeom& g, int q, int s, const unsigned (&w)[8],
                                               int rot) {
    const __half2 k1152 = __halves2half2(__ushort_as_half((unsigned short)0x6480), __ushort_as_half((unsigned short)0x6480));
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const unsigned c = (unsigned)((cc + rot) & 3);
        const unsigned sel = c | ((4u + c) << 4);
        unsigned h[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const unsigned t = __byte_perm(w[2 * p], w[2 * p + 1], sel);
            const unsigned u = __byte_perm(t, 0x64646464u, 0x4140u);
            const __half2 v = __hsub2(*reinterpret_cast<const __half2*>(&u), k1152);
            h[p] = h2_bits(v);
        }
        *reinterpret_cast<uint4*>(A + g.a_off(4 * q + (int)c, 8 * s)) = make_uint4(h[0], h[1], h[2], h[3]);
    }
}

// Per-tile centre and power of two of a float tile from each worker's local
// max / min (all worker threads): max |p - centre| * 2^e in [2^14, 2^15).
__device__ __forceinline__ TileScale tile_scale_from(const F2DTcArgs& a, float* red, float mx, float mn, int wtid) {
    const int warp = wtid >> 5, lane = wtid & 31;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if (lane == 0) {
        red[warp] = mx;
        red[8 + warp] = mn;
    }
    workers_sync<kTcWorkers>();
    if (wtid == 0) {
        float gmx = -3.4e38f, gmn = 3.4e38f;
        for (int w = 0; w < kTcWorkers / 32; ++w) {
            gmx = fmaxf(gmx, red[w]);
            gmn = fminf(gmn, red[8 + w]);
        }
        const float c = 0.5f * gmx + 0.5f * gmn;
        const float r = fmaxf(gmx - c, c - gmn);
        int ex = 0;
        if (r > 0.f && r <= 3.0e38f) {
            frexpf(r, &ex);  // r = f 2^ex, f in [0.5, 1)
            ex = 15 - ex;
            ex = ex < -120 ? -120 : (ex > 120 ? 120 : ex);
        }
        red[16] = (float)ex;
        red[17] = (c == c && fabsf(c) <= 3.0e38f) ? c : 0.f;
    }
    workers_sync<kTcWorkers>();
    const int ex = (int)red[16];
    TileScale ts;
    ts.centre = red[17];
    ts.escale = ldexpf(1.f, ex);
    ts.unscale = a.tap_unscale * ldexpf(1.f, -ex);
    ts.offset = fmaf(ts.centre, a.tap_sum, a.delta);
    return ts;
}

// Stores one prefetched float item as FP16 hi and lo parts of the centred,
// scaled pixels (rotated chunk order, as store_item_raw).
__device__ __forceinline__ void store_item_split(unsigned char* A0, unsigned char* A1, const TcGeom& g, int q, int s,
                                                 const float (&v)[8][4], const TileScale& ts, int rot) {
#pragma unroll
    for (int cc = 0; cc < 4; ++cc) {
        const int c = (cc + rot) & 3;
        unsigned hi[4], lo[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            float x0 = 0.f, x1 = 0.f;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k == c) {
                    x0 = (v[2 * p][k] - ts.centre) * ts.escale;
                    x1 = (v[2 * p + 1][k] - ts.centre) * ts.escale;
                }
            const __half2 h = __floats2half2_rn(x0, x1);
            hi[p] = h2_bits(h);
            const float2 hf = __half22float2(h);
            lo[p] = h2_bits(__floats2half2_rn(x0 - hf.x, x1 - hf.y));
        }
        const int off = g.a_off(4 * q + c, 8 * s);
        *reinterpret_cast<uint4*>(A0 + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(A1 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
}

// Stages tile (tx0, ty0) into A buffer `abuf` (all worker threads).
template <typename Tin>
__device__ __forceinline__ TileScale stage_tile(const F2DTcArgs& a, const TcGeom& g, unsigned char* sm, int abuf,
                                                float* red, int tx0, int ty0, int wtid) {
    constexpr bool FSRC = sizeof(Tin) == 4;
    const int nq = g.XR / 4, ns = g.KR / 8, items = nq * ns;
    const int gx_base = tx0 - g.axa, gy_base = ty0 - a.ay;
    // Operands are centred: uint8 pixels minus 128 (exact in FP16); float
    // tiles about the middle of their range, scaled by a power of two so
    // that the largest centred magnitude lies in [2^14, 2^15).  The epilogue
    // adds centre * sum(taps) back.
    TileScale ts{1.f, 128.f, a.tap_unscale, 0.f};
    if constexpr (FSRC) {
        const int warp = wtid >> 5, lane = wtid & 31;
        float mx = -3.4e38f, mn = 3.4e38f;
        for (int it = wtid; it < items; it += kTcWorkers) {
            float v[8][4];
            load_item<Tin>(a, gy_base + 8 * (it / nq), gx_base + 4 * (it % nq), v);
#pragma unroll
            for (int j = 0; j < 8; ++j)
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    mx = fmaxf(mx, v[j][c]);
                    mn = fminf(mn, v[j][c]);
                }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        }
        if (lane == 0) {
            red[warp] = mx;
            red[8 + warp] = mn;
        }
        workers_sync<kTcWorkers>();
        if (wtid == 0) {
            float gmx = -3.4e38f, gmn = 3.4e38f;
            for (int w = 0; w < kTcWorkers / 32; ++w) {
                gmx = fmaxf(gmx, red[w]);
                gmn = fminf(gmn, red[8 + w]);
            }
            const float c = 0.5f * gmx + 0.5f * gmn;
            const float r = fmaxf(gmx - c, c - gmn);
            int ex = 0;
            if (r > 0.f && r <= 3.0e38f) {
                frexpf(r, &ex);  // r = f 2^ex, f in [0.5, 1)
                ex = 15 - ex;
                ex = ex < -120 ? -120 : (ex > 120 ? 120 : ex);
            }
            red[16] = (float)ex;
            red[17] = (c == c && fabsf(c) <= 3.0e38f) ? c : 0.f;
        }
        workers_sync<kTcWorkers>();
        const int ex = (int)red[16];
        ts.centre = red[17];
        ts.escale = ldexpf(1.f, ex);
        ts.unscale = a.tap_unscale * ldexpf(1.f, -ex);
    }
    ts.offset = fmaf(ts.centre, a.tap_sum, a.delta);
    unsigned char* A0 = sm + g.a_buf(abuf, 0);
    unsigned char* A1 = sm + g.a_buf(abuf, FSRC ? 1 : 0);
    for (int it = wtid; it < items; it += kTcWorkers) {
        const int q = it % nq, s = it / nq;
        float v[8][4];
        load_item<Tin>(a, gy_base + 8 * s, gx_base + 4 * q, v);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            unsigned hi[4], lo[4];
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const float x0 = (v[2 * p][c] - ts.centre) * ts.escale, x1 = (v[2 * p + 1][c] - ts.centre) * ts.escale;
                const __half2 h = __floats2half2_rn(x0, x1);
                hi[p] = h2_bits(h);
                if constexpr (FSRC) {
                    const float2 hf = __half22float2(h);
                    lo[p] = h2_bits(__floats2half2_rn(x0 - hf.x, x1 - hf.y));
                }
            }
            const int off = g.a_off(4 * q + c, 8 * s);
            *reinterpret_cast<uint4*>(A0 + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            if constexpr (FSRC) *reinterpret_cast<uint4*>(A1 + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
    }
    return ts;
}

// Reads accumulator set `set` of tile (tx0, ty0) and stores the results
// (all worker threads; warp w reads TMEM lanes 32 (w mod 4) .. +31).
template <typename Tout>
__device__ __forceinline__ void epilogue_tile(const F2DTcArgs& a, uint32_t tbase, int set, int tx0, int ty0,
                                              const TileScale& ts, int wtid) {
    const int warp = wtid >> 5, lane = wtid & 31;
    const int x = tx0 + 32 * (warp & 3) + lane;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int gi = 2 * (warp >> 2) + h;  // warps 0-3: groups 0, 1; warps 4-7: groups 2, 3
        float v[16], w[16], u[16], z[16];
        const uint32_t ta = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(set * kSetCols + 64 * gi);
        tmem_ld16(ta, v);
        tmem_ld16(ta + (uint32_t)kCorrCol, w);
        if (a.kw > 1) {
            tmem_ld16(ta + (uint32_t)kOddCol, u);
            tmem_ld16(ta + (uint32_t)(kOddCol + kCorrCol), z);
        } else {
#pragma unroll
            for (int n = 0; n < 16; ++n) u[n] = z[n] = 0.f;
        }
        if (x < a.rowlen) {
#pragma unroll
            for (int n = 0; n < 16; ++n) {
                const int y = ty0 + kTcN * gi + n;
                if (y < a.H) {
                    const float acc = (v[n] + w[n]) + (u[n] + z[n]);
                    row_ptr_mut<Tout>(a.dst, a.dpitch, y)[x] = sat_from_f<Tout>(fmaf(acc, ts.unscale, ts.offset));
                }
            }
        }
    }
}

// Issues the MMAs of one tile from A buffer `abuf` into accumulator set
// `set` (one thread).  Descriptors advance by adding (offset >> 4) to the
// start-address field, which never carries: shared addresses stay below
// 2^18 bytes.
template <bool FSRC>
__device__ __forceinline__ void issue_tile(const F2DTcArgs& a, const TcGeom& g, uint32_t sm_base, uint32_t tbase,
                                           int abuf, int set) {
    const uint64_t da0 = tc_smem_desc(sm_base + (uint32_t)g.a_buf(abuf, 0), (uint32_t)g.lboA, 128);
    const uint64_t da1 = tc_smem_desc(sm_base + (uint32_t)g.a_buf(abuf, FSRC ? 1 : 0), (uint32_t)g.lboA, 128);
    (void)da1;
    const uint64_t db = tc_smem_desc(sm_base, 512, 128);  // 32 rows: hi taps, then lo taps
    const int ksteps = g.Kt / 16;
    const uint32_t lbo16 = (uint32_t)g.lboA >> 4;
    constexpr uint32_t id32 = tc_idesc(2 * kTcN), id16 = tc_idesc(kTcN);
    for (int gi = 0; gi < kTcGroups; ++gi) {
        const uint32_t d0 = tbase + (uint32_t)(set * kSetCols + 64 * gi);
        uint32_t first[2] = {0u, 0u};  // accumulate flags of the even and odd accumulators
        for (int i = 0; i < a.kw; ++i) {
            const uint32_t dm = d0 + (uint32_t)((i & 1) * kOddCol), dc = dm + (uint32_t)kCorrCol;
            const uint32_t ash16 = (uint32_t)(i * g.C + g.axa - g.axs);  // 16-byte rows
            const uint32_t bi16 = (uint32_t)(i * g.bytesBi) >> 4;
            uint32_t acc = first[i & 1];
#pragma unroll 4
            for (int ks = 0; ks < ksteps; ++ks) {
                const uint32_t ao = (uint32_t)(2 * gi + 2 * ks) * lbo16 + ash16;
                const uint32_t bo = bi16 + (uint32_t)(ks * 64);  // 2 slabs of 512 bytes
                tc_mma(dm, da0 + ao, db + bo, id32, acc);        // hi and lo taps: main and correction
                if constexpr (FSRC) tc_mma(dc, da1 + ao, db + bo, id16, 1u);  // lo pixels x hi taps
                acc = 1u;
            }
            first[i & 1] = 1u;
        }
    }
}

// Pipeline (per CTA, tiles t_0, t_1, ... of this CTA; buffer b = k mod 2):
//   workers: stage t_k into A[b], arrive full[b]; then read out t_{k-1}
//            (wait mma[b^1], tcgen05.ld, store), arrive tfree[b^1];
//   issuer:  wait full[b] and (k >= 2) tfree[b], issue t_k's MMAs into
//            accumulator set b, commit to mma[b].
// So staging of t_k and the read-out of t_{k-1} overlap the MMAs of t_{k-1}
// and t_k.  A[b] is free again once mma[b] of t_{k-2} has fired, which the
// workers saw in the read-out of t_{k-2}.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(kTcThreads, 1) filter2d_tc_kernel(const __grid_constant__ F2DTcArgs a) {
    constexpr bool FSRC = sizeof(Tin) == 4;
    extern __shared__ __align__(1024) unsigned char sm[];
    const TcGeom g(a.kw, a.kh, a.ax, a.ay, FSRC, a.C);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + g.offBar);   // [2]
    uint64_t* mma = full + 2;                                        // [2]
    uint64_t* tfree = full + 4;                                      // [2]
    uint64_t* drained = full + 6;                                    // teardown
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + g.offBar + 64);
    float* red = reinterpret_cast<float*>(sm + g.offBar + 80);       // 8 maxima, 8 minima, scale, centre
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // ---- once per CTA: B parts, barriers, tensor memory
    {
        const int n16 = g.bytesB / 16;
        uint4* b = reinterpret_cast<uint4*>(sm);
        for (int i = tid; i < n16; i += kTcThreads) b[i] = __ldg(a.btab + i);
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(&full[b], kTcWorkers);
            mbar_init(&mma[b], 1);
            mbar_init(&tfree[b], kTcWorkers);
        }
        mbar_init(drained, 1);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t sm_base = smem_u32(sm);

    if (warp == kTcWorkers / 32) {
        // ---- the MMA issuer
        if (lane == 0) {
            int k = 0;
            for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++k) {
                const int b = k & 1;
                if (!mbar_wait(&full[b], (unsigned)(k >> 1) & 1u, a.err, kErrTcWait, a.wait_ns)) break;
                if (k >= 2 && !mbar_wait(&tfree[b], (unsigned)((k - 2) >> 1) & 1u, a.err, kErrTcWait, a.wait_ns))
                    break;
                tc_fence_after();
                issue_tile<FSRC>(a, g, sm_base, tbase, b, b);
                tc_commit(&mma[b]);
            }
            tc_commit(drained);  // fires once every MMA issued above has completed
        }
        __syncwarp();
    } else {
        // ---- staging and read-out.  This CTA's tiles are t_j = blockIdx.x +
        // j gridDim.x.  Tile j+1 is staged one step ahead: in step j the
        // workers issue tile j+1's loads, read tile j-1 out while the tensor
        // cores run tile j, then convert and store tile j+1 (A buffer (j+1)
        // mod 2, free since tile j-1's MMAs completed).  A wait that times out
        // skips its read-out but never leaves the loop: the staging steps of
        // float tiles hold barriers that every worker must reach.
        const int nq = g.XR / 4, ns = g.KR / 8, items = nq * ns;
        const int ntl = a.ntiles > (int)blockIdx.x ? (a.ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
        const bool packed = !FSRC && a.byte_border;
        TileScale sc0{}, sc1{};  // scales of the tiles in A buffers 0 and 1
        auto tile_xy = [&](int j, int& tx0, int& ty0) {
            const int t = (int)blockIdx.x + j * (int)gridDim.x;
            tx0 = (t % a.tiles_x) * kTcM;
            ty0 = (t / a.tiles_x) * kTcRows;
        };
        constexpr int kTcItemsPerThread = tc_items_per_thread(FSRC);
        unsigned raw[kTcItemsPerThread][8];
        float fv[FSRC ? kTcItemsPerThread : 1][8][4];
        auto issue_loads = [&](int j) {
            int tx0, ty0;
            tile_xy(j, tx0, ty0);
#pragma unroll
            for (int r = 0; r < kTcItemsPerThread; ++r) {
                const int it = tid + r * kTcWorkers;
                if (it >= items) continue;
                const int gy0 = ty0 - a.ay + 8 * (it / nq), gx0 = tx0 - g.axa + 4 * (it % nq);
                if constexpr (FSRC) load_item<Tin>(a, gy0, gx0, fv[r]);
                else if (packed) load_item_raw(a, gy0, gx0, raw[r]);
            }
        };
        auto store_tile = [&](int j) {
            int tx0, ty0;
            tile_xy(j, tx0, ty0);
            const int b = j & 1;
            if constexpr (FSRC) {
                float mx = -3.4e38f, mn = 3.4e38f;
#pragma unroll
                for (int r = 0; r < kTcItemsPerThread; ++r) {
                    if (tid + r * kTcWorkers >= items) continue;
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj)
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            mx = fmaxf(mx, fv[r][jj][c]);
                            mn = fminf(mn, fv[r][jj][c]);
                        }
                }
                const TileScale ts = tile_scale_from(a, red, mx, mn, tid);
                unsigned char* A0 = sm + g.a_buf(b, 0);
                unsigned char* A1 = sm + g.a_buf(b, 1);
#pragma unroll
                for (int r = 0; r < kTcItemsPerThread; ++r) {
                    const int it = tid + r * kTcWorkers;
                    if (it < items) store_item_split(A0, A1, g, it % nq, it / nq, fv[r], ts, lane);
                }
                (b ? sc1 : sc0) = ts;
            } else if (packed) {
                unsigned char* A0 = sm + g.a_buf(b, 0);
#pragma unroll
                for (int r = 0; r < kTcItemsPerThread; ++r) {
                    const int it = tid + r * kTcWorkers;
                    if (it < items) store_item_raw(A0, g, it % nq, it / nq, raw[r], lane);
                }
                (b ? sc1 : sc0) = TileScale{1.f, 128.f, a.tap_unscale, fmaf(128.f, a.tap_sum, a.delta)};
            } else {
                (b ? sc1 : sc0) = stage_tile<Tin>(a, g, sm, b, red, tx0, ty0, tid);
            }
            fence_async_smem();
            mbar_arrive(&full[b]);
        };
        auto read_out = [&](int j) {
            const int pb = j & 1;
            int px, py;
            tile_xy(j, px, py);
            if (mbar_wait(&mma[pb], (unsigned)(j >> 1) & 1u, a.err, kErrTcWait, a.wait_ns)) {
                tc_fence_after();
                epilogue_tile<Tout>(a, tbase, pb, px, py, pb ? sc1 : sc0, tid);
                tc_fence_before();
            }
        };
        if (ntl > 0) {
            issue_loads(0);
            store_tile(0);
        }
        for (int j = 0; j < ntl; ++j) {
            if (j + 1 < ntl) issue_loads(j + 1);
            if (j >= 1) {
                read_out(j - 1);
                mbar_arrive(&tfree[(j - 1) & 1]);
            }
            if (j + 1 < ntl) store_tile(j + 1);
        }
        if (ntl > 0) read_out(ntl - 1);
    }

    // ---- teardown: every MMA has completed before the columns are freed
    // (its own bound, not the pipeline's; if even that gives up, the columns
    // stay allocated rather than freed under a running MMA)
    __syncthreads();
    if (warp == 0) {
        bool ok = true;
        if (lane == 0) ok = mbar_wait(drained, 0, a.err, kErrTcDrain, kDrainNs);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        tc_fence_after();
        if (ok)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTmemCols)
                         : "memory");
    }
}

bool tc_supported(int sdt, int ddt) {
    return (sdt == IPFC_U8 && (ddt == IPFC_U8 || ddt == IPFC_F32 || ddt == IPFC_I16 || ddt == IPFC_U16)) ||
           (sdt == IPFC_F32 && ddt == IPFC_F32);
}

template <typename Tin, typename Tout>
cudaError_t tc_launch_typed(const F2DTcArgs& a, const TcGeom& g, cudaStream_t s) {
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)filter2d_tc_kernel<Tin, Tout>, 227 * 1024, &done);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int grid = a.ntiles < sms ? a.ntiles : sms;
    if (g.smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    // One CTA per SM: it allocates all 512 tensor-memory columns, so a second
    // resident CTA would only wait for them.  Asking for more than half the
    // SM's shared memory keeps the second one off.
    const int smem = g.smem > 120 * 1024 ? g.smem : 120 * 1024;
    filter2d_tc_kernel<Tin, Tout><<<grid, kTcThreads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

// Builds B (taps hi in rows 0-15, lo in rows 16-31, scaled by 2^s) in the
// shared layout.
void tc_build_b(const TcGeom& g, const float* taps, std::vector<__half>& out, float* tap_unscale) {
    double mx = 0;
    for (int j = 0; j < g.kh; ++j)
        for (int i = 0; i < g.kw; ++i) mx = std::fmax(mx, std::fabs((double)taps[(size_t)j * g.kw + i]));
    int ex = 0;
    if (mx > 0) {
        std::frexp(mx, &ex);
        ex = 15 - ex;  // max |w| * 2^s in [2^14, 2^15)
    }
    *tap_unscale = (float)std::ldexp(1.0, -ex);
    out.assign((size_t)g.bytesB / 2, __float2half(0.f));
    for (int i = 0; i < g.kw; ++i)
        for (int n = 0; n < kTcN; ++n)
            for (int j = 0; j < g.kh; ++j) {
                const int k = n + j;
                const double w = std::ldexp((double)taps[(size_t)j * g.kw + i], ex);
                const __half hi = __double2half(w);
                const __half lo = __double2half(w - (double)__half2float(hi));
                out[(size_t)g.b_off(i, n, k) / 2] = hi;
                out[(size_t)g.b_off(i, kTcN + n, k) / 2] = lo;
            }
}

// Single-channel images of the supported types, and uint8 images of 3 or 4
// interleaved channels, while the staged tile fits shared memory and the
// staging items fit the workers.
bool filter2d_tc_eligible(int sdt, int ddt, int C, int kw, int kh) {
    if (!(tc_supported(sdt, ddt) && kw >= 1 && kh >= 1 && kw <= kTcMaxKw && kh <= kTcMaxKh)) return false;
    if (!(C == 1 || ((C == 3 || C == 4) && sdt == IPFC_U8))) return false;
    const TcGeom g(kw, kh, kw / 2, kh / 2, sdt == IPFC_F32, C);
    const int items = (g.XR / 4) * (g.KR / 8);
    return g.smem <= 227 * 1024 && items <= tc_items_per_thread(sdt == IPFC_F32) * kTcWorkers;
}

// Launches the tensor-core form; taps are the dense kw x kh kernel (host).
cudaError_t filter2d_tc_launch(int sdt, int ddt, const void* src, long long spitch, void* dst, long long dpitch, int W,
                               int H, int C, const float* taps, int kw, int kh, int ax, int ay, int border, float delta,
                               float bv, cudaStream_t s) {
    const TcGeom g(kw, kh, ax, ay, sdt == IPFC_F32, C);
    if (g.smem > 227 * 1024 || (g.XR / 4) * (g.KR / 8) > tc_items_per_thread(sdt == IPFC_F32) * kTcWorkers)
        return cudaErrorInvalidConfiguration;
    std::vector<__half> bt;
    F2DTcArgs a;
    std::memset(&a, 0, sizeof(a));
    tc_build_b(g, taps, bt, &a.tap_unscale);
    double tsum = 0;
    for (int k = 0; k < kw * kh; ++k) tsum += (double)taps[k];
    a.tap_sum = (float)tsum;
    uint4* dbt = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dbt, bt.size() * sizeof(__half), s);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(dbt, bt.data(), bt.size() * sizeof(__half), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        a.src = src;
        a.spitch = spitch;
        a.dst = dst;
        a.dpitch = dpitch;
        a.W = W;
        a.H = H;
        a.C = C;
        a.rowlen = W * C;
        a.border = border;
        a.delta = delta;
        a.bv = bv;
        a.kw = kw;
        a.kh = kh;
        a.ax = ax;
        a.ay = ay;
        a.tiles_x = (W * C + kTcM - 1) / kTcM;
        a.ntiles = a.tiles_x * ((H + kTcRows - 1) / kTcRows);
        a.btab = dbt;
        a.byte_border = (sdt == IPFC_U8 && (border != IPFC_BORDER_CONSTANT ||
                                            (bv >= 0.f && bv <= 255.f && bv == std::floor(bv)))) ? 1 : 0;
        a.bvb = (border == IPFC_BORDER_CONSTANT && a.byte_border) ? (unsigned char)bv : 0;
        a.err = device_error_word();
        a.wait_ns = device_wait_limit_ns();
        if (sdt == IPFC_F32) e = tc_launch_typed<float, float>(a, g, s);
        else if (ddt == IPFC_U8) e = tc_launch_typed<uint8_t, uint8_t>(a, g, s);
        else if (ddt == IPFC_U16) e = tc_launch_typed<uint8_t, uint16_t>(a, g, s);
        else if (ddt == IPFC_I16) e = tc_launch_typed<uint8_t, int16_t>(a, g, s);
        else e = tc_launch_typed<uint8_t, float>(a, g, s);
    }
    cudaFreeAsync(dbt, s);
    return e;
}

}  // namespace ipfc
