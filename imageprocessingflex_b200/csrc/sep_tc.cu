// sep_tc.cu -- separable correlation (gaussianBlur, sepFilter2D) of uint8
// images with the column pass on tcgen05 tensor cores and the row pass on the
// CUDA cores.
//
// Same result definition as sep_fast (after include/ipf/filter.hpp:37-90);
// the passes are separable, so the column pass runs first.  Both passes on
// the CUDA cores cost 2K FP32 multiply-adds per output sample, which caps a
// CUDA-core kernel well below the HBM bound on B200; here the column pass
// moves to the tensor cores:
//
//  * a CTA tile is 256 interleaved source samples (two MMA blocks of M = 128)
//    by 48 output rows.  The source tile, borders resolved in both
//    directions at load, is staged transposed (sample-major, rows
//    contiguous) as FP16 K-major core matrices, uint8 values centred by 128
//    (exact in FP16);
//  * the column pass is D[m][n] = sum_k A[m][16 g + k] B[n][k] (N = 32, K =
//    the window rows padded to 16), B holding the vertical taps as a band,
//    hi parts in rows 0-15 and lo parts in rows 16-31 (one MMA fills the
//    hi and the correction accumulator); FP32 accumulation in tensor
//    memory (256 columns per CTA);
//  * the worker warps read the column results (main + correction, scaled,
//    + 128 * sum(ky)) out of tensor memory into a pair-interleaved shared
//    buffer P[y][j] = {V[y][j], V[y][j + D]} (D = half the tile's output
//    samples), so that the row pass computes outputs q and q + D with one
//    fma.rn.f32x2 per tap;
//  * the row pass rounds pairs of outputs with packed round-toward-minus-
//    infinity adds (exact round-half-away, see sep_fast.cuh) and stores 8
//    bytes per half.
// Two CTAs per SM, each with 8 worker warps and one MMA warp (one CTA's staging
// and row pass fill the other's waits), mbarrier handshakes, every
// wait bounded (a timeout records kErrSepTcWait in the device error word).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/ipfc.h"
#include "common.cuh"
#include "filter2d_tc.cuh"
#include "sep_fast.cuh"
#include "tc_common.cuh"

namespace ipfc {

int set_error(int code, const char* fmt, ...);
unsigned* device_error_word();
cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

constexpr unsigned kErrSepTcWait = 0x301u;

namespace {

constexpr int kStM = 128;                 // MMA M (samples)
constexpr int kStBlocks = 2;              // M blocks per tile
constexpr int kStXR = kStM * kStBlocks;   // staged samples per tile row
constexpr int kStGroups = 3;              // 16-row MMA groups per tile
constexpr int kStRows = 16 * kStGroups;   // output rows per tile
constexpr int kStWorkers = 256;
constexpr int kStThreads = kStWorkers + 32;
constexpr int kStRun = 8;                 // outputs per row-pass item (each half)
constexpr int kStTmemCols = 256;          // 2 blocks x 3 groups x 32, one set per CTA, two CTAs per SM
constexpr int kStMaxBBytes = 2048;        // B for K <= 17 (Kt = 32)
constexpr int kStItemsPerThread = 2;      // staging work items per worker thread (at most)
constexpr int kStCtasPerSm = 2;

struct SepTcArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H;
    int border;
    float bv;
    float delta;
    float ky_unscale;  // 2^-s of the vertical taps
    float ky_sum;      // sum of the vertical taps (FP64, rounded once)
    int tiles_x, ntiles;
    int clamp;         // outputs may leave [0, 255]: saturate
    int vec_store;     // destination base and pitch allow 8-byte stores
    unsigned char bvb; // Constant border value as a byte (integer in [0, 255])
    unsigned* err;
    unsigned long long kx2[kFastMaxTaps];  // horizontal taps, each packed twice
    uint4 btab[kStMaxBBytes / 16];         // vertical taps B in the shared layout
};

// Tile geometry for K taps and C channels (host and device).
struct StGeom {
    int HX, HXa, OUT, D, PW, Kt, KR, lboA, bytesA, bytesB, offA, offP, offBar, smem;
    __host__ __device__ StGeom(int K, int C) {
        HX = (K / 2) * C;
        HXa = (HX + 3) / 4 * 4;
        OUT = (kStXR - 2 * HXa) / 16 * 16;
        D = OUT / 2;
        PW = ((D + 2 * HXa) + 15) / 16 * 16 + 2;  // float2 per row, = 2 (mod 16): 16-byte rows spread over banks
        Kt = (K + 15 + 15) / 16 * 16;
        KR = 16 * (kStGroups - 1) + Kt;
        lboA = kStXR * 16;
        bytesA = (KR / 8) * lboA;
        bytesB = (Kt / 8) * 512;
        offA = bytesB;
        offP = offA + bytesA;                     // one A buffer, one P buffer
        offBar = offP + kStRows * PW * 8;
        smem = offBar + 128;
    }
};

// 8 rows x 4 samples of the source at (gy0, flat sample gq0), borders
// resolved in both directions, as one 32-bit word (4 bytes) per row.
__device__ __forceinline__ void st_load_raw(const SepTcArgs& a, int C, int gy0, int gq0, unsigned (&w)[8]) {
    const int rowlen = a.W * C;
    const bool cols_in = gq0 >= 0 && gq0 + 4 <= rowlen;
    int cx[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) cx[c] = cols_in ? gq0 + c : border_sample(gq0 + c, a.W, C, a.border);
    const unsigned cfill = 0x01010101u * a.bvb;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int sy = border_index(gy0 + j, a.H, a.border);
        if (sy < 0) {
            w[j] = cfill;
            continue;
        }
        const uint8_t* row = row_ptr<uint8_t>(a.src, a.spitch, sy);
        if (cols_in && (((uintptr_t)(row + gq0)) & 3) == 0) {
            w[j] = __ldg(reinterpret_cast<const unsigned*>(row + gq0));
            continue;
        }
        unsigned x = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) x |= (cx[c] < 0 ? (unsigned)a.bvb : (unsigned)__ldg(row + cx[c])) << (8 * c);
        w[j] = x;
    }
}

// The 4 staged 16-byte rows (one per sample) of one work item: sample c's 8
// source rows as FP16 values centred by 128.  uint8 b -> f16 bits 0x6400 | b
// (= 1024 + b, two bytes per PRMT pair), minus 1152 (0x6480): b - 128, exact.
__device__ __forceinline__ void st_store_item(unsigned char* A, int lboA, int q, int s, const unsigned (&w)[8],
                                              int rot) {
    const __half2 k1152 = __halves2half2(__ushort_as_half((unsigned short)0x6480), __ushort_as_half((unsigned short)0x6480));
    // lanes store their four chunks in rotated order: 16-byte stores of one
    // instruction then land 80 bytes apart, on distinct bank groups
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
        *reinterpret_cast<uint4*>(A + s * lboA + (4 * q + (int)c) * 16) = make_uint4(h[0], h[1], h[2], h[3]);
    }
}

template <int K, int C>
__global__ void __launch_bounds__(kStThreads, kStCtasPerSm) sep_tc_kernel(const __grid_constant__ SepTcArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const StGeom g(K, C);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + g.offBar);  // A staged
    uint64_t* mma = full + 1;                                       // column pass done
    uint64_t* tfree = full + 2;                                     // accumulators read out
    uint64_t* drained = full + 3;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + g.offBar + 64);
    float2* P = reinterpret_cast<float2*>(sm + g.offP);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    {
        const int n16 = g.bytesB / 16;
        uint4* b = reinterpret_cast<uint4*>(sm);
        for (int i = tid; i < n16; i += kStThreads) b[i] = a.btab[i];
    }
    if (tid == 0) {
        mbar_init(full, kStWorkers);
        mbar_init(mma, 1);
        mbar_init(tfree, kStWorkers);
        mbar_init(drained, 1);
    }
    if (warp == 0) tmem_alloc(tslot, kStTmemCols);
    fence_async_smem();
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;
    const uint32_t sm_base = smem_u32(sm);
    const int rowlen = a.W * C;

    if (warp == kStWorkers / 32) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint64_t db = tc_smem_desc(sm_base, 512, 128);
            constexpr uint32_t id32 = tc_idesc(32);
            const uint32_t lbo16 = (uint32_t)g.lboA >> 4;
            int k = 0;
            for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++k) {
                if (!mbar_wait(full, (unsigned)k & 1u, a.err, kErrSepTcWait)) break;
                if (k >= 1 && !mbar_wait(tfree, (unsigned)(k - 1) & 1u, a.err, kErrSepTcWait)) break;
                tc_fence_after();
                const uint64_t da = tc_smem_desc(sm_base + (uint32_t)g.offA, (uint32_t)g.lboA, 128);
                for (int mb = 0; mb < kStBlocks; ++mb)
                    for (int gi = 0; gi < kStGroups; ++gi) {
                        const uint32_t d = tbase + (uint32_t)(mb * 32 * kStGroups + 32 * gi);
                        for (int ks = 0; ks < g.Kt / 16; ++ks) {
                            const uint32_t ao = (uint32_t)(mb * kStM) + (uint32_t)(2 * gi + 2 * ks) * lbo16;
                            tc_mma(d, da + ao, db + (uint32_t)(ks * 64), id32, ks > 0 ? 1u : 0u);
                        }
                    }
                tc_commit(mma);
            }
            tc_commit(drained);
        }
        __syncwarp();
    } else {
        // ---- workers.  Iteration k: issue the loads of tile k's staging items
        // (into registers), read out tile k-1 and run its row pass while they
        // are in flight, then convert and store tile k's items and hand it to
        // the MMA warp.
        const int nq = kStXR / 4, ns = g.KR / 8, items = nq * ns;
        const float off = 128.f * a.ky_sum;
        int k = 0, ptx = 0, pty = 0;
        for (int t = blockIdx.x;; t += gridDim.x, ++k) {
            const bool have = t < a.ntiles;
            int tq0 = 0, ty0 = 0;
            unsigned raw[kStItemsPerThread][8];
            if (have) {
                tq0 = (t % a.tiles_x) * g.OUT;
                ty0 = (t / a.tiles_x) * kStRows;
                const int gq_base = tq0 - g.HXa, gy_base = ty0 - K / 2;
#pragma unroll
                for (int r = 0; r < kStItemsPerThread; ++r) {
                    const int it = tid + r * kStWorkers;
                    if (it < items) st_load_raw(a, C, gy_base + 8 * (it / nq), gq_base + 4 * (it % nq), raw[r]);
                }
            }
            if (k >= 1) {
                // read out tile k-1 into P.  Warp w reads TMEM lanes 32 (w mod 4)
                // .. +31 of M block (w / 4); all kStGroups groups.
                float2* Pb = P;
                const bool ok = mbar_wait(mma, (unsigned)(k - 1) & 1u, a.err, kErrSepTcWait);
                if (ok) {
                    tc_fence_after();
                    const int mb = warp >> 2;
                    const int xr = mb * kStM + 32 * (warp & 3) + lane;  // this thread's staged sample
#pragma unroll
                    for (int gi = 0; gi < kStGroups; ++gi) {
                        float mv[16], cv[16];
                        const uint32_t ta = tbase + ((uint32_t)(32 * (warp & 3)) << 16) +
                                            (uint32_t)(mb * 32 * kStGroups + 32 * gi);
                        tmem_ld16(ta, mv);
                        tmem_ld16(ta + 16u, cv);
#pragma unroll
                        for (int n = 0; n < 16; ++n) {
                            const float v = fmaf(mv[n] + cv[n], a.ky_unscale, off);
                            const int y = 16 * gi + n;
                            if (xr < g.PW) reinterpret_cast<float*>(Pb + y * g.PW + xr)[0] = v;
                            if (xr >= g.D && xr - g.D < g.PW) reinterpret_cast<float*>(Pb + y * g.PW + xr - g.D)[1] = v;
                        }
                    }
                    tc_fence_before();
                }
                mbar_arrive(tfree);
                workers_sync<kStWorkers>();
                // row pass of tile k-1
                if (ok) {
                    constexpr int NW = kStRun + 2 * (K / 2) * C;  // window (float2) per item
                    const int runs = g.D / kStRun;
                    for (int it = tid; it < runs * kStRows; it += kStWorkers) {
                        const int y = it % kStRows, run = it / kStRows;
                        const int gy = pty + y;
                        const int o = run * kStRun;
                        // 16-byte aligned: PW, o and HXa - HX are all even
                        const float4* pw4 = reinterpret_cast<const float4*>(Pb + y * g.PW + o + g.HXa - g.HX);
                        f2p w[NW + 1];
#pragma unroll
                        for (int j = 0; j < (NW + 1) / 2; ++j) {
                            const float4 f = pw4[j];
                            w[2 * j] = pk2(f.x, f.y);
                            w[2 * j + 1] = pk2(f.z, f.w);
                        }
                        f2p acc[kStRun];
#pragma unroll
                        for (int u = 0; u < kStRun; ++u) acc[u] = pk2(a.delta, a.delta);
#pragma unroll
                        for (int i = 0; i < K; ++i)
#pragma unroll
                            for (int u = 0; u < kStRun; ++u) acc[u] = ffma2p(a.kx2[i], w[u + i * C], acc[u]);
                        if (gy >= a.H) continue;
                        unsigned lo0 = 0, lo1 = 0, hi0 = 0, hi1 = 0;
#pragma unroll
                        for (int u = 0; u < kStRun; ++u) {
                            float2 v = upk2(acc[u]);
                            if (a.clamp) v = make_float2(fminf(fmaxf(v.x, 0.f), 255.f), fminf(fmaxf(v.y, 0.f), 255.f));
                            const float2 m = round_pair_u(v);
                            const unsigned bx = __float_as_uint(m.x), byv = __float_as_uint(m.y);
                            if (u < 4) {
                                lo0 = __byte_perm(lo0, bx, byte_insert_sel(u));
                                hi0 = __byte_perm(hi0, byv, byte_insert_sel(u));
                            } else {
                                lo1 = __byte_perm(lo1, bx, byte_insert_sel(u - 4));
                                hi1 = __byte_perm(hi1, byv, byte_insert_sel(u - 4));
                            }
                        }
                        unsigned char* drow = reinterpret_cast<unsigned char*>(a.dst) + (long long)gy * a.dpitch;
                        const int q0 = ptx + o, q1 = ptx + o + g.D;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int q = h ? q1 : q0;
                            const unsigned w0 = h ? hi0 : lo0, w1 = h ? hi1 : lo1;
                            if (q >= rowlen) continue;
                            if (a.vec_store && q + kStRun <= rowlen) {
                                *reinterpret_cast<uint2*>(drow + q) = make_uint2(w0, w1);
                            } else {
                                for (int e = 0; e < kStRun && q + e < rowlen; ++e)
                                    drow[q + e] = (unsigned char)((e < 4 ? w0 : w1) >> (8 * (e & 3)));
                            }
                        }
                    }
                }
            }
            if (!have) break;
            {
                unsigned char* A = sm + g.offA;
#pragma unroll
                for (int r = 0; r < kStItemsPerThread; ++r) {
                    const int it = tid + r * kStWorkers;
                    if (it < items) st_store_item(A, g.lboA, it % nq, it / nq, raw[r], lane);
                }
                fence_async_smem();
                mbar_arrive(full);
            }
            ptx = tq0;
            pty = ty0;
        }
    }

    __syncthreads();
    if (warp == 0) {
        if (lane == 0) mbar_wait(drained, 0, a.err, kErrSepTcWait);
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tbase, kStTmemCols);
    }
}

template <int K, int C>
cudaError_t sep_tc_launch_kc(const SepTcArgs& a, cudaStream_t s) {
    const StGeom g(K, C);
    static unsigned done = 0;
    cudaError_t e = ensure_smem_attr((const void*)sep_tc_kernel<K, C>, 227 * 1024, &done);
    if (e != cudaSuccess) return e;
    if (g.smem > 227 * 1024) return cudaErrorInvalidConfiguration;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int grid = a.ntiles < kStCtasPerSm * sms ? a.ntiles : kStCtasPerSm * sms;
    sep_tc_kernel<K, C><<<grid, kStThreads, g.smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

bool sep_tc_supported(int K, int C) {
    if (!(K == 13 && (C == 1 || C == 3 || C == 4))) return false;
    const StGeom g(K, C);
    return g.bytesB <= kStMaxBBytes && (kStXR / 4) * (g.KR / 8) <= kStItemsPerThread * kStWorkers;
}

// Launches the tensor-core separable kernel for uint8 -> uint8 with K taps
// per axis (centred) on C channels; false when (K, C) is not instantiated.
bool sep_tc_launch(const void* src, long long spitch, void* dst, long long dpitch, int W, int H, int C,
                   const double* kx, const double* ky, int K, int border, double delta, double bv, int clamp,
                   cudaStream_t s, cudaError_t* err) {
    if (!sep_tc_supported(K, C)) return false;
    // the staged tile holds bytes: a Constant border value must be one
    if (border == IPFC_BORDER_CONSTANT && !(bv >= 0 && bv <= 255 && bv == std::floor(bv))) return false;
    const StGeom g(K, C);
    // vertical taps: banded B, hi rows 0-15, lo rows 16-31, scaled by 2^s
    double mx = 0, sum = 0;
    for (int j = 0; j < K; ++j) {
        mx = std::fmax(mx, std::fabs(ky[j]));
        sum += ky[j];
    }
    int ex = 0;
    if (mx > 0) {
        std::frexp(mx, &ex);
        ex = 15 - ex;
    }
    std::vector<__half> bt((size_t)g.bytesB / 2, __float2half(0.f));
    for (int n = 0; n < 16; ++n)
        for (int j = 0; j < K; ++j) {
            const int kk = n + j;
            const double w = std::ldexp(ky[j], ex);
            const __half hi = __double2half(w);
            const __half lo = __double2half(w - (double)__half2float(hi));
            const int base = (kk >> 3) * 512 + (kk & 7) * 2;
            bt[(size_t)(base + (n >> 3) * 128 + (n & 7) * 16) / 2] = hi;
            bt[(size_t)(base + ((16 + n) >> 3) * 128 + (n & 7) * 16) / 2] = lo;
        }
    SepTcArgs a;
    std::memset(&a, 0, sizeof(a));
    a.src = src;
    a.spitch = spitch;
    a.dst = dst;
    a.dpitch = dpitch;
    a.W = W;
    a.H = H;
    a.border = border;
    a.bv = (float)bv;
    a.bvb = border == IPFC_BORDER_CONSTANT ? (unsigned char)bv : 0;
    a.delta = (float)delta;
    a.ky_unscale = (float)std::ldexp(1.0, -ex);
    a.ky_sum = (float)sum;
    a.tiles_x = (W * C + g.OUT - 1) / g.OUT;
    a.ntiles = a.tiles_x * ((H + kStRows - 1) / kStRows);
    a.clamp = clamp;
    a.vec_store = (((uintptr_t)dst) % 8 == 0 && dpitch % 8 == 0) ? 1 : 0;
    a.err = device_error_word();
    for (int i = 0; i < K; ++i) {
        const float f = (float)kx[i];
        unsigned u;
        std::memcpy(&u, &f, 4);
        a.kx2[i] = ((unsigned long long)u << 32) | u;
    }
    std::memcpy(a.btab, bt.data(), (size_t)g.bytesB);
    cudaError_t e;
    if (C == 1) e = sep_tc_launch_kc<13, 1>(a, s);
    else if (C == 3) e = sep_tc_launch_kc<13, 3>(a, s);
    else e = sep_tc_launch_kc<13, 4>(a, s);
    *err = e;
    return true;
}

}  // namespace ipfc
