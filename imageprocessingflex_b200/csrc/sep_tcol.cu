// sep_tcol.cu -- separable correlation of uint8 images (sepFilter2D,
// gaussianBlur, include/ipf/filter.hpp:37-90, 197-203, 262-267) with the
// column pass on tcgen05 tensor cores and the row pass on CUDA cores reading
// tensor memory directly.  Geometry and the GEMM form: sep_tcol.cuh.
//
// One persistent CTA per SM walks its share of (band, slab) units (128
// output rows x 128 interleaved samples), runs of one band bracketed by halo
// steps (TcolWalk).  Warp roles:
//  * warp 0: allocates 512 tensor-memory columns (four slab buffers); its
//    lane 0 issues, per step, KR/16 K steps x (A_hi, A_lo) MMAs into the
//    step's buffer and commits them to the B-empty and T-full barriers;
//  * warps 1-4 (producers): per step, load the band's KR source rows of the
//    slab (16-byte loads; at the image's edges 16 independent byte loads of
//    border-resolved samples, Constant as the border byte), convert
//    uint8 - 128 to FP16 exactly (byte permutes into 0x64xx, minus 1152) and
//    store them into one of two B buffers;
//  * warps 5-12 (row pass): warp w reads tensor-memory lanes 32 (w mod 4) ..
//    +31 -- one output row per thread -- and half the slab's columns, plus
//    C*(K/2) columns either side from the neighbouring slab buffers; runs the
//    K horizontal taps (FP32 FMAs with the taps as constant-bank operands);
//    rounds with one add toward -inf onto 2^23 (the +0.5 and every constant
//    term are folded into the accumulator's start value); packs bytes and
//    stores 16-byte runs of its output row.
// Handshakes are mbarriers (B full/empty, T full/empty) with bounded waits.
// A wait that gives up records kErrTcolWait in the device error word and
// sets an abort flag that every role checks per step.  Tensor memory is
// freed only after a final commit barrier shows every issued MMA complete;
// if even that bounded wait gives up, the memory is left allocated rather
// than freed under a running MMA (kErrTcolDrain).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "../../include/ipfc.h"
#include "common.cuh"
#include "sep_fast.cuh"
#include "sep_tcol.cuh"
#include "tc_common.cuh"

namespace ipfc {

unsigned* device_error_word();
unsigned long long device_wait_limit_ns();
cudaError_t ensure_smem_attr(const void* func, int bytes, unsigned* done_mask);

constexpr unsigned kErrTcolWait = 0x301u;   // a pipeline wait gave up
constexpr unsigned kErrTcolDrain = 0x302u;  // the final MMA drain gave up: tensor memory left allocated
constexpr int kTcolMaxCtas = 160;           // balanced unit split passed by value up to this grid
constexpr int kTcolMaxBuiltK = 15;          // odd K from 3 up to this are instantiated (KR = 144 rows)

struct TcolArgs {
    const unsigned char* src;
    long long spitch;
    unsigned char* dst;
    long long dpitch;
    int W, H, rowlen;
    int border;
    unsigned bvb;        // the Constant border value (a byte)
    int nb, ns, units;   // bands, slabs per band, nb * ns
    int clamp;           // outputs may leave [0, 255]
    int vec_store;       // destination base and pitch are 16-byte aligned
    float off;           // 128 * sum(ky) * sum(kx) + delta + 0.5
    unsigned long long wait_ns;   // a pipeline wait gives up after this long
    unsigned short ahi[kTcolMaxK + 1], alo[kTcolMaxK + 1];  // FP16 bits of ky * 2^e (hi, lo)
    unsigned long long kx2[kTcolMaxK + 1];                   // kx * 2^-e in both FP32 lanes
    unsigned* err;
    int nsplit;                      // > 0: CTA b walks units split[b] .. split[b+1]-1
    int split[kTcolMaxCtas + 1];
};

namespace {

// Bounded wait on a barrier phase.  The bound is wall time (a.wait_ns on
// the global timer), not a poll count: each poll may suspend the thread.
// Gives up early when another role has set the abort flag; a wait that runs
// out records kErrTcolWait and sets it.
__device__ __forceinline__ bool tcol_wait(uint64_t* bar, unsigned parity, const TcolArgs& a, volatile int* abort_flag) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        // sleeps (up to 50 us per poll) rather than spinning
        if (mbar_try_wait_sleep(bar, parity, 50000u)) return true;
        if (*abort_flag) return false;
        if (globaltimer_ns() - t0 > a.wait_ns) break;
    }
    if (a.err) atomicCAS(a.err, 0u, kErrTcolWait);
    *abort_flag = 1;
    return false;
}

// tcgen05.ld of 16 consecutive columns of this warp's lane quarter; the
// registers are valid after tcol_ld_wait on the same array.
__device__ __forceinline__ void tcol_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t* r = reinterpret_cast<uint32_t*>(v);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
// Waits for this thread's outstanding tensor-memory loads; the array is an
// in/out operand so no use of it moves above the wait.
__device__ __forceinline__ void tcol_ld_wait(float (&v)[16]) {
    uint32_t* r = reinterpret_cast<uint32_t*>(v);
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])::"memory");
}

// uint8 word -> two FP16x2 words of (byte - 128), exact.
__device__ __forceinline__ void tcol_cvt_word(unsigned w, unsigned& h01, unsigned& h23) {
    const __half2 k1152 = __halves2half2(__ushort_as_half((unsigned short)0x6480), __ushort_as_half((unsigned short)0x6480));
    const unsigned u01 = __byte_perm(w, 0x64646464u, 0x4140u);
    const unsigned u23 = __byte_perm(w, 0x64646464u, 0x4342u);
    h01 = h2_bits(__hsub2(*reinterpret_cast<const __half2*>(&u01), k1152));
    h23 = h2_bits(__hsub2(*reinterpret_cast<const __half2*>(&u23), k1152));
}

// 16 samples of source row srow (a row of the image) at the
// border-resolved sample indices sx (-1: Constant), packed
// as bytes, Constant as the border byte.  The 16 loads are unconditional (a
// Constant sample reads the row's first byte and is replaced afterwards), so
// that no branch separates them.
__device__ __forceinline__ uint4 tcol_gather16(const TcolArgs& a, const unsigned char* srow, const int (&sx)[16]) {
    unsigned b[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) b[e] = __ldg(srow + (sx[e] >= 0 ? sx[e] : 0));
    unsigned w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int e = 0; e < 16; ++e) w[e >> 2] |= (sx[e] >= 0 ? b[e] : a.bvb) << (8 * (e & 3));
    return make_uint4(w[0], w[1], w[2], w[3]);
}

// Two FP32 lanes in one 64-bit register pair (low: first).
__device__ __forceinline__ uint64_t tcol_pack2(float lo, float hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void tcol_unpack2(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
// d = a * b + c on both lanes, each rounded to nearest: the same result as
// two fmaf.
__device__ __forceinline__ uint64_t tcol_fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Horizontal taps of one 16-output chunk of a row, from the chunk's window
// v (group 0 = 16*GH columns left of the chunk), rounded and packed as 16
// bytes.  Output o = off + sum_i kx[i] v[o + C (i - K/2)], two outputs per
// packed FMA:
//  * taps whose offset C (i - K/2) is even read aligned register pairs for
//    the output pairs (2k, 2k+1) -- accumulators E[k], started at off;
//  * taps with odd offsets (odd C only) read aligned pairs for the output
//    pairs (2k-1, 2k) -- accumulators O[k], started at 0 -- and
//    acc(o) = E + O at the end.
// The FP32 sum order differs from one FMA chain only by that final add.
template <int K, int C, int GH, bool CLAMP>
__device__ __forceinline__ void tcol_row_chunk(const TcolArgs& a, const float (&v)[1 + 2 * GH][16],
                                               unsigned (&words)[4]) {
    constexpr int H2 = K / 2;
    constexpr bool kOdd = (C & 1) != 0;
    static_assert(!kOdd || 16 * GH >= C * H2 + 1, "odd-offset pairs stay inside the window");
    auto pair = [&](int c) -> uint64_t { return tcol_pack2(v[c >> 4][c & 15], v[(c + 1) >> 4][(c + 1) & 15]); };
    const uint64_t off2 = tcol_pack2(a.off, a.off);
    uint64_t E[8], O[kOdd ? 9 : 1];
#pragma unroll
    for (int k = 0; k < 8; ++k) E[k] = off2;
#pragma unroll
    for (int k = 0; k < (kOdd ? 9 : 1); ++k) O[k] = 0ull;
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const int d = C * (i - H2) + 16 * GH;
        const uint64_t kk = a.kx2[i];
        if (((C * (i - H2)) & 1) == 0) {
#pragma unroll
            for (int k = 0; k < 8; ++k) E[k] = tcol_fma2(kk, pair(2 * k + d), E[k]);
        } else if constexpr (kOdd) {
#pragma unroll
            for (int k = 0; k < 9; ++k) O[k] = tcol_fma2(kk, pair(2 * k - 1 + d), O[k]);
        }
    }
    float acc[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) tcol_unpack2(E[k], acc[2 * k], acc[2 * k + 1]);
    if constexpr (kOdd) {
        float ol[9], oh[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) tcol_unpack2(O[k], ol[k], oh[k]);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            acc[2 * k] += oh[k];
            acc[2 * k + 1] += ol[k + 1];
        }
    }
#pragma unroll
    for (int t4 = 0; t4 < 4; ++t4) {
        unsigned wd = 0;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            float x = acc[4 * t4 + t];
            if constexpr (CLAMP) x = fminf(fmaxf(x, 0.f), 255.f);
            const float r = __fadd_rd(x, 8388608.0f);
            wd = __byte_perm(wd, __float_as_uint(r), byte_insert_sel(t));
        }
        words[t4] = wd;
    }
}

}  // namespace

template <int K, int C, bool CLAMP>
__global__ void __launch_bounds__(kTcolThreads, 1) sep_tcol_kernel(const __grid_constant__ TcolArgs a) {
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr int KR = tcol_kr(K);
    constexpr int KSTEPS = KR / 16;
    constexpr int KG = KR / 8;
    constexpr int GH = tcol_halo_groups(K, C);  // halo groups of 16 columns either side
    constexpr int R = C * (K / 2);
    static_assert(GH <= 2, "row-pass window: at most 32 columns of halo");
    constexpr int NG = 1 + 2 * GH;  // column groups one row-pass chunk reads

    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + tcol_off_bar(K));
    uint64_t* bfull = bars;        // [2] producers -> MMA
    uint64_t* bempty = bars + 2;   // [2] MMA commit -> producers
    uint64_t* tfull = bars + 4;    // [4] MMA commit -> row pass
    uint64_t* tempty = bars + 8;   // [4] row pass -> MMA
    uint64_t* drain = bars + 12;   // final commit
    volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 13);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 14);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = smem_u32(sm);

    // ---- set-up: barriers, tensor memory, the banded tap operands A_hi, A_lo
    if (tid == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bfull[i], 32 * kTcolProdWarps);
            mbar_init(&bempty[i], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&tfull[i], 1);
            mbar_init(&tempty[i], kTcolRowWarps);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 0) tmem_alloc(tslot, kTcolTmemCols);
    // the taps into shared memory first: the A build below indexes them by
    // lane, which the parameter bank would serve one address at a time
    unsigned short* taps = reinterpret_cast<unsigned short*>(bars + 16);  // [2][32]
    if (tid < 2 * 32) taps[tid] = (tid & 32) ? a.alo[tid & 31] : a.ahi[tid & 31];
    __syncthreads();
    // A: one 16-byte core-matrix row (fixed m, 8 consecutive k) per item
    for (int it = tid; it < 2 * kTcolM * KG; it += kTcolThreads) {
        const int hl = it / (kTcolM * KG), rest = it % (kTcolM * KG);
        const int m = rest % kTcolM, kg = rest / kTcolM;
        const unsigned short* tap = taps + 32 * hl;
        unsigned w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int j0 = 8 * kg + 2 * e - m, j1 = j0 + 1;
            const unsigned lo = (j0 >= 0 && j0 < K) ? tap[j0] : 0u;
            const unsigned hi = (j1 >= 0 && j1 < K) ? tap[j1] : 0u;
            w[e] = lo | (hi << 16);
        }
        *reinterpret_cast<uint4*>(sm + tcol_off_a(hl, K) + tcol_a_off(m, 8 * kg)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;

    const int u0 = a.nsplit ? a.split[blockIdx.x] : (int)((long long)blockIdx.x * a.units / gridDim.x);
    const int u1 = a.nsplit ? a.split[blockIdx.x + 1] : (int)((long long)(blockIdx.x + 1) * a.units / gridDim.x);

    if (warp == 0) {
        // ------------------------------------------------------------ MMA issue
        if (lane == 0) {
            TcolWalk walk(u0, u1, a.ns);
            TcolStep st;
            int g = 0;
            bool issued = false;
            const uint32_t a_hi = sbase + tcol_off_a(0, K), a_lo = sbase + tcol_off_a(1, K);
            while (walk.next(st)) {
                if (*abort_flag) break;
                const int bb = g & 1, tb = g & 3;
                if (!tcol_wait(&bfull[bb], (unsigned)(g >> 1) & 1u, a, abort_flag)) break;
                if (g >= 4 && !tcol_wait(&tempty[tb], (unsigned)((g - 4) >> 2) & 1u, a, abort_flag)) break;
                tc_fence_after();
                const int n0 = st.kind == 2 ? 0 : st.kind == 0 ? kTcolN - 16 * GH : 0;
                const int nn = st.kind == 1 ? kTcolN : 16 * GH;
                const uint32_t idesc = tcol_idesc(nn);
                const uint32_t bsm = sbase + tcol_off_b(bb, K);
                const uint32_t d = tbase + (uint32_t)(tb * kTcolN + n0);
#pragma unroll 1
                for (int ks = 0; ks < KSTEPS; ++ks) {
                    const uint64_t bd = tcol_desc_b(bsm, ks, n0);
                    tc_mma(d, tcol_desc_a(a_hi, ks), bd, idesc, ks > 0 ? 1u : 0u);
                    tc_mma(d, tcol_desc_a(a_lo, ks), bd, idesc, 1u);
                }
                tc_commit(&bempty[bb]);
                tc_commit(&tfull[tb]);
                issued = true;
                ++g;
            }
            if (issued) tc_commit(drain);
            // leave the drain barrier's phase complete when nothing was issued
            else mbar_arrive(drain);
        }
        __syncwarp();
    } else if (warp <= kTcolProdWarps) {
        // ------------------------------------------------------------ producers
        // Each lane loads and converts the same items of every step -- rows
        // 8 kg + r8 for its warp's kg, samples n .. n+15 -- into registers
        // one step ahead: the loads of step g+1 are issued as soon as step g
        // is handed over, and land while the warp waits for step g+1's B
        // buffer.  One register buffer: with a second one copied into it at
        // the end of each step, the copy stalled on those loads and the
        // hand-overs came 1-2 us later (measured per warp).
        const int pw = warp - 1, r8 = lane & 7, c4 = lane >> 3;
        static_assert(kTcolProdWarps % 2 == 0, "the items of one warp share the half of the slab");
        const int n = 64 * (pw & 1) + 16 * c4;  // this lane's chunk of the slab
        constexpr int ITEMS = KG * 2;           // (K group, half of the slab)
        constexpr int PER = (ITEMS + kTcolProdWarps - 1) / kTcolProdWarps;
        // loads this lane's items of step q (rows outside the image under
        // Constant and chunks outside the step's range are left unloaded)
        auto load = [&](const TcolStep& q, uint4 (&raw)[PER]) {
            const int n_lo = q.kind == 0 ? kTcolN - 16 * GH : 0;
            const int n_hi = q.kind == 2 ? 16 * GH : kTcolN;
            if (n < n_lo || n >= n_hi) return;
            const int y0 = q.band * kTcolM - K / 2;
            const int gx = q.slab * kTcolN + n;
            const bool inside = gx >= 0 && gx + 16 <= a.rowlen;
            int sx[16];  // in [0, rowlen) or -1 (Constant); read at the image's left and right edges only
            if (!inside) {
#pragma unroll
                for (int e = 0; e < 16; ++e) sx[e] = border_sample(gx + e, a.W, C, a.border);
            }
#pragma unroll
            for (int r = 0; r < PER; ++r) {
                const int it = pw + r * kTcolProdWarps;
                if (it >= ITEMS) continue;
                const int sy = border_index(y0 + 8 * (it >> 1) + r8, a.H, a.border);
                if (sy < 0) {
                    const unsigned f = 0x01010101u * a.bvb;
                    raw[r] = make_uint4(f, f, f, f);
                } else if (inside) {
                    raw[r] = __ldg(reinterpret_cast<const uint4*>(a.src + (long long)sy * a.spitch + gx));
                } else {
                    raw[r] = tcol_gather16(a, a.src + (long long)sy * a.spitch, sx);
                }
            }
        };
        TcolWalk walk(u0, u1, a.ns), ahead(u0, u1, a.ns);
        TcolStep st, sa;
        uint4 cur[PER];
        if (ahead.next(sa)) load(sa, cur);
        int g = 0;
        while (walk.next(st)) {
            if (*abort_flag) break;
            const int bb = g & 1;
            if (g >= 2 && !tcol_wait(&bempty[bb], (unsigned)((g - 2) >> 1) & 1u, a, abort_flag)) break;
            unsigned char* B = sm + tcol_off_b(bb, K);
            const int n_lo = st.kind == 0 ? kTcolN - 16 * GH : 0;
            const int n_hi = st.kind == 2 ? 16 * GH : kTcolN;
            if (n >= n_lo && n < n_hi) {
#pragma unroll
                for (int r = 0; r < PER; ++r) {
                    const int it = pw + r * kTcolProdWarps;
                    if (it >= ITEMS) continue;
                    const int k = 8 * (it >> 1) + r8;
                    unsigned h[8];
                    tcol_cvt_word(cur[r].x, h[0], h[1]);
                    tcol_cvt_word(cur[r].y, h[2], h[3]);
                    tcol_cvt_word(cur[r].z, h[4], h[5]);
                    tcol_cvt_word(cur[r].w, h[6], h[7]);
                    *reinterpret_cast<uint4*>(B + tcol_b_off(n, k)) = make_uint4(h[0], h[1], h[2], h[3]);
                    *reinterpret_cast<uint4*>(B + tcol_b_off(n + 8, k)) = make_uint4(h[4], h[5], h[6], h[7]);
                }
            }
            fence_async_smem();
            mbar_arrive(&bfull[bb]);
            // the next step's items, in flight while this warp waits for
            // that step's B buffer
            if (ahead.next(sa)) load(sa, cur);
            ++g;
        }
    } else {
        // ------------------------------------------------------------ row pass
        const int rw = warp - 1 - kTcolProdWarps;  // 0 .. kTcolRowWarps-1
        const int q = warp & 3;                    // tensor-memory lane quarter of this warp
        const int h = rw >> 2;                     // which part of the slab's chunks (3, 3 or 2 of 16 columns)
        const int ch0 = tcol_row_chunk0(h), nch = tcol_row_chunk0(h + 1) - ch0;
        const uint32_t tlane = tbase + ((uint32_t)(32 * q) << 16);
        TcolWalk walk(u0, u1, a.ns);
        TcolStep st, prev{0, 0, 0};
        int g = 0, ga = 0;  // step index, and the index of the current run's left halo
        auto release = [&](int gg) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[gg & 3]);
        };
        while (walk.next(st)) {
            // warp-uniform decisions: every lane leaves together, so no
            // .sync.aligned instruction below runs with part of the warp
            if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
            const bool ok = tcol_wait(&tfull[g & 3], (unsigned)(g >> 2) & 1u, a, abort_flag);
            if (!__all_sync(0xffffffffu, ok)) break;
            tc_fence_after();
            if (st.kind == 0) ga = g;
            if (prev.kind == 1 && st.kind != 0) {
                // row pass of slab prev (step g-1): buffers g-2, g-1, g
                const int m = 32 * q + lane;
                const int y = prev.band * kTcolM + m;
                const int xs = prev.slab * kTcolN + 16 * ch0;  // first output sample of this thread
                // column group rg (relative to 64h, in 16s) -> tensor-memory address
                auto gaddr = [&](int rg) -> uint32_t {
                    const int col = 16 * (ch0 + rg);  // relative to slab g-1's buffer, may leave [0,128)
                    const int dg = col < 0 ? -1 : (col >= kTcolN ? 1 : 0);
                    const int buf = (g - 1 + dg) & 3;
                    return tlane + (uint32_t)(buf * kTcolN + (col - dg * kTcolN));
                };
                unsigned char* drow = a.dst + (long long)y * a.dpitch;
                const bool row_ok = y < a.H;
                // this warp's chunks of 16 outputs, one compiled body: the chunk's
                // window (its 16 columns and GH groups either side) is read
                // from tensor memory afresh, so the loop stays small enough
                // for the instruction cache
#pragma unroll 1
                for (int j = 0; j < nch; ++j) {
                    float v[NG][16];
                    __syncwarp();
                    static_for<0, NG>([&](auto I) {
                        constexpr int i = decltype(I)::value;
                        tcol_ld16(gaddr(j + i - GH), v[i]);
                    });
                    static_for<0, NG>([&](auto I) { tcol_ld_wait(v[decltype(I)::value]); });
                    unsigned words[4];
                    tcol_row_chunk<K, C, GH, CLAMP>(a, v, words);
                    const int xo = xs + 16 * j;
                    if (row_ok && xo < a.rowlen) {
                        if (a.vec_store && xo + 16 <= a.rowlen) {
                            *reinterpret_cast<uint4*>(drow + xo) = make_uint4(words[0], words[1], words[2], words[3]);
                        } else {
#pragma unroll
                            for (int e = 0; e < 16; ++e)
                                if (xo + e < a.rowlen) drow[xo + e] = (unsigned char)(words[e >> 2] >> (8 * (e & 3)));
                        }
                    }
                }
                (void)R;
            }
            // buffers no longer read: step g-2 when it belongs to this run, and
            // at the run's end its last two
            __syncwarp();
            if (st.kind != 0 && g - 2 >= ga) release(g - 2);
            if (st.kind == 2) {
                release(g - 1);
                release(g);
            }
            prev = st;
            ++g;
        }
    }

    // ---- teardown: every MMA complete before the tensor memory is freed
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        bool drained = true;
        if (lane == 0) {
            // every issued MMA completes in microseconds; this bound is its
            // own, independent of the (possibly shortened) pipeline bound
            drained = mbar_wait(drain, 0, a.err, kErrTcolDrain, kDrainNs);
        }
        drained = __shfl_sync(0xffffffffu, drained ? 1 : 0, 0) != 0;
        tc_fence_after();
        if (drained) tmem_dealloc(tbase, kTcolTmemCols);
    }
}

namespace {

// The split of the last (units, slabs per band, grid) this thread launched:
// a run of calls on one image size bisects once.
void tcol_split(TcolArgs& a, int grid) {
    thread_local int c_units = -1, c_ns = -1, c_grid = -1;
    thread_local int c_split[kTcolMaxCtas + 1];
    if (a.units != c_units || a.ns != c_ns || grid != c_grid) {
        tcol_split_units(a.units, a.ns, grid, c_split);
        c_units = a.units;
        c_ns = a.ns;
        c_grid = grid;
    }
    a.nsplit = grid;
    std::memcpy(a.split, c_split, sizeof(int) * (size_t)(grid + 1));
}

// The saturation is compiled out when the host has shown that every output
// stays inside [0, 255] (non-negative taps whose product of sums keeps the
// extreme inputs in range): the row pass then spends no issue slots on it.
template <int K, int C>
cudaError_t tcol_launch_kc(TcolArgs a, cudaStream_t s) {
    static unsigned done[2] = {0, 0};
    const void* fn = a.clamp ? (const void*)sep_tcol_kernel<K, C, true> : (const void*)sep_tcol_kernel<K, C, false>;
    cudaError_t e = ensure_smem_attr(fn, tcol_smem(K), &done[a.clamp ? 1 : 0]);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const int grid = a.units < sms ? a.units : sms;
    if (grid <= kTcolMaxCtas) tcol_split(a, grid);
    if (a.clamp)
        sep_tcol_kernel<K, C, true><<<grid, kTcolThreads, tcol_smem(K), s>>>(a);
    else
        sep_tcol_kernel<K, C, false><<<grid, kTcolThreads, tcol_smem(K), s>>>(a);
    return cudaGetLastError();
}

template <int K>
bool tcol_launch_k(int C, const TcolArgs& a, cudaStream_t s, cudaError_t* e) {
    if (C == 1) {
        *e = tcol_launch_kc<K, 1>(a, s);
        return true;
    }
    if constexpr (3 * (K / 2) <= 32) {
        if (C == 3) {
            *e = tcol_launch_kc<K, 3>(a, s);
            return true;
        }
    }
    if constexpr (4 * (K / 2) <= 32) {
        if (C == 4) {
            *e = tcol_launch_kc<K, 4>(a, s);
            return true;
        }
    }
    return false;
}

}  // namespace

// (K, C) combinations instantiated: odd K from 3 to 15 (144 staged rows; from
// 17 taps the 160-row band's producer registers spill) with C in {1, 3, 4}
// while the row pass reaches at most 32 columns either side (C * (K/2) <= 32).
bool sep_tcol_supported(int K, int C) {
    if (!(C == 1 || C == 3 || C == 4)) return false;
    if (K < 3 || K > kTcolMaxBuiltK || (K & 1) == 0) return false;
    return C * (K / 2) <= 32;
}

// Launches the tensor-core column-pass kernel for uint8 -> uint8 with K
// centred taps per axis on C channels; false when the call is outside what
// it covers (the caller then uses the CUDA-core kernel).
bool sep_tcol_launch(const void* src, long long spitch, void* dst, long long dpitch, int W, int H, int C,
                     const double* kx, const double* ky, int K, int border, double delta, double bv, int clamp,
                     cudaStream_t s, cudaError_t* err) {
    if (!sep_tcol_supported(K, C)) return false;
    if (((uintptr_t)src & 15) || (spitch & 15) || spitch <= 0 || spitch >= (1LL << 40)) return false;
    if (dpitch <= 0 || dpitch >= (1LL << 40)) return false;
    if (border == IPFC_BORDER_CONSTANT && !(bv == std::floor(bv) && bv >= 0.0 && bv <= 255.0)) return false;
    double mx = 0, sy = 0, sx = 0;
    for (int j = 0; j < K; ++j) {
        if (!std::isfinite(ky[j]) || !std::isfinite(kx[j])) return false;
        mx = std::fmax(mx, std::fabs(ky[j]));
        sy += ky[j];
        sx += kx[j];
    }
    int ex = 0;
    if (mx > 0) {
        int e2 = 0;
        std::frexp(mx, &e2);  // mx = f 2^e2, f in [0.5, 1)
        ex = 14 - e2;         // largest scaled tap in [2^13, 2^14)
    }
    TcolArgs a;
    std::memset(&a, 0, sizeof(a));
    a.src = static_cast<const unsigned char*>(src);
    a.spitch = spitch;
    a.dst = static_cast<unsigned char*>(dst);
    a.dpitch = dpitch;
    a.W = W;
    a.H = H;
    a.rowlen = W * C;
    a.border = border;
    a.bvb = border == IPFC_BORDER_CONSTANT ? (unsigned)bv : 0u;
    a.nb = (H + kTcolM - 1) / kTcolM;
    a.ns = (a.rowlen + kTcolN - 1) / kTcolN;
    a.units = a.nb * a.ns;
    a.clamp = clamp;
    a.vec_store = (((uintptr_t)dst & 15) == 0 && (dpitch & 15) == 0) ? 1 : 0;
    a.off = (float)(128.0 * sy * sx + delta + 0.5);
    a.wait_ns = device_wait_limit_ns();
    for (int j = 0; j < K; ++j) {
        const double w = std::ldexp(ky[j], ex);
        const __half hi = __double2half(w);
        const __half lo = __double2half(w - (double)__half2float(hi));
        a.ahi[j] = __half_as_ushort(hi);
        a.alo[j] = __half_as_ushort(lo);
        const float kxs = std::ldexp((float)kx[j], -ex);
        unsigned kb = 0;
        std::memcpy(&kb, &kxs, sizeof(kb));
        a.kx2[j] = ((unsigned long long)kb << 32) | kb;
    }
    a.err = device_error_word();
    cudaError_t e = cudaErrorInvalidValue;
    bool launched = false;
    switch (K) {
        case 3: launched = tcol_launch_k<3>(C, a, s, &e); break;
        case 5: launched = tcol_launch_k<5>(C, a, s, &e); break;
        case 7: launched = tcol_launch_k<7>(C, a, s, &e); break;
        case 9: launched = tcol_launch_k<9>(C, a, s, &e); break;
        case 11: launched = tcol_launch_k<11>(C, a, s, &e); break;
        case 13: launched = tcol_launch_k<13>(C, a, s, &e); break;
        case 15: launched = tcol_launch_k<15>(C, a, s, &e); break;
        default: return false;
    }
    if (!launched) return false;
    *err = e;
    return true;
}

}  // namespace ipfc
