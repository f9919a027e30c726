// sep_fast.cuh -- the fast fused separable correlation (compile-time taps).
//
// Same result definition as the generic form (sep_filter.cu, after
// include/ipf/filter.hpp:37-90) for equal horizontal and vertical tap counts
// K, channel counts 1, 3, 4 and the source/destination types instantiated in
// sep_fast_*.cu.  The column pass runs first -- a separable sum does not
// depend on the order -- because that order converts every source sample to
// FP32 exactly once:
//
//  * One CTA owns a strip of PX output pixels (all channels) and a run of
//    rows.  In the column pass each thread owns NCOL adjacent interleaved
//    source samples of the halo'd strip (4 for 8-bit sources, 2 for float),
//    converts them once per row and scatters them into a ring of K
//    accumulator pairs in registers with fma.rn.f32x2 (one instruction per
//    two samples; every ring index is a compile-time constant).  Each row's
//    samples are loaded K rows ahead of use through the read-only path (one
//    32-bit load per thread for 8-bit sources, the same instruction in every
//    lane); lanes with border-mapped samples add up to two cp.async word
//    copies per row and assemble their bytes at use; border rows resolve
//    through a non-inlined slow path.
//  * Finished column-pass rows go to shared memory split by channel
//    (planar), TB = K rows per band.  Then the CTA switches to the row
//    pass: one thread per (band row, run of RUN output pixels) reads its
//    window with 128-bit shared loads per channel, accumulates the K
//    horizontal taps, rounds pairs of outputs with two packed
//    round-toward-minus-infinity adds, byte-packs the interleaved output in
//    registers with PRMT and stores it with 64/128-bit stores.
//
// FP32 throughput bounds this kernel (2K multiply-adds per output sample);
// the design keeps every other instruction per sample to a few.
#pragma once

#include "common.cuh"

namespace ipfc {

constexpr int kFastThreads = 256;
constexpr int kFastMaxTaps = 32;
// Up to this many taps two CTAs share an SM (128 registers a thread); longer
// kernels need more registers for the K-deep accumulator ring and run one.
constexpr int kFastTwoCtaTaps = 15;

struct SepFastArgs {
    const void* src;
    long long spitch;
    void* dst;
    long long dpitch;
    int W, H;
    int border;
    float delta;
    float bv;
    int rows_per_cta;
    int strips;
    int vec_store;  // destination base and pitch allow 8/16-byte stores
    int vec_load;   // source base and pitch allow NCOL-sample loads
    int clamp;      // outputs may leave the destination range: saturate
    float kx[kFastMaxTaps];
    unsigned long long kx2[kFastMaxTaps];  // horizontal taps, each packed twice (f32x2)
    unsigned long long ky2[kFastMaxTaps];  // vertical taps, each packed twice (f32x2)
};

// ---- geometry (compile time) ------------------------------------------------
template <int K, int C, int NCOL>
struct FastGeom {
    static constexpr int RUN = 8;            // output pixels per row-pass item
    static constexpr int RX = K / 2;         // left halo (pixels)
    static constexpr int HX = K - 1;         // total horizontal halo
    // samples the threads cover; thread groups start NCOL-aligned
    static constexpr int ALIGN = NCOL;
    static constexpr int SPAN = NCOL * kFastThreads - (ALIGN - 1);
    static constexpr int TB = K;             // band rows: a multiple of K
    // utilisation (x1e6) of the column pass (threads with columns) times the
    // row pass (row-pair items over whole rounds) for strip width px
    static constexpr long long score(int px) {
        const int iw = (px + HX) * C;
        const int vthreads = (iw + NCOL - 1) / NCOL + 1;
        const int items = TB * (px / RUN);
        const int rounds = (items + kFastThreads - 1) / kFastThreads;
        return (long long)1000000 * vthreads / kFastThreads * items / (rounds * kFastThreads);
    }
    static constexpr int best_px() {
        int best = RUN;
        long long bs = -1;
        for (int px = RUN; (px + HX) * C <= SPAN; px += RUN)
            if (score(px) > bs) {
                bs = score(px);
                best = px;
            }
        return best;
    }
    static constexpr int PX = best_px();
    static constexpr int IW = (PX + HX) * C;  // source samples per strip row
    static constexpr int RUNS = PX / RUN;
    static constexpr int VW = PX + HX;        // plane row width (pixels)
    // row stride = 4 (mod 32) floats: lanes reading 16 B at the same column
    // of consecutive rows hit distinct 16-byte bank groups.  Column VW is
    // always padding: lanes without a column store there.
    static constexpr int VW4 = (VW + 1 + 3) / 4 * 4;
    static constexpr int VWP = VW4 + ((4 - VW4 % 32) + 32) % 32;
    static constexpr int PLANE = TB * VWP;
    static constexpr size_t PLANES_BYTES = sizeof(float) * (size_t)C * PLANE;
    // border lanes' extra words: K rows x 2 words x one per thread
    static constexpr size_t RING_BYTES = sizeof(unsigned) * 2 * K * kFastThreads;
    static constexpr size_t SMEM = PLANES_BYTES + RING_BYTES;
};

// ---- packed FP32 (fma/add .f32x2, sm_100a) ----------------------------------
// Accumulators, taps and operands stay packed in 64-bit registers across
// the hot loops.
typedef unsigned long long f2p;

__device__ __forceinline__ f2p pk2(float x, float y) {
    f2p p;
    asm("mov.b64 %0, {%1, %2};" : "=l"(p) : "f"(x), "f"(y));
    return p;
}
__device__ __forceinline__ float2 upk2(f2p p) {
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(p));
    return d;
}
__device__ __forceinline__ f2p ffma2p(f2p a, f2p b, f2p c) {
    f2p d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2p fadd2p(f2p a, f2p b) {
    f2p d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2p fadd2p_rm(f2p a, f2p b) {
    f2p d;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float lo_f(f2p p) { return __uint_as_float((unsigned)p); }
__device__ __forceinline__ float hi_f(f2p p) { return __uint_as_float((unsigned)(p >> 32)); }

// Round half away from zero to an unsigned integer in the low mantissa bits:
// floor(v +rm 0.5) equals round-half-away for every v >= 0 (a sum rounded
// toward -inf never lands on an integer the exact sum does not reach), and
// adding 2^23 rounded toward -inf leaves that floor in the low bits of a
// float in [2^23, 2^24).
__device__ __forceinline__ float2 round_pair_u(float2 v) {
    const f2p t = fadd2p_rm(pk2(v.x, v.y), pk2(0.5f, 0.5f));
    return upk2(fadd2p_rm(t, pk2(8388608.0f, 8388608.0f)));
}

// Signed destinations: exact round half away from zero, then saturate.
__device__ __forceinline__ int round_s_sat(float v, int lo, int hi) {
    const float t = truncf(v);
    const float r = fabsf(v - t) >= 0.5f ? t + copysignf(1.0f, v) : t;
    const float c = fminf(fmaxf(r, (float)lo), (float)hi);
    return (int)c;
}

// Border rows: kept out of line so the in-range test is all the hot loop
// executes for interior rows.  A row that reads the Constant value maps to
// row 0 (any readable row: the caller replaces those samples).
static __device__ __noinline__ int border_row_any_slow(int y, int n, int mode) {
    return max(border_index(y, n, mode), 0);
}
__device__ __forceinline__ int row_any(int y, int n, int mode) {
    return ((unsigned)y < (unsigned)n) ? y : border_row_any_slow(y, n, mode);
}

// Compile-time loop: f(std::integral_constant<int, I>) for I in [I0, N).
template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}

// 4-byte asynchronous copy global -> shared; only the first `n` (0..4) bytes
// are read, the rest of the destination word is zero-filled.  The source is
// 4-byte aligned.
__device__ __forceinline__ void cp_async4(unsigned* dst, const void* src, int n) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// PRMT selector that replaces byte `pos` of the first operand with byte 0 of
// the second.
__host__ __device__ constexpr unsigned byte_insert_sel(int pos) {
    return (0x3210u & ~(0xFu << (4 * pos))) | (4u << (4 * pos));
}

// ---- the row pass ------------------------------------------------------------
// Row pass over one band: thread = (band row, run of RUN output pixels).
// Inlined at its hot call site (once per band inside the unrolled loop);
// sep_row_pass_cold is the out-of-line copy for the last, partial band.
template <int K, int C, typename Tout, typename G>
__device__ __forceinline__ void sep_row_pass(const SepFastArgs& a, const float* vbuf, int rows_in_band, int band_start,
                                          int x0) {
    __syncthreads();
    for (int it = threadIdx.x; it < G::TB * G::RUNS; it += kFastThreads) {
        const int r = it % G::TB, g = it / G::TB;
        if (r >= rows_in_band) continue;
        const int y = band_start + r;
        const int p0 = g * G::RUN;  // strip-relative output pixel
        constexpr int NWORDS = (G::RUN * C * (int)sizeof(Tout) + 3) / 4;
        unsigned words[NWORDS];
#pragma unroll
        for (int w = 0; w < NWORDS; ++w) words[w] = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            constexpr int NW4 = (G::RUN + G::HX + 3) / 4;
            float win[NW4 * 4];
            const float4* src4 = reinterpret_cast<const float4*>(vbuf + c * G::PLANE + r * G::VWP + p0);
#pragma unroll
            for (int q = 0; q < NW4; ++q) {
                const float4 v4 = src4[q];
                win[4 * q] = v4.x;
                win[4 * q + 1] = v4.y;
                win[4 * q + 2] = v4.z;
                win[4 * q + 3] = v4.w;
            }
#pragma unroll
            for (int u = 0; u < G::RUN; u += 2) {
                float2 s = make_float2(a.delta, a.delta);
#pragma unroll
                for (int i = 0; i < K; ++i) {
                    s.x = fmaf(a.kx[i], win[u + i], s.x);
                    s.y = fmaf(a.kx[i], win[u + 1 + i], s.y);
                }
                const int e0 = u * C + c, e1 = (u + 1) * C + c;  // interleaved positions
                if constexpr (sizeof(Tout) == 1) {
                    if (a.clamp) s = make_float2(fminf(fmaxf(s.x, 0.f), 255.f), fminf(fmaxf(s.y, 0.f), 255.f));
                    const float2 m = round_pair_u(s);
                    // the byte is the low byte of the float's bit pattern
                    words[e0 >> 2] = __byte_perm(words[e0 >> 2], __float_as_uint(m.x), byte_insert_sel(e0 & 3));
                    words[e1 >> 2] = __byte_perm(words[e1 >> 2], __float_as_uint(m.y), byte_insert_sel(e1 & 3));
                } else if constexpr (std::is_same<Tout, int16_t>::value) {
                    words[e0 >> 1] |= (unsigned)(round_s_sat(s.x, -32768, 32767) & 0xffff) << (16 * (e0 & 1));
                    words[e1 >> 1] |= (unsigned)(round_s_sat(s.y, -32768, 32767) & 0xffff) << (16 * (e1 & 1));
                } else if constexpr (std::is_same<Tout, uint16_t>::value) {
                    if (a.clamp)
                        s = make_float2(fminf(fmaxf(s.x, 0.f), 65535.f), fminf(fmaxf(s.y, 0.f), 65535.f));
                    const float2 m = round_pair_u(s);
                    words[e0 >> 1] |= (__float_as_uint(m.x) & 0xffffu) << (16 * (e0 & 1));
                    words[e1 >> 1] |= (__float_as_uint(m.y) & 0xffffu) << (16 * (e1 & 1));
                } else {
                    words[e0] = __float_as_uint(s.x);
                    words[e1] = __float_as_uint(s.y);
                }
            }
        }
        if (y >= a.H) continue;
        const int px = x0 + p0;
        constexpr int NBYTES = G::RUN * C * (int)sizeof(Tout);
        // one 32 x 32 -> 64-bit multiply-add (pitches are below 2^31)
        unsigned char* db = static_cast<unsigned char*>(a.dst) + (size_t)(unsigned)(px * C * (int)sizeof(Tout)) +
                            (unsigned long long)(unsigned)y * (unsigned)a.dpitch;
        if (px + G::RUN <= a.W && a.vec_store) {
            if constexpr (NBYTES % 16 == 0) {
#pragma unroll
                for (int q = 0; q < NBYTES / 16; ++q)
                    reinterpret_cast<uint4*>(db)[q] =
                        make_uint4(words[4 * q], words[4 * q + 1], words[4 * q + 2], words[4 * q + 3]);
            } else {
#pragma unroll
                for (int q = 0; q < NBYTES / 8; ++q)
                    reinterpret_cast<uint2*>(db)[q] = make_uint2(words[2 * q], words[2 * q + 1]);
            }
        } else {
            const int nbytes = min(G::RUN, a.W - px) * C * (int)sizeof(Tout);
#pragma unroll
            for (int e = 0; e < NBYTES; ++e)
                if (e < nbytes) db[e] = (unsigned char)((words[e >> 2] >> (8 * (e & 3))) & 0xffu);
        }
    }
    __syncthreads();
}

template <int K, int C, typename Tout, typename G>
__device__ __noinline__ void sep_row_pass_cold(const SepFastArgs& a, const float* vbuf, int rows_in_band,
                                               int band_start, int x0) {
    sep_row_pass<K, C, Tout, G>(a, vbuf, rows_in_band, band_start, x0);
}

// ---- one tile: a strip of PX output pixels x a chunk of a.rows_per_cta rows
// Called by sep_fast_kernel (one tile per CTA) and by the persistent batch
// kernel (batch.cu, tiles from a queue).  `a` may live in the parameter
// space or in shared memory; vbuf is G::SMEM bytes of shared memory.
template <int K, int C, typename Tin, typename Tout>
__device__ __forceinline__ void sep_fast_tile(const SepFastArgs& a, float* vbuf, int strip, int chunk) {
    constexpr int NCOL = sizeof(Tin) == 1 ? 4 : 2;
    constexpr int NP = NCOL / 2;  // accumulator pairs per ring slot
    using G = FastGeom<K, C, NCOL>;
    const int tid = threadIdx.x;
    const int x0 = strip * G::PX;                  // first output pixel of the strip
    const int r0 = chunk * a.rows_per_cta;         // first output row
    if (r0 >= a.H) return;
    const int nrows = min(a.rows_per_cta, a.H - r0);
    const int rowlen = a.W * C;

    // --- this thread's NCOL source columns: strip-relative samples s0 .. s0+NCOL-1
    const int g0 = (x0 - G::RX) * C;               // global sample of strip sample 0
    const int lead = g0 & (G::ALIGN - 1);          // thread groups start on an aligned global sample
    const int s0 = NCOL * tid - lead;
    // samples that a stored output reads: the strip's outputs inside the image and their halo
    const int used = min(G::IW, (min(G::PX, a.W - x0) + G::HX) * C);
    const bool active = s0 + NCOL - 1 >= 0 && s0 < used;
    int idx[NCOL];
    bool vec = active && a.vec_load;
#pragma unroll
    for (int k = 0; k < NCOL; ++k) {
        const int g = g0 + s0 + k;
        idx[k] = !active ? -1 : (((unsigned)g < (unsigned)rowlen) ? g : border_sample(g, a.W, C, a.border));
        vec = vec && idx[k] == idx[0] + k;
    }
    vec = vec && idx[0] >= 0 && (idx[0] & (NCOL - 1)) == 0;
    unsigned cmask = 0;  // columns that read the Constant border value
#pragma unroll
    for (int k = 0; k < NCOL; ++k) cmask |= (active && idx[k] < 0 ? 1u : 0u) << k;

    // Load plan.  The row loop prefetches K rows ahead, and a prefetch only
    // overlaps the work in between when it is one load straight into its ring
    // register, the same instruction in every lane (a load whose value merges
    // across a branch makes the warp wait for it).  So:
    //  * every lane loads one aligned in-row word per row (element c0) into the
    //    register ring: its own NCOL samples when they are in order and
    //    aligned, any in-row word otherwise;
    //  * a lane whose samples are border-mapped or straddle the row end also
    //    copies the other aligned words that hold them (c1, c2; n1, n2 of their
    //    bytes lie in the row, the rest is zero-filled and never read) into a
    //    shared ring with cp.async, and assembles its samples at use -- two
    //    byte permutes (8-bit) or a select (float).  Warps without such lanes
    //    skip the copies (a warp-uniform branch, no register involved);
    //  * unaligned sources (or a lane needing more than three words) fall back
    //    to one load per sample for the warp.
    // Lanes whose sample reads the Constant value take any byte there.
    int c0 = 0, c1 = 0, c2 = 0, n1 = 0, n2 = 0;
    unsigned selA = 0x3210u, selB = 0x3210u;  // 8-bit: t = prmt(reg, w1, selA); raw = prmt(t, w2, selB)
    bool extra = false, fail = !a.vec_load || rowlen < NCOL;
    if (!fail && active) {
        if (vec) {
            c0 = idx[0];
        } else if constexpr (sizeof(Tin) == 1) {
            int wk[NCOL];
#pragma unroll
            for (int k = 0; k < NCOL; ++k) wk[k] = idx[k] >= 0 ? (idx[k] & ~3) : -1;
            // register word: the first word that lies wholly in the row (else word 0, unused)
            int wa = -1;
#pragma unroll
            for (int k = NCOL - 1; k >= 0; --k)
                if (wk[k] >= 0 && wk[k] + 4 <= rowlen) wa = wk[k];
            c0 = wa < 0 ? 0 : wa;
            int wb = -1, wc = -1;
#pragma unroll
            for (int k = 0; k < NCOL; ++k) {
                const int w = wk[k];
                if (w < 0 || w == wa || w == wb || w == wc) continue;
                if (wb < 0) wb = w;
                else if (wc < 0) wc = w;
                else fail = true;
            }
            selA = 0;
            selB = 0;
#pragma unroll
            for (int k = 0; k < NCOL; ++k) {
                const int w = wk[k], p = idx[k] & 3;
                const unsigned na = (w >= 0 && w == wb) ? 4u + p : (w >= 0 && w == wa) ? (unsigned)p : 0u;
                const unsigned nb = (w >= 0 && w == wc && w != wa && w != wb) ? 4u + p : (unsigned)k;
                selA |= na << (4 * k);
                selB |= nb << (4 * k);
            }
            if (wb >= 0) {
                c1 = wb;
                n1 = min(4, rowlen - wb);
            }
            if (wc >= 0) {
                c2 = wc;
                n2 = min(4, rowlen - wc);
            }
            extra = selA != 0x3210u || selB != 0x3210u;
        } else {
            // float: each sample is its own word, both from the shared ring
            extra = true;
            c1 = max(idx[0], 0);
            n1 = idx[0] >= 0 ? 4 : 0;
            c2 = max(idx[1], 0);
            n2 = idx[1] >= 0 ? 4 : 0;
        }
    }
    const bool wbytes = __any_sync(0xffffffffu, fail);
    const bool wextra = !wbytes && __any_sync(0xffffffffu, extra);
#pragma unroll
    for (int k = 0; k < NCOL; ++k) idx[k] = max(idx[k], 0);
    unsigned* xring = reinterpret_cast<unsigned*>(reinterpret_cast<char*>(vbuf) + G::PLANES_BYTES) + tid;
    const unsigned char* cbase = static_cast<const unsigned char*>(a.src) + (size_t)c0 * sizeof(Tin);
    // Shared offset of each column in band row 0; a lane without that column
    // stores into the padding column (never read as a window value).
    int vdst[NCOL];
#pragma unroll
    for (int k = 0; k < NCOL; ++k) {
        const int s = s0 + k;
        vdst[k] = (active && s >= 0 && s < G::IW) ? (s % C) * G::PLANE + s / C : G::VW;
    }

    f2p acc[K][NP];
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int q = 0; q < NP; ++q) acc[j][q] = 0ull;

    const int T = nrows + K - 1;                   // source rows walked
    const int ybase = r0 - K / 2;                  // image row of source row 0
    int band_start = r0;                           // image row of band row 0
    // Output i (source row t = K-1+i, ring step u = t mod K) goes to band row
    // i mod TB = (u + 1) mod K: TB = K, so every store offset is a
    // compile-time constant, and band m is full at step u = K-2, t = (m+2)K-2.
    static_assert(G::TB == K, "band rows follow the ring");

    // ------------------------------------------------------------- column pass
    // The raw samples of the next K rows, loaded K rows ahead of use.
    using Raw = typename std::conditional<sizeof(Tin) == 1, unsigned, uint2>::type;
    Raw raw[K];
    // Rows past the last one walked are not loaded (a CTA-uniform test); rows
    // outside the image resolve out of line, Constant rows to row 0 (their
    // samples are replaced by the border value below).  `slot` is the ring
    // position (t mod K), a compile-time constant at every call.
    auto fetch = [&](int t, int slot) -> Raw {
        Raw r{};
        if (t < T) {
            // row address: one 32 x 32 -> 64-bit multiply-add onto the lane's
            // own base (pitches are below 2^31)
            const unsigned sy = (unsigned)row_any(ybase + t, a.H, a.border);
            if (!wbytes) {
                const unsigned char* p = cbase + (unsigned long long)sy * (unsigned)a.spitch;
                if constexpr (sizeof(Tin) == 1) {
                    r = __ldg(reinterpret_cast<const unsigned*>(p));
                } else {
                    const float2 v = __ldg(reinterpret_cast<const float2*>(p));
                    r = make_uint2(__float_as_uint(v.x), __float_as_uint(v.y));
                }
            }
            const Tin* srow = reinterpret_cast<const Tin*>(static_cast<const unsigned char*>(a.src) +
                                                           (unsigned long long)sy * (unsigned)a.spitch);
            if (!wbytes) {
                if (wextra) {
                    cp_async4(xring + (2 * slot) * kFastThreads, srow + c1, n1);
                    cp_async4(xring + (2 * slot + 1) * kFastThreads, srow + c2, n2);
                }
            } else if constexpr (sizeof(Tin) == 1) {
#pragma unroll
                for (int k = 0; k < NCOL; ++k) r |= (unsigned)__ldg(srow + idx[k]) << (8 * k);
            } else {
                r = make_uint2(__float_as_uint(__ldg(srow + idx[0])), __float_as_uint(__ldg(srow + idx[1])));
            }
        }
        if (wextra) cp_async_commit();
        return r;
    };
    static_for<0, K>([&](auto U) { raw[decltype(U)::value] = fetch(decltype(U)::value, decltype(U)::value); });
    const f2p mbias = pk2(-8388608.0f, -8388608.0f);
    const bool cfix = a.border == IPFC_BORDER_CONSTANT;  // Constant rows / columns take the border value

    for (int tb = 0; tb < T; tb += K) {
        static_for<0, K>([&](auto U) {
            constexpr int u = decltype(U)::value;
            const int t = tb + u;
            if (t < T) {
                f2p x[NP];
                Raw v = raw[u];
                if (wextra) {  // this row's copies: the oldest of the K groups in flight
                    cp_async_wait<K - 1>();
                    const unsigned w1 = xring[(2 * u) * kFastThreads], w2 = xring[(2 * u + 1) * kFastThreads];
                    if constexpr (sizeof(Tin) == 1) v = __byte_perm(__byte_perm(v, w1, selA), w2, selB);
                    else if (extra) v = make_uint2(w1, w2);
                }
                if constexpr (sizeof(Tin) == 1) {
                    // byte k -> 2^23 + byte (PRMT into the mantissa), then one packed add
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        const unsigned f0 = __byte_perm(v, 0x4B000000u, 0x7440 | (2 * q));
                        const unsigned f1 = __byte_perm(v, 0x4B000000u, 0x7440 | (2 * q + 1));
                        x[q] = fadd2p(((f2p)f1 << 32) | f0, mbias);
                    }
                } else {
                    x[0] = ((f2p)v.y << 32) | v.x;
                }
                raw[u] = fetch(t + K, u);
                if (cfix) {
                    const bool const_row = (unsigned)(ybase + t) >= (unsigned)a.H;
                    if (const_row || cmask) {
#pragma unroll
                        for (int q = 0; q < NP; ++q) {
                            float2 v = upk2(x[q]);
                            if (const_row || ((cmask >> (2 * q)) & 1u)) v.x = a.bv;
                            if (const_row || ((cmask >> (2 * q + 1)) & 1u)) v.y = a.bv;
                            x[q] = pk2(v.x, v.y);
                        }
                    }
                }
                // source row t feeds output o = t - j with tap j (ring slot (u - j) mod K)
                static_for<0, K>([&](auto J) {
                    constexpr int j = decltype(J)::value;
                    constexpr int slot = (u - j + K) % K;
#pragma unroll
                    for (int q = 0; q < NP; ++q) acc[slot][q] = ffma2p(a.ky2[j], x[q], acc[slot][q]);
                });
                constexpr int done = (u + 1) % K;  // slot of output t - (K - 1), and its band row
                if (t >= K - 1) {
                    constexpr int off = done * G::VWP;
#pragma unroll
                    for (int q = 0; q < NP; ++q) {
                        vbuf[vdst[2 * q] + off] = lo_f(acc[done][q]);
                        vbuf[vdst[2 * q + 1] + off] = hi_f(acc[done][q]);
                    }
                }
#pragma unroll
                for (int q = 0; q < NP; ++q) acc[done][q] = 0ull;
                if constexpr (u == K - 2) {
                    if (t >= 2 * K - 2) {
                        sep_row_pass<K, C, Tout, G>(a, vbuf, G::TB, band_start, x0);
                        band_start += G::TB;
                    }
                }
            }
        });
    }
    const int rem = nrows % G::TB;  // outputs of the last, partial band
    if (rem > 0) sep_row_pass_cold<K, C, Tout, G>(a, vbuf, rem, band_start, x0);
}

// ---- the kernel: one tile per CTA --------------------------------------------
template <int K, int C, typename Tin, typename Tout>
__global__ void __launch_bounds__(kFastThreads, (K <= kFastTwoCtaTaps ? 2 : 1))
    sep_fast_kernel(const __grid_constant__ SepFastArgs a) {
    extern __shared__ __align__(128) float vbuf[];  // C planes x TB rows x VWP
    sep_fast_tile<K, C, Tin, Tout>(a, vbuf, blockIdx.x % a.strips, blockIdx.x / a.strips);
}

}  // namespace ipfc
