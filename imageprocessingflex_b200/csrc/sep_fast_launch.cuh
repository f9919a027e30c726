// sep_fast_launch.cuh -- launch geometry of sep_fast_kernel and the table of
// instantiated (K, C, source, destination) combinations.
#pragma once

#include "sep_fast.cuh"
#include "sep_filter.cuh"

namespace ipfc {

// Launches one instantiation: strips of PX pixels across, and as many row
// chunks as fill one wave of resident CTAs (so the grid has no tail wave).
template <int K, int C, typename Tin, typename Tout>
cudaError_t launch_sep_fast(const SepFastArgs& in, cudaStream_t s) {
    using G = FastGeom<K, C, (sizeof(Tin) == 1 ? 4 : 2)>;
    auto kern = sep_fast_kernel<K, C, Tin, Tout>;
    static unsigned smem_done = 0;
    cudaError_t e = ensure_smem_attr((const void*)kern, (int)G::SMEM, &smem_done);
    if (e != cudaSuccess) return e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    // Resident CTAs per SM, cached per device (devices past the table are
    // queried every call).  Racing threads store the same value.
    static int occ_cache[32] = {0};
    const bool cached = dev >= 0 && dev < 32;
    int occ = cached ? __atomic_load_n(&occ_cache[dev], __ATOMIC_ACQUIRE) : 0;
    if (occ == 0) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kFastThreads, G::SMEM);
        if (e != cudaSuccess) return e;
        occ = occ > 0 ? occ : 1;
        if (cached) __atomic_store_n(&occ_cache[dev], occ, __ATOMIC_RELEASE);
    }
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    SepFastArgs a = in;
    a.strips = (a.W + G::PX - 1) / G::PX;
    const int slots = sms * occ;
    int chunks = slots / a.strips;
    if (chunks < 1) chunks = 1;
    a.rows_per_cta = (a.H + chunks - 1) / chunks;
    chunks = (a.H + a.rows_per_cta - 1) / a.rows_per_cta;
    kern<<<a.strips * chunks, kFastThreads, G::SMEM, s>>>(a);
    return cudaGetLastError();
}

// Each instantiation file provides one of these; it returns false when the
// combination is not its own.
bool sep_fast_u8c1a(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_u8c1b(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_u8c3a(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_u8c3b(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_u8c4a(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_u8c4b(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_misca(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);
bool sep_fast_miscb(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err);

// Tries every instantiation file; true when one of them launched.
inline bool sep_fast_dispatch(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s,
                              cudaError_t* err) {
    return sep_fast_u8c1a(K, C, sdt, ddt, a, s, err) ||
           sep_fast_u8c1b(K, C, sdt, ddt, a, s, err) ||
           sep_fast_u8c3a(K, C, sdt, ddt, a, s, err) ||
           sep_fast_u8c3b(K, C, sdt, ddt, a, s, err) ||
           sep_fast_u8c4a(K, C, sdt, ddt, a, s, err) ||
           sep_fast_u8c4b(K, C, sdt, ddt, a, s, err) ||
           sep_fast_misca(K, C, sdt, ddt, a, s, err) ||
           sep_fast_miscb(K, C, sdt, ddt, a, s, err);
}

}  // namespace ipfc
