// Single-channel float32 -> float32 instantiations of the fast separable kernel, K = 19 .. 31.
#include "sep_fast_launch.cuh"

namespace ipfc {

bool sep_fast_miscb(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err) {
    if (C != 1 || sdt != IPFC_F32 || ddt != IPFC_F32) return false;
    switch (K) {
        case 19: *err = launch_sep_fast<19, 1, float, float>(a, s); return true;
        case 21: *err = launch_sep_fast<21, 1, float, float>(a, s); return true;
        case 23: *err = launch_sep_fast<23, 1, float, float>(a, s); return true;
        case 25: *err = launch_sep_fast<25, 1, float, float>(a, s); return true;
        case 27: *err = launch_sep_fast<27, 1, float, float>(a, s); return true;
        case 29: *err = launch_sep_fast<29, 1, float, float>(a, s); return true;
        case 31: *err = launch_sep_fast<31, 1, float, float>(a, s); return true;
        default: return false;
    }
}

}  // namespace ipfc
