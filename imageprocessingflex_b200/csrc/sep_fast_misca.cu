// Single-channel instantiations of the fast separable kernel: uint8 -> int16 / float32 for K = 3, 5 (Sobel), float32 -> float32 for K = 3 .. 17.
#include "sep_fast_launch.cuh"

namespace ipfc {

bool sep_fast_misca(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err) {
    if (C != 1) return false;
    if (sdt == IPFC_U8 && ddt == IPFC_I16) {
        if (K == 3) { *err = launch_sep_fast<3, 1, uint8_t, int16_t>(a, s); return true; }
        if (K == 5) { *err = launch_sep_fast<5, 1, uint8_t, int16_t>(a, s); return true; }
        return false;
    }
    if (sdt == IPFC_U8 && ddt == IPFC_F32) {
        if (K == 3) { *err = launch_sep_fast<3, 1, uint8_t, float>(a, s); return true; }
        if (K == 5) { *err = launch_sep_fast<5, 1, uint8_t, float>(a, s); return true; }
        return false;
    }
    if (sdt != IPFC_F32 || ddt != IPFC_F32) return false;
    switch (K) {
        case 3: *err = launch_sep_fast<3, 1, float, float>(a, s); return true;
        case 5: *err = launch_sep_fast<5, 1, float, float>(a, s); return true;
        case 7: *err = launch_sep_fast<7, 1, float, float>(a, s); return true;
        case 9: *err = launch_sep_fast<9, 1, float, float>(a, s); return true;
        case 11: *err = launch_sep_fast<11, 1, float, float>(a, s); return true;
        case 13: *err = launch_sep_fast<13, 1, float, float>(a, s); return true;
        case 15: *err = launch_sep_fast<15, 1, float, float>(a, s); return true;
        case 17: *err = launch_sep_fast<17, 1, float, float>(a, s); return true;
        default: return false;
    }
}

}  // namespace ipfc
