// uint8 -> uint8 instantiations of the fast separable kernel: 1 channel(s), K = 15 .. 25.
#include "sep_fast_launch.cuh"

namespace ipfc {

bool sep_fast_u8c1b(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err) {
    if (sdt != IPFC_U8 || ddt != IPFC_U8 || C != 1) return false;
    switch (K) {
        case 15: *err = launch_sep_fast<15, 1, uint8_t, uint8_t>(a, s); return true;
        case 17: *err = launch_sep_fast<17, 1, uint8_t, uint8_t>(a, s); return true;
        case 19: *err = launch_sep_fast<19, 1, uint8_t, uint8_t>(a, s); return true;
        case 21: *err = launch_sep_fast<21, 1, uint8_t, uint8_t>(a, s); return true;
        case 23: *err = launch_sep_fast<23, 1, uint8_t, uint8_t>(a, s); return true;
        case 25: *err = launch_sep_fast<25, 1, uint8_t, uint8_t>(a, s); return true;
        default: return false;
    }
}

}  // namespace ipfc
