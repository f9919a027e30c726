// uint8 -> uint8 instantiations of the fast separable kernel: 1 channel(s), K = 3 .. 13.
#include "sep_fast_launch.cuh"

namespace ipfc {

bool sep_fast_u8c1a(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err) {
    if (sdt != IPFC_U8 || ddt != IPFC_U8 || C != 1) return false;
    switch (K) {
        case 3: *err = launch_sep_fast<3, 1, uint8_t, uint8_t>(a, s); return true;
        case 5: *err = launch_sep_fast<5, 1, uint8_t, uint8_t>(a, s); return true;
        case 7: *err = launch_sep_fast<7, 1, uint8_t, uint8_t>(a, s); return true;
        case 9: *err = launch_sep_fast<9, 1, uint8_t, uint8_t>(a, s); return true;
        case 11: *err = launch_sep_fast<11, 1, uint8_t, uint8_t>(a, s); return true;
        case 13: *err = launch_sep_fast<13, 1, uint8_t, uint8_t>(a, s); return true;
        default: return false;
    }
}

}  // namespace ipfc
