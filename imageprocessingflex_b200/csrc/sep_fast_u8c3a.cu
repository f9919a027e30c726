// uint8 -> uint8 instantiations of the fast separable kernel: 3 channel(s), K = 3 .. 13.
#include "sep_fast_launch.cuh"

namespace ipfc {

bool sep_fast_u8c3a(int K, int C, int sdt, int ddt, const SepFastArgs& a, cudaStream_t s, cudaError_t* err) {
    if (sdt != IPFC_U8 || ddt != IPFC_U8 || C != 3) return false;
    switch (K) {
        case 3: *err = launch_sep_fast<3, 3, uint8_t, uint8_t>(a, s); return true;
        case 5: *err = launch_sep_fast<5, 3, uint8_t, uint8_t>(a, s); return true;
        case 7: *err = launch_sep_fast<7, 3, uint8_t, uint8_t>(a, s); return true;
        case 9: *err = launch_sep_fast<9, 3, uint8_t, uint8_t>(a, s); return true;
        case 11: *err = launch_sep_fast<11, 3, uint8_t, uint8_t>(a, s); return true;
        case 13: *err = launch_sep_fast<13, 3, uint8_t, uint8_t>(a, s); return true;
        default: return false;
    }
}

}  // namespace ipfc
