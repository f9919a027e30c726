// Host check of the kernels' store rounding (sat_from_f in common.cuh,
// compiled here for the host from the same source) against the oracle's
// restatement of ipf's saturate_cast (orc_saturate, after
// include/ipf/core.hpp:69-103): round half away from zero, clamp to the
// type's range, NaN -> 0.
//
// Every one of the 2^32 float bit patterns (NaNs, infinities, subnormals and
// both zeros included) is converted to uint8, uint16 and int16 and compared.
// Prints "ok <cases checked>" and exits 0, or prints the first failures and
// exits 1.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "common.cuh"

extern "C" double orc_saturate(double v, int dt);

namespace {
constexpr int kU8 = 0, kU16 = 1, kI16 = 2;  // the oracle's element codes

float from_bits(uint32_t b) {
    float f;
    std::memcpy(&f, &b, sizeof f);
    return f;
}
}  // namespace

int main() {
    long long bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (long long i = 0; i < (1ll << 32); ++i) {
        const float v = from_bits((uint32_t)i);
        const double d = (double)v;
        const int u8 = ipfc::sat_from_f<uint8_t>(v), u16 = ipfc::sat_from_f<uint16_t>(v),
                  i16 = ipfc::sat_from_f<int16_t>(v);
        const bool ok = u8 == (int)orc_saturate(d, kU8) && u16 == (int)orc_saturate(d, kU16) &&
                        i16 == (int)orc_saturate(d, kI16);
        if (!ok) {
            ++bad;
            if (bad < 5) std::printf("bits %08llx (%.9g): u8 %d u16 %d i16 %d\n", i, (double)v, u8, u16, i16);
        }
    }
    if (bad) {
        std::printf("FAILED %lld\n", bad);
        return 1;
    }
    std::printf("ok %lld\n", 3 * (1ll << 32));
    return 0;
}
