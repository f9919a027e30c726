// seeded.cpp -- seeded test-image generator (TEST INFRASTRUCTURE ONLY).
//
// Reproduces the sample stream of the reference test helper randomImage()
// (tests/test_util.hpp:13-24): one std::mt19937(seed) engine, one draw per
// sample in memory order, std::uniform_int_distribution<long long>(0, max)
// for integer types and std::uniform_real_distribution<double>(0, 1) cast to
// the element type for floating types.  Uses only the C++ standard library,
// so its stream equals the reference's on the same libstdc++.
#include <cstddef>
#include <cstdint>
#include <random>

extern "C" {

// dt: 0 u8, 1 u16, 2 i16, 3 i32, 4 f32, 5 f64 (same codes as oracle.c).
// For i16 the reference's PixelTraits max is 32767; for i32 it is 255.
int orc_random_image(void* out, int dt, std::size_t n, unsigned seed) {
    std::mt19937 rng(seed);
    switch (dt) {
        case 0: {
            auto* p = static_cast<std::uint8_t*>(out);
            for (std::size_t i = 0; i < n; ++i)
                p[i] = static_cast<std::uint8_t>(std::uniform_int_distribution<long long>(0, 255)(rng));
            return 0;
        }
        case 1: {
            auto* p = static_cast<std::uint16_t*>(out);
            for (std::size_t i = 0; i < n; ++i)
                p[i] = static_cast<std::uint16_t>(std::uniform_int_distribution<long long>(0, 65535)(rng));
            return 0;
        }
        case 2: {
            auto* p = static_cast<std::int16_t*>(out);
            for (std::size_t i = 0; i < n; ++i)
                p[i] = static_cast<std::int16_t>(std::uniform_int_distribution<long long>(0, 32767)(rng));
            return 0;
        }
        case 3: {
            auto* p = static_cast<std::int32_t*>(out);
            for (std::size_t i = 0; i < n; ++i)
                p[i] = static_cast<std::int32_t>(std::uniform_int_distribution<long long>(0, 255)(rng));
            return 0;
        }
        case 4: {
            auto* p = static_cast<float*>(out);
            for (std::size_t i = 0; i < n; ++i)
                p[i] = static_cast<float>(std::uniform_real_distribution<double>(0.0, 1.0)(rng));
            return 0;
        }
        case 5: {
            auto* p = static_cast<double*>(out);
            for (std::size_t i = 0; i < n; ++i) p[i] = std::uniform_real_distribution<double>(0.0, 1.0)(rng);
            return 0;
        }
        default:
            return 1;
    }
}

}  // extern "C"
