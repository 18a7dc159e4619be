// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Exhaustive check of the division shortcut the BC7 kernels use for the
// statistics' divisions by a pixel count (bptc_math.cuh, div_count): for an
// integer-valued x in [0, 2^24] and n in [1, 16], with r = RN(1 / n),
// RN(fma(RN(x - q*n), r, q)), q = RN(x * r), must equal the IEEE x / n.
#include <cmath>
#include <cstdint>
#include <cstring>

extern "C" uint64_t oracle_check_div_count(void) {
    uint64_t bad = 0;
    for (int n = 1; n <= 16; n++) {
        const float fn = (float)n;
        const float r = 1.0f / fn;
        for (uint32_t i = 0; i <= (1u << 24); i++) {
            const float x = (float)i;
            float q = x * r;
            float fast = std::fma(std::fma(-q, fn, x), r, q);
            float ieee = x / fn;
            uint32_t a, b;
            std::memcpy(&a, &fast, 4);
            std::memcpy(&b, &ieee, 4);
            bad += a != b;
        }
    }
    return bad;
}
