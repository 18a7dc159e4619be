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

// The same shortcut for the constant divisors of the encoders' scale
// conversions (bc_common.cuh, div_const): x / d for d in {31, 255, 65535} and
// every finite float x, in parallel over the 2^32 bit patterns. The only
// accepted difference is x = -0, where the shortcut gives +0. Returns the
// number of other mismatches.
#include <thread>
#include <vector>

extern "C" uint64_t oracle_check_div_const(float d, int threads) {
    if (threads < 1) threads = 1;
    const float r = 1.0f / d;
    std::vector<uint64_t> bad((size_t)threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([&, t] {
            const uint64_t lo = (1ull << 32) * (uint64_t)t / (uint64_t)threads;
            const uint64_t hi = (1ull << 32) * (uint64_t)(t + 1) / (uint64_t)threads;
            uint64_t b = 0;
            for (uint64_t u = lo; u < hi; u++) {
                uint32_t bits = (uint32_t)u;
                float x;
                std::memcpy(&x, &bits, 4);
                if (!std::isfinite(x) || bits == 0x80000000u) continue;
                float q = x * r;
                float fast = std::fma(std::fma(-q, d, x), r, q);
                float ieee = x / d;
                uint32_t a, c;
                std::memcpy(&a, &fast, 4);
                std::memcpy(&c, &ieee, 4);
                b += a != c;
            }
            bad[(size_t)t] = b;
        });
    }
    uint64_t total = 0;
    for (int t = 0; t < threads; t++) {
        pool[(size_t)t].join();
        total += bad[(size_t)t];
    }
    return total;
}

// The index fit's projection divides one integer by another (sums of
// products of 8-bit values: numerator magnitude <= 4 * 255 * 255, divisor in
// [1, 4 * 255 * 255]); the BC7 kernels do it with the divisor's reciprocal
// and one fused correction step (bptc_math.cuh, block_quant). Checked here
// for every positive numerator and divisor in that range; the steps are odd
// in x, so negative numerators follow, and a zero numerator gives +0 either
// way (the projection sum starts at +0 and is never -0).
extern "C" uint64_t oracle_check_div_int_pairs(int threads) {
    const int M = 4 * 255 * 255;
    if (threads < 1) threads = 1;
    std::vector<uint64_t> bad((size_t)threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++) {
        pool.emplace_back([&, t] {
            const int lo = 1 + (int)((int64_t)M * t / threads), hi = 1 + (int)((int64_t)M * (t + 1) / threads);
            uint64_t b = 0;
            for (int y = lo; y < hi; y++) {
                const float fy = (float)y, r = 1.0f / fy;
                for (int x = 1; x <= M; x++) {
                    const float fx = (float)x;
                    float q = fx * r;
                    float fast = std::fma(std::fma(-q, fy, fx), r, q);
                    b += fast != fx / fy;
                }
            }
            bad[(size_t)t] = b;
        });
    }
    uint64_t total = 0;
    for (int t = 0; t < threads; t++) {
        pool[(size_t)t].join();
        total += bad[(size_t)t];
    }
    return total;
}

// The mode-4/5 scalar-channel fit divides an 8-bit difference x in
// [-255, 255] by (d + 0.001), d an 8-bit difference in [-255, 255]
// (channel_opt_quant); the BC7 kernels use the reciprocal and one fused
// correction step. Every (x, d) pair is checked here.
extern "C" uint64_t oracle_check_div_channel(void) {
    uint64_t bad = 0;
    for (int d = -255; d <= 255; d++) {
        const float den = (float)d + 0.001f, r = 1.0f / den;
        for (int xi = -255; xi <= 255; xi++) {
            const float x = (float)xi;
            float q = x * r;
            float fast = std::fma(std::fma(-q, den, x), r, q);
            float ieee = x / den;
            uint32_t a, b;
            std::memcpy(&a, &fast, 4);
            std::memcpy(&b, &ieee, 4);
            bad += a != b;
        }
    }
    return bad;
}
