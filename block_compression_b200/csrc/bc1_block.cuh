// BC1 colour-block primitives shared by the BC1-BC5 kernels (bc15.cu) and
// the endpoint-refinement kernels (refine.cu): the RGB565 conversions of the
// encoder (src/encode/bc1_to_5.rs:258-278) and the bit-exact colour-block
// decoder (src/decode/block.rs:124-197).
#pragma once
#include "bc_common.cuh"

namespace bcn {

BCN_DEV void dec_rgb565(float c[3], int p) {
    int b5 = p & 31, g6 = (p >> 5) & 63, r5 = (p >> 11) & 31;
    c[0] = (float)((r5 << 3) + (r5 >> 2));
    c[1] = (float)((g6 << 2) + (g6 >> 4));
    c[2] = (float)((b5 << 3) + (b5 >> 2));
}

BCN_DEV int enc_rgb565(float c0, float c1, float c2) {
    int r = (int)c0, g = (int)c1, b = (int)c2;
    int r5 = (r * 31 + 128 + ((r * 31) >> 8)) >> 8;
    int g6 = (g * 63 + 128 + ((g * 63) >> 8)) >> 8;
    int b5 = (b * 31 + 128 + ((b * 31) >> 8)) >> 8;
    return (r5 << 11) + (g6 << 5) + b5;
}

// block.rs:124-197; opaque forces the four-colour mode (BC2/BC3 colour).
BCN_DEV void decode_color(uint32_t c01, uint32_t idx, bool opaque, uint32_t out[16]) {
    uint32_t c0 = c01 & 0xFFFF, c1 = c01 >> 16;
    uint32_t r0 = (c0 >> 11) & 0x1F, g0 = (c0 >> 5) & 0x3F, b0 = c0 & 0x1F;
    uint32_t r1 = (c1 >> 11) & 0x1F, g1 = (c1 >> 5) & 0x3F, b1 = c1 & 0x1F;
    uint32_t ref[4];
    ref[0] = 0xFF000000u | (((b0 * 527 + 23) >> 6) << 16) | (((g0 * 259 + 33) >> 6) << 8) | ((r0 * 527 + 23) >> 6);
    ref[1] = 0xFF000000u | (((b1 * 527 + 23) >> 6) << 16) | (((g1 * 259 + 33) >> 6) << 8) | ((r1 * 527 + 23) >> 6);
    if (c0 > c1 || opaque) {
        ref[2] = 0xFF000000u | ((((2 * b0 + b1) * 351 + 61) >> 7) << 16) | ((((2 * g0 + g1) * 2763 + 1039) >> 11) << 8) |
                 (((2 * r0 + r1) * 351 + 61) >> 7);
        ref[3] = 0xFF000000u | ((((b0 + 2 * b1) * 351 + 61) >> 7) << 16) | ((((g0 + 2 * g1) * 2763 + 1039) >> 11) << 8) |
                 (((r0 + 2 * r1) * 351 + 61) >> 7);
    } else {
        ref[2] = 0xFF000000u | ((((b0 + b1) * 1053 + 125) >> 8) << 16) | ((((g0 + g1) * 4145 + 1019) >> 11) << 8) |
                 (((r0 + r1) * 1053 + 125) >> 8);
        ref[3] = 0;
    }
#pragma unroll
    for (int k = 0; k < 16; k++) out[k] = ref[(idx >> (2 * k)) & 3];
}

}  // namespace bcn
