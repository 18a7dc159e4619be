// BC1-BC5 block primitives shared by the BC1-BC5 kernels (bc15.cu), the
// per-block decoders (bc_decode.cu) and the endpoint-refinement kernels
// (refine.cu): the RGB565 conversions of the encoder
// (src/encode/bc1_to_5.rs:258-278) and the bit-exact colour-block and
// smooth-alpha decoders (src/decode/block.rs:124-258).
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

// block.rs:221-258. The 8-entry palette is kept as 8 bytes in two registers
// and indexed with a byte permute (no local-memory array).
BCN_DEV void decode_smooth(uint32_t lo, uint32_t hi, uint32_t out[16]) {
    uint32_t a0 = lo & 0xFF, a1 = (lo >> 8) & 0xFF;
    uint32_t p_lo, p_hi;
    if (a0 > a1) {
        p_lo = a0 | (a1 << 8) | (((6 * a0 + a1) / 7) << 16) | (((5 * a0 + 2 * a1) / 7) << 24);
        p_hi = ((4 * a0 + 3 * a1) / 7) | (((3 * a0 + 4 * a1) / 7) << 8) | (((2 * a0 + 5 * a1) / 7) << 16) |
               (((a0 + 6 * a1) / 7) << 24);
    } else {
        p_lo = a0 | (a1 << 8) | (((4 * a0 + a1) / 5) << 16) | (((3 * a0 + 2 * a1) / 5) << 24);
        p_hi = ((2 * a0 + 3 * a1) / 5) | (((a0 + 4 * a1) / 5) << 8) | (0u << 16) | (255u << 24);
    }
    // 48 index bits: pixels 0-7 in the low 24, pixels 8-15 in the high 24
    uint32_t i0 = (lo >> 16) | ((hi & 0xFF) << 16), i1 = hi >> 8;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t sel = ((k < 8 ? i0 : i1) >> (3 * (k & 7))) & 7u;
        out[k] = __byte_perm(p_lo, p_hi, sel) & 0xFFu;
    }
}

}  // namespace bcn
