// Shared device-side pieces of the sm_100a BCn kernels: BPTC tables, the
// integer/bit helpers of the reference encoder (src/encode/common.rs), and
// the float conventions every kernel relies on.
//
// Bit-exactness with the reference CPU encoder rests on three build rules
// (set in build.py): --fmad=false (no FMA contraction), IEEE division and
// square root (-prec-div=true -prec-sqrt=true), no fast-math. Under them
// every f32 operation rounds exactly as the Rust code's does, as long as the
// kernels keep the reference's operation order, which they do in every sum
// that feeds a decision.
//
// Conversions: CUDA's float->int cast (cvt.rzi) saturates and maps NaN to 0,
// the same as Rust's `as i32` / `as u32`; fminf/fmaxf are IEEE minNum/maxNum
// like Rust's f32::min/max.
#pragma once
#include <cstdint>

namespace bcn {

#define BCN_DEV __device__ __forceinline__

// Rust f32::clamp: `if x < lo { x = lo } if x > hi { x = hi }` (NaN passes).
BCN_DEV float clampf_r(float x, float lo, float hi) {
    x = x < lo ? lo : x;
    x = x > hi ? hi : x;
    return x;
}
// Byte k of w as a float, without an int->float conversion: the byte is
// placed in the mantissa of 2^23 (0x4B0000bb) and 2^23 subtracted, which is
// exact for 0..255.
BCN_DEV float byte_to_float(uint32_t w, int k) {
    return __int_as_float((int)__byte_perm(w, 0x4B000000u, 0x7540u | (uint32_t)k)) - 8388608.0f;
}

// x / D for the constant divisors D = 31, 255 and 65535 of the encoders'
// scale conversions: q = RN(x * RN(1/D)) and one correction step
// q + RN(x - q * D) * RN(1/D) with fused multiply-adds (Markstein's
// correction, IBM J. Res. Develop. 34(1), 1990). Equal to the IEEE x / D for
// every finite float x except x = -0, which gives +0 (checked exhaustively by
// the oracle test over all 2^32 bit patterns). Every caller scales the
// quotient and adds a non-zero constant before rounding to an integer, so the
// sign of a zero quotient does not matter; no caller passes an infinity.
template <int D>
BCN_DEV float div_const(float x) {
    static_assert(D == 31 || D == 255 || D == 65535, "divisor not covered by the exhaustive check");
    constexpr float d = (float)D;
    const float r = 1.0f / d;
    float q = x * r;
    return fmaf(fmaf(-q, d, x), r, q);
}

BCN_DEV int clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }
BCN_DEV float sqf(float x) { return x * x; }

// ---- BPTC partition tables ---------------------------------------------------
// Subset map of the 64 two-subset (0..63) and 64 three-subset (64..127)
// partitions, 2 bits per pixel, pixel k at bits 2k..2k+1. Format constants
// of the BPTC specification, in the packed form of src/encode/common.rs:23-47.
#define BCN_PARTITION_MAP_VALUES \
    0x50505050, 0x40404040, 0x54545454, 0x54505040, 0x50404000, 0x55545450, 0x55545040, 0x54504000, \
    0x50400000, 0x55555450, 0x55544000, 0x54400000, 0x55555440, 0x55550000, 0x55555500, 0x55000000, \
    0x55150100, 0x00004054, 0x15010000, 0x00405054, 0x00004050, 0x15050100, 0x05010000, 0x40505054, \
    0x00404050, 0x05010100, 0x14141414, 0x05141450, 0x01155440, 0x00555500, 0x15014054, 0x05414150, \
    0x44444444, 0x55005500, 0x11441144, 0x05055050, 0x05500550, 0x11114444, 0x41144114, 0x44111144, \
    0x15055054, 0x01055040, 0x05041050, 0x05455150, 0x14414114, 0x50050550, 0x41411414, 0x00141400, \
    0x00041504, 0x00105410, 0x10541000, 0x04150400, 0x50410514, 0x41051450, 0x05415014, 0x14054150, \
    0x41050514, 0x41505014, 0x40011554, 0x54150140, 0x50505500, 0x00555050, 0x15151010, 0x54540404, \
    0xAA685050, 0x6A5A5040, 0x5A5A4200, 0x5450A0A8, 0xA5A50000, 0xA0A05050, 0x5555A0A0, 0x5A5A5050, \
    0xAA550000, 0xAA555500, 0xAAAA5500, 0x90909090, 0x94949494, 0xA4A4A4A4, 0xA9A59450, 0x2A0A4250, \
    0xA5945040, 0x0A425054, 0xA5A5A500, 0x55A0A0A0, 0xA8A85454, 0x6A6A4040, 0xA4A45000, 0x1A1A0500, \
    0x0050A4A4, 0xAAA59090, 0x14696914, 0x69691400, 0xA08585A0, 0xAA821414, 0x50A4A450, 0x6A5A0200, \
    0xA9A58000, 0x5090A0A8, 0xA8A09050, 0x24242424, 0x00AA5500, 0x24924924, 0x24499224, 0x50A50A50, \
    0x500AA550, 0xAAAA4444, 0x66660000, 0xA5A0A5A0, 0x50A050A0, 0x69286928, 0x44AAAA44, 0x66666600, \
    0xAA444444, 0x54A854A8, 0x95809580, 0x96969600, 0xA85454A8, 0x80959580, 0xAA141414, 0x96960000, \
    0xAAAA1414, 0xA05050A0, 0xA0A5A5A0, 0x96000000, 0x40804080, 0xA9A8A9A8, 0xAAAAAA44, 0x2A4A5254,
__constant__ __device__ const uint32_t kPartitionMap[128] = {BCN_PARTITION_MAP_VALUES};

// Anchor pixels of subsets 1 and 2 (high / low nibble) per partition
// (src/encode/common.rs:85-101; subset 0's anchor is always pixel 0).
#define BCN_ANCHOR_VALUES \
    0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, \
    0xF0, 0x20, 0x80, 0x20, 0x20, 0x80, 0x80, 0xF0, 0x20, 0x80, 0x20, 0x20, 0x80, 0x80, 0x20, 0x20, \
    0xF0, 0xF0, 0x60, 0x80, 0x20, 0x80, 0xF0, 0xF0, 0x20, 0x80, 0x20, 0x20, 0x20, 0xF0, 0xF0, 0x60, \
    0x60, 0x20, 0x60, 0x80, 0xF0, 0xF0, 0x20, 0x20, 0xF0, 0xF0, 0xF0, 0xF0, 0xF0, 0x20, 0x20, 0xF0, \
    0x3F, 0x38, 0xF8, 0xF3, 0x8F, 0x3F, 0xF3, 0xF8, 0x8F, 0x8F, 0x6F, 0x6F, 0x6F, 0x5F, 0x3F, 0x38, \
    0x3F, 0x38, 0x8F, 0xF3, 0x3F, 0x38, 0x6F, 0xA8, 0x53, 0x8F, 0x86, 0x6A, 0x8F, 0x5F, 0xFA, 0xF8, \
    0x8F, 0xF3, 0x3F, 0x5A, 0x6A, 0xA8, 0x89, 0xFA, 0xF6, 0x3F, 0xF8, 0x5F, 0xF3, 0xF6, 0xF6, 0xF8, \
    0x3F, 0xF3, 0x5F, 0x5F, 0x5F, 0x8F, 0x5F, 0xAF, 0x5F, 0xAF, 0x8F, 0xDF, 0xF3, 0xCF, 0x3F, 0x38,
__constant__ __device__ const uint8_t kAnchors[128] = {BCN_ANCHOR_VALUES};

// Host/device-constexpr derivation of the per-subset pixel mask from the
// subset map (bit k set when pixel k belongs to `subset`). It equals the
// reference's packed mask table (src/encode/common.rs:49-83) for subsets 0
// and 1; for subset 2 the reference returns `!mask0 & !mask1` whose low 16
// bits are the same set (only the low 16 bits are ever consumed).
//
// Bit-parallel form: a 2-bit field equals `subset` exactly when both bits of
// ~(map ^ subset replicated into every field) are set; the 16 field flags
// (bits 0, 2, ..., 30) are then gathered into bits 0..15 by the usual
// halving compress (checked against the per-field definition for every
// field value, position and subset, and on random maps, by the CPU tests).
__host__ __device__ __forceinline__ uint32_t subset_mask_from_map(uint32_t map, uint32_t subset) {
    uint32_t x = ~(map ^ (subset * 0x55555555u));
    x &= (x >> 1) & 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0F0F0F0Fu;
    x = (x | (x >> 4)) & 0x00FF00FFu;
    return (x | (x >> 8)) & 0x0000FFFFu;
}

// Reference semantics of get_pattern_mask(part_id, j) for the bits the
// encoder uses (pixel masks and flip masks only ever read bits 0..15).
BCN_DEV uint32_t pattern_mask(const uint32_t* map_table, int part_id, uint32_t j) {
    return subset_mask_from_map(map_table[part_id], j);
}

// Index weights of the BPTC interpolation (common.rs:6-21).
BCN_DEV int unquant_weight(uint32_t bits, int index) {
    // Packed 4-bit-per-entry would cost shifts; small switch tables are cheaper
    // as immediates.
    if (bits == 2) {
        const int w[4] = {0, 21, 43, 64};
        return w[index & 3];
    }
    if (bits == 3) {
        const int w[8] = {0, 9, 18, 27, 37, 46, 55, 64};
        return w[index & 7];
    }
    const int w[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};
    return w[index & 15];
}

// 128-bit block writer (common.rs:103-109), five words like the reference so
// the anchor-bit removal shifts (common.rs:111-124) see the same overflow word.
struct BitWriter {
    uint32_t d[5];
    uint32_t pos;
    BCN_DEV void clear() {
        d[0] = d[1] = d[2] = d[3] = d[4] = 0;
        pos = 0;
    }
    BCN_DEV void put(uint32_t bits, uint32_t v) {
        uint32_t w = pos >> 5, s = pos & 31;
        // Unrolled selects keep d[] in registers (no dynamic indexing).
#pragma unroll
        for (int i = 0; i < 5; i++) {
            if (i == (int)w) d[i] |= v << s;
            if (s + bits > 32 && i == (int)w + 1) d[i] |= v >> (32 - s);
        }
        pos += bits;
    }
};

// common.rs:111-124
BCN_DEV void data_shl_1bit_from(uint32_t d[5], uint32_t from_bits) {
    if (from_bits < 96) {
        uint32_t shifted = (d[2] >> 1) | (d[3] << 31);
        uint32_t mask = ((1u << (from_bits - 64)) - 1) >> 1;
        d[2] = (mask & d[2]) | (~mask & shifted);
        d[3] = (d[3] >> 1) | (d[4] << 31);
        d[4] >>= 1;
    } else if (from_bits < 128) {
        uint32_t shifted = (d[3] >> 1) | (d[4] << 31);
        uint32_t mask = ((1u << (from_bits - 96)) - 1) >> 1;
        d[3] = (mask & d[3]) | (~mask & shifted);
        d[4] >>= 1;
    }
}

// common.rs:520-547: index bits with the first index one bit short.
BCN_DEV void code_qblock(BitWriter& bw, uint32_t q0, uint32_t q1, uint32_t bits, uint32_t flips) {
    uint32_t levels = 1u << bits;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t q = ((k < 8 ? q0 : q1) >> (4 * (k & 7))) & 15;
        if ((flips >> k) & 1) q = (levels - 1) - q;
        bw.put(k == 0 ? bits - 1 : bits, q);
    }
}

// common.rs:549-562
BCN_DEV void adjust_skip_mode01237(uint32_t d[5], uint32_t mode, int part_id) {
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t packed = kAnchors[part_id];
    uint32_t s1 = packed >> 4, s2 = packed & 15;
    if (pairs > 2 && s1 < s2) {
        uint32_t t = s1;
        s1 = s2;
        s2 = t;
    }
    data_shl_1bit_from(d, 128 + (pairs - 1) - (15 - s1) * bits);
    if (pairs > 2) data_shl_1bit_from(d, 128 + (pairs - 1) - (15 - s2) * bits);
}

// common.rs:564-581 (qep is endpoint pair layout [ch0..ch3 of e0 | e1])
BCN_DEV void apply_swap_mode456(int* qep, uint32_t channels, uint32_t& q0, uint32_t& q1, uint32_t bits) {
    uint32_t levels = 1u << bits;
    if ((q0 & 15) >= levels / 2) {
        for (uint32_t p = 0; p < channels; p++) {
            int t = qep[p];
            qep[p] = qep[channels + p];
            qep[channels + p] = t;
        }
        q0 = 0x11111111u * (levels - 1) - q0;
        q1 = 0x11111111u * (levels - 1) - q1;
    }
}

// common.rs:583-613
BCN_DEV uint32_t apply_swap_mode01237(int qep[24], uint32_t q0, uint32_t q1, uint32_t mode, int part_id) {
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t levels = 1u << bits;
    uint32_t packed = kAnchors[part_id];
    uint32_t map = kPartitionMap[part_id];
    uint32_t flips = 0;
    for (uint32_t j = 0; j < pairs; j++) {
        uint32_t k0 = j == 0 ? 0 : (j == 1 ? (packed >> 4) : (packed & 15));
        uint32_t q = ((k0 < 8 ? q0 : q1) >> (4 * (k0 & 7))) & 15;
        if (q >= levels / 2) {
            for (int p = 0; p < 4; p++) {
                int t = qep[8 * j + p];
                qep[8 * j + p] = qep[8 * j + 4 + p];
                qep[8 * j + 4 + p] = t;
            }
            flips |= subset_mask_from_map(map, j);
        }
    }
    return flips;
}

}  // namespace bcn
