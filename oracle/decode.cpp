// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Restatement of the reference decoders: src/decode/block.rs (a port of
// bcdec.h v0.98) and the image drivers of src/decode.rs.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle_decode.h"

namespace oracle {

namespace {

// block.rs:124-197
void decode_color_block(const uint8_t* cb, uint8_t* out, size_t pitch, bool opaque_mode) {
    uint32_t ref[4];
    uint16_t c0 = (uint16_t)(cb[0] | (cb[1] << 8));
    uint16_t c1 = (uint16_t)(cb[2] | (cb[3] << 8));
    uint32_t r0 = (c0 >> 11) & 0x1F, g0 = (c0 >> 5) & 0x3F, b0 = c0 & 0x1F;
    uint32_t r1 = (c1 >> 11) & 0x1F, g1 = (c1 >> 5) & 0x3F, b1 = c1 & 0x1F;
    uint32_t r = (r0 * 527 + 23) >> 6, g = (g0 * 259 + 33) >> 6, b = (b0 * 527 + 23) >> 6;
    ref[0] = 0xFF000000u | (b << 16) | (g << 8) | r;
    r = (r1 * 527 + 23) >> 6;
    g = (g1 * 259 + 33) >> 6;
    b = (b1 * 527 + 23) >> 6;
    ref[1] = 0xFF000000u | (b << 16) | (g << 8) | r;
    if (c0 > c1 || opaque_mode) {
        r = ((2 * r0 + r1) * 351 + 61) >> 7;
        g = ((2 * g0 + g1) * 2763 + 1039) >> 11;
        b = ((2 * b0 + b1) * 351 + 61) >> 7;
        ref[2] = 0xFF000000u | (b << 16) | (g << 8) | r;
        r = ((r0 + r1 * 2) * 351 + 61) >> 7;
        g = ((g0 + g1 * 2) * 2763 + 1039) >> 11;
        b = ((b0 + b1 * 2) * 351 + 61) >> 7;
        ref[3] = 0xFF000000u | (b << 16) | (g << 8) | r;
    } else {
        r = ((r0 + r1) * 1053 + 125) >> 8;
        g = ((g0 + g1) * 4145 + 1019) >> 11;
        b = ((b0 + b1) * 1053 + 125) >> 8;
        ref[2] = 0xFF000000u | (b << 16) | (g << 8) | r;
        ref[3] = 0;
    }
    uint32_t idx = (uint32_t)cb[4] | ((uint32_t)cb[5] << 8) | ((uint32_t)cb[6] << 16) | ((uint32_t)cb[7] << 24);
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            uint32_t color = ref[idx & 3];
            uint8_t* o = out + i * pitch + j * 4;
            o[0] = (uint8_t)color;
            o[1] = (uint8_t)(color >> 8);
            o[2] = (uint8_t)(color >> 16);
            o[3] = (uint8_t)(color >> 24);
            idx >>= 2;
        }
    }
}

// block.rs:202-215
void decode_sharp_alpha_block(const uint8_t* cb, uint8_t* out, size_t pitch) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            uint8_t a = (cb[i * 2 + j / 2] >> ((j % 2) * 4)) & 0x0F;
            out[i * pitch + j * 4 + 3] = (uint8_t)(a * 17);
        }
}

// block.rs:221-258
void decode_smooth_alpha_block(const uint8_t* cb, uint8_t* out, size_t pitch, size_t pixel_size) {
    uint64_t block = 0;
    for (int i = 0; i < 8; i++) block |= (uint64_t)cb[i] << (8 * i);
    uint8_t a[8];
    a[0] = (uint8_t)(block & 0xFF);
    a[1] = (uint8_t)((block >> 8) & 0xFF);
    if (a[0] > a[1]) {
        a[2] = (uint8_t)((6 * a[0] + a[1]) / 7);
        a[3] = (uint8_t)((5 * a[0] + 2 * a[1]) / 7);
        a[4] = (uint8_t)((4 * a[0] + 3 * a[1]) / 7);
        a[5] = (uint8_t)((3 * a[0] + 4 * a[1]) / 7);
        a[6] = (uint8_t)((2 * a[0] + 5 * a[1]) / 7);
        a[7] = (uint8_t)((a[0] + 6 * a[1]) / 7);
    } else {
        a[2] = (uint8_t)((4 * a[0] + a[1]) / 5);
        a[3] = (uint8_t)((3 * a[0] + 2 * a[1]) / 5);
        a[4] = (uint8_t)((2 * a[0] + 3 * a[1]) / 5);
        a[5] = (uint8_t)((a[0] + 4 * a[1]) / 5);
        a[6] = 0x00;
        a[7] = 0xFF;
    }
    uint64_t indices = block >> 16;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            out[i * pitch + j * pixel_size] = a[indices & 7];
            indices >>= 3;
        }
}

// block.rs:1341-1403
struct BitStream {
    uint64_t low, high;
    explicit BitStream(const uint8_t* d) {
        low = 0;
        high = 0;
        for (int i = 0; i < 8; i++) low |= (uint64_t)d[i] << (8 * i);
        for (int i = 0; i < 8; i++) high |= (uint64_t)d[8 + i] << (8 * i);
    }
    uint32_t read_bits(uint32_t n) {
        uint64_t mask = (n >= 64) ? ~0ull : ((1ull << n) - 1);
        uint32_t bits = (uint32_t)(low & mask);
        low = (n >= 64) ? 0 : (low >> n);
        // Rust `x << (64 - n)` for n == 0 would be a shift by 64; it is never reached.
        if (n > 0) low |= (high & mask) << (64 - n);
        high = (n >= 64) ? 0 : (high >> n);
        return bits;
    }
    int32_t read_bit_i32() { return (int32_t)read_bits(1); }
    int32_t read_bits_i32(uint32_t n) { return (int32_t)read_bits(n); }
    int32_t read_bits_reversed(uint32_t n) {
        int32_t bits = read_bits_i32(n);
        int32_t result = 0;
        for (uint32_t i = 0; i < n; i++) {
            result <<= 1;
            result |= bits & 1;
            bits >>= 1;
        }
        return result;
    }
};

// block.rs:1256-1258
inline int32_t interpolate(int32_t a, int32_t b, const int32_t* weights, int32_t index) {
    return (a * (64 - weights[index]) + b * weights[index] + 32) >> 6;
}

// block.rs:1262-1266
inline int32_t extend_sign(int32_t val, int32_t bits) {
    return (int32_t)((uint32_t)val << (32 - bits)) >> (32 - bits);
}

// block.rs:1268-1279
inline int32_t transform_inverse(int32_t val, int32_t a0, int32_t bits, bool is_signed) {
    int32_t t = (val + a0) & ((1 << bits) - 1);
    return is_signed ? extend_sign(t, bits) : t;
}

// block.rs:1281-1313
inline int32_t unquantize(int32_t val, int32_t bits, bool is_signed) {
    if (!is_signed) {
        if (bits >= 15) return val;
        if (val == 0) return 0;
        if (val == ((1 << bits) - 1)) return 0xFFFF;
        return ((val << 16) + 0x8000) >> bits;
    }
    if (bits >= 16) return val;
    bool s = val < 0;
    int32_t v = s ? -val : val;
    int32_t unq;
    if (v == 0) unq = 0;
    else if (v >= ((1 << (bits - 1)) - 1)) unq = 0x7FFF;
    else unq = ((v << 15) + 0x4000) >> (bits - 1);
    return s ? -unq : unq;
}

// block.rs:1315-1336
inline uint16_t finish_unquantize(int32_t val, bool is_signed) {
    if (!is_signed) return (uint16_t)((val * 31) >> 6);
    int32_t scaled = val < 0 ? -(((-val) * 31) >> 5) : (val * 31) >> 5;
    uint32_t sign_bit = 0;
    int32_t mag = scaled;
    if (scaled < 0) {
        sign_bit = 0x8000;
        mag = -scaled;
    }
    return (uint16_t)(sign_bit | (uint32_t)mag);
}

}  // namespace

// IEEE binary16 -> binary32, exact (half::f16::to_f32).
float half_to_float(uint16_t h) {
    uint32_t sign = (uint32_t)(h >> 15) << 31;
    uint32_t exp = (h >> 10) & 0x1F;
    uint32_t man = h & 0x3FF;
    uint32_t bits;
    if (exp == 0) {
        if (man == 0) {
            bits = sign;
        } else {
            int e = -1;
            do {
                e++;
                man <<= 1;
            } while ((man & 0x400) == 0);
            man &= 0x3FF;
            bits = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 31) {
        bits = sign | 0x7F800000u | (man << 13);
    } else {
        bits = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// ---- block decoders (block.rs public API) ---------------------------------

void decode_block_bc1(const uint8_t* c, uint8_t* o, size_t pitch) { decode_color_block(c, o, pitch, false); }

void decode_block_bc2(const uint8_t* c, uint8_t* o, size_t pitch) {
    decode_color_block(c + 8, o, pitch, true);
    decode_sharp_alpha_block(c, o, pitch);
}

void decode_block_bc3(const uint8_t* c, uint8_t* o, size_t pitch) {
    decode_color_block(c + 8, o, pitch, true);
    decode_smooth_alpha_block(c, o + 3, pitch, 4);
}

void decode_block_bc4(const uint8_t* c, uint8_t* o, size_t pitch) { decode_smooth_alpha_block(c, o, pitch, 1); }

void decode_block_bc5(const uint8_t* c, uint8_t* o, size_t pitch) {
    decode_smooth_alpha_block(c, o, pitch, 2);
    decode_smooth_alpha_block(c + 8, o + 1, pitch, 2);
}

// block.rs:262-769
void decode_block_bc6h(const uint8_t* c, uint16_t* o, size_t pitch, bool is_signed) {
    static const uint8_t kBits[4][14] = {
        {10, 7, 11, 11, 11, 9, 8, 8, 8, 6, 10, 11, 12, 16},
        {5, 6, 5, 4, 4, 5, 6, 5, 5, 6, 10, 9, 8, 4},
        {5, 6, 4, 5, 4, 5, 5, 6, 5, 6, 10, 9, 8, 4},
        {5, 6, 4, 4, 5, 5, 5, 5, 6, 6, 10, 9, 8, 4},
    };
    static const int32_t w3[8] = {0, 9, 18, 27, 37, 46, 55, 64};
    static const int32_t w4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};
    BitStream bs(c);
    int32_t r[4] = {0}, g[4] = {0}, b[4] = {0};
    uint32_t mode = bs.read_bits(2);
    if (mode > 1) mode |= bs.read_bits(3) << 2;
    int32_t partition = 0;
    switch (mode) {
        case 0x00:
            g[2] |= bs.read_bit_i32() << 4; b[2] |= bs.read_bit_i32() << 4; b[3] |= bs.read_bit_i32() << 4;
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(5); g[3] |= bs.read_bit_i32() << 4; g[2] |= bs.read_bits_i32(4);
            g[1] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32(); g[3] |= bs.read_bits_i32(4);
            b[1] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4);
            r[2] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 3; partition = bs.read_bits_i32(5); mode = 0;
            break;
        case 0x01:
            g[2] |= bs.read_bit_i32() << 5; g[3] |= bs.read_bit_i32() << 4; g[3] |= bs.read_bit_i32() << 5;
            r[0] |= bs.read_bits_i32(7); b[3] |= bs.read_bit_i32(); b[3] |= bs.read_bit_i32() << 1;
            b[2] |= bs.read_bit_i32() << 4; g[0] |= bs.read_bits_i32(7); b[2] |= bs.read_bit_i32() << 5;
            b[3] |= bs.read_bit_i32() << 2; g[2] |= bs.read_bit_i32() << 4; b[0] |= bs.read_bits_i32(7);
            b[3] |= bs.read_bit_i32() << 3; b[3] |= bs.read_bit_i32() << 5; b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(6); g[2] |= bs.read_bits_i32(4); g[1] |= bs.read_bits_i32(6);
            g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(6); b[2] |= bs.read_bits_i32(4);
            r[2] |= bs.read_bits_i32(6); r[3] |= bs.read_bits_i32(6); partition = bs.read_bits_i32(5); mode = 1;
            break;
        case 0x02:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(5); r[0] |= bs.read_bit_i32() << 10; g[2] |= bs.read_bits_i32(4);
            g[1] |= bs.read_bits_i32(4); g[0] |= bs.read_bit_i32() << 10; b[3] |= bs.read_bit_i32();
            g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(4); b[0] |= bs.read_bit_i32() << 10;
            b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 3;
            partition = bs.read_bits_i32(5); mode = 2;
            break;
        case 0x06:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(4); r[0] |= bs.read_bit_i32() << 10; g[3] |= bs.read_bit_i32() << 4;
            g[2] |= bs.read_bits_i32(4); g[1] |= bs.read_bits_i32(5); g[0] |= bs.read_bit_i32() << 10;
            g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(4); b[0] |= bs.read_bit_i32() << 10;
            b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(4);
            b[3] |= bs.read_bit_i32(); b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(4);
            g[2] |= bs.read_bit_i32() << 4; b[3] |= bs.read_bit_i32() << 3; partition = bs.read_bits_i32(5);
            mode = 3;
            break;
        case 0x0A:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(4); r[0] |= bs.read_bit_i32() << 10; b[2] |= bs.read_bit_i32() << 4;
            g[2] |= bs.read_bits_i32(4); g[1] |= bs.read_bits_i32(4); g[0] |= bs.read_bit_i32() << 10;
            b[3] |= bs.read_bit_i32(); g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(5);
            b[0] |= bs.read_bit_i32() << 10; b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(4);
            b[3] |= bs.read_bit_i32() << 1; b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(4);
            b[3] |= bs.read_bit_i32() << 4; b[3] |= bs.read_bit_i32() << 3; partition = bs.read_bits_i32(5);
            mode = 4;
            break;
        case 0x0E:
            r[0] |= bs.read_bits_i32(9); b[2] |= bs.read_bit_i32() << 4; g[0] |= bs.read_bits_i32(9);
            g[2] |= bs.read_bit_i32() << 4; b[0] |= bs.read_bits_i32(9); b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(5); g[3] |= bs.read_bit_i32() << 4; g[2] |= bs.read_bits_i32(4);
            g[1] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32(); g[3] |= bs.read_bits_i32(4);
            b[1] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4);
            r[2] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 3; partition = bs.read_bits_i32(5); mode = 5;
            break;
        case 0x12:
            r[0] |= bs.read_bits_i32(8); g[3] |= bs.read_bit_i32() << 4; b[2] |= bs.read_bit_i32() << 4;
            g[0] |= bs.read_bits_i32(8); b[3] |= bs.read_bit_i32() << 2; g[2] |= bs.read_bit_i32() << 4;
            b[0] |= bs.read_bits_i32(8); b[3] |= bs.read_bit_i32() << 3; b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(6); g[2] |= bs.read_bits_i32(4); g[1] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32(); g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(6);
            r[3] |= bs.read_bits_i32(6); partition = bs.read_bits_i32(5); mode = 6;
            break;
        case 0x16:
            r[0] |= bs.read_bits_i32(8); b[3] |= bs.read_bit_i32(); b[2] |= bs.read_bit_i32() << 4;
            g[0] |= bs.read_bits_i32(8); g[2] |= bs.read_bit_i32() << 5; g[2] |= bs.read_bit_i32() << 4;
            b[0] |= bs.read_bits_i32(8); g[3] |= bs.read_bit_i32() << 5; b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(5); g[3] |= bs.read_bit_i32() << 4; g[2] |= bs.read_bits_i32(4);
            g[1] |= bs.read_bits_i32(6); g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 3;
            partition = bs.read_bits_i32(5); mode = 7;
            break;
        case 0x1A:
            r[0] |= bs.read_bits_i32(8); b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bit_i32() << 4;
            g[0] |= bs.read_bits_i32(8); b[2] |= bs.read_bit_i32() << 5; g[2] |= bs.read_bit_i32() << 4;
            b[0] |= bs.read_bits_i32(8); b[3] |= bs.read_bit_i32() << 5; b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(5); g[3] |= bs.read_bit_i32() << 4; g[2] |= bs.read_bits_i32(4);
            g[1] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32(); g[3] |= bs.read_bits_i32(4);
            b[1] |= bs.read_bits_i32(6); b[2] |= bs.read_bits_i32(4); r[2] |= bs.read_bits_i32(5);
            b[3] |= bs.read_bit_i32() << 2; r[3] |= bs.read_bits_i32(5); b[3] |= bs.read_bit_i32() << 3;
            partition = bs.read_bits_i32(5); mode = 8;
            break;
        case 0x1E:
            r[0] |= bs.read_bits_i32(6); g[3] |= bs.read_bit_i32() << 4; b[3] |= bs.read_bit_i32();
            b[3] |= bs.read_bit_i32() << 1; b[2] |= bs.read_bit_i32() << 4; g[0] |= bs.read_bits_i32(6);
            g[2] |= bs.read_bit_i32() << 5; b[2] |= bs.read_bit_i32() << 5; b[3] |= bs.read_bit_i32() << 2;
            g[2] |= bs.read_bit_i32() << 4; b[0] |= bs.read_bits_i32(6); g[3] |= bs.read_bit_i32() << 5;
            b[3] |= bs.read_bit_i32() << 3; b[3] |= bs.read_bit_i32() << 5; b[3] |= bs.read_bit_i32() << 4;
            r[1] |= bs.read_bits_i32(6); g[2] |= bs.read_bits_i32(4); g[1] |= bs.read_bits_i32(6);
            g[3] |= bs.read_bits_i32(4); b[1] |= bs.read_bits_i32(6); b[2] |= bs.read_bits_i32(4);
            r[2] |= bs.read_bits_i32(6); r[3] |= bs.read_bits_i32(6); partition = bs.read_bits_i32(5); mode = 9;
            break;
        case 0x03:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(10); g[1] |= bs.read_bits_i32(10); b[1] |= bs.read_bits_i32(10);
            mode = 10;
            break;
        case 0x07:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(9); r[0] |= bs.read_bit_i32() << 10; g[1] |= bs.read_bits_i32(9);
            g[0] |= bs.read_bit_i32() << 10; b[1] |= bs.read_bits_i32(9); b[0] |= bs.read_bit_i32() << 10;
            mode = 11;
            break;
        case 0x0B:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(8); r[0] |= bs.read_bits_reversed(2) << 10; g[1] |= bs.read_bits_i32(8);
            g[0] |= bs.read_bits_reversed(2) << 10; b[1] |= bs.read_bits_i32(8); b[0] |= bs.read_bits_reversed(2) << 10;
            mode = 12;
            break;
        case 0x0F:
            r[0] |= bs.read_bits_i32(10); g[0] |= bs.read_bits_i32(10); b[0] |= bs.read_bits_i32(10);
            r[1] |= bs.read_bits_i32(4); r[0] |= bs.read_bits_reversed(6) << 10; g[1] |= bs.read_bits_i32(4);
            g[0] |= bs.read_bits_reversed(6) << 10; b[1] |= bs.read_bits_i32(4); b[0] |= bs.read_bits_reversed(6) << 10;
            mode = 13;
            break;
        default:
            for (int i = 0; i < 4; i++)
                for (int k = 0; k < 12; k++) o[i * pitch + k] = 0;
            return;
    }
    int num_partitions = mode >= 10 ? 0 : 1;
    int32_t bits0 = kBits[0][mode];
    if (is_signed) {
        r[0] = extend_sign(r[0], bits0);
        g[0] = extend_sign(g[0], bits0);
        b[0] = extend_sign(b[0], bits0);
    }
    if ((mode != 9 && mode != 10) || is_signed) {
        for (int i = 1; i < (num_partitions + 1) * 2; i++) {
            r[i] = extend_sign(r[i], kBits[1][mode]);
            g[i] = extend_sign(g[i], kBits[2][mode]);
            b[i] = extend_sign(b[i], kBits[3][mode]);
        }
    }
    if (mode != 9 && mode != 10) {
        for (int i = 1; i < (num_partitions + 1) * 2; i++) {
            r[i] = transform_inverse(r[i], r[0], bits0, is_signed);
            g[i] = transform_inverse(g[i], g[0], bits0, is_signed);
            b[i] = transform_inverse(b[i], b[0], bits0, is_signed);
        }
    }
    for (int i = 0; i < (num_partitions + 1) * 2; i++) {
        r[i] = unquantize(r[i], bits0, is_signed);
        g[i] = unquantize(g[i], bits0, is_signed);
        b[i] = unquantize(b[i], bits0, is_signed);
    }
    const int32_t* weights = mode >= 10 ? w4 : w3;
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            int32_t ps;
            if (mode >= 10) ps = (i | j) == 0 ? 128 : 0;
            else ps = bc6h_partition_set(partition, i * 4 + j);
            uint32_t index_bits = mode >= 10 ? 4 : 3;
            if (ps & 0x80) index_bits -= 1;
            ps &= 1;
            int32_t index = bs.read_bits_i32(index_bits);
            int e = ps * 2;
            uint16_t* out = o + i * pitch + j * 3;
            out[0] = finish_unquantize(interpolate(r[e], r[e + 1], weights, index), is_signed);
            out[1] = finish_unquantize(interpolate(g[e], g[e + 1], weights, index), is_signed);
            out[2] = finish_unquantize(interpolate(b[e], b[e + 1], weights, index), is_signed);
        }
    }
}

// block.rs:774-796
void decode_block_bc6h_float(const uint8_t* c, float* o, size_t pitch, bool is_signed) {
    uint16_t block[48];
    std::memset(block, 0, sizeof(block));
    decode_block_bc6h(c, block, 12, is_signed);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 3; k++) o[i * pitch + j * 3 + k] = half_to_float(block[i * 12 + j * 3 + k]);
}

// block.rs:801-1252
void decode_block_bc7(const uint8_t* c, uint8_t* o, size_t pitch) {
    static const uint8_t kBits[2][8] = {{4, 6, 5, 7, 5, 7, 7, 5}, {0, 0, 0, 0, 6, 8, 7, 5}};
    static const int32_t w2[4] = {0, 21, 43, 64};
    static const int32_t w3[8] = {0, 9, 18, 27, 37, 46, 55, 64};
    static const int32_t w4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};
    const uint32_t has_pbits = 0xCB;  // 0b11001011
    BitStream bs(c);
    uint32_t mode = 0;
    while (mode < 8 && bs.read_bits(1) == 0) mode++;
    if (mode >= 8) {
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 16; j++) o[i * pitch + j] = 0;
        return;
    }
    uint32_t partition = 0, num_partitions = 1, rotation = 0, isb = 0;
    if (mode == 0 || mode == 1 || mode == 2 || mode == 3 || mode == 7) {
        num_partitions = (mode == 0 || mode == 2) ? 3 : 2;
        partition = bs.read_bits(mode == 0 ? 4 : 6);
    }
    uint32_t num_endpoints = num_partitions * 2;
    if (mode == 4 || mode == 5) {
        rotation = bs.read_bits(2);
        if (mode == 4) isb = bs.read_bits(1);
    }
    int32_t ep[6][4];
    std::memset(ep, 0, sizeof(ep));
    for (int i = 0; i < 3; i++)
        for (uint32_t j = 0; j < num_endpoints; j++) ep[j][i] = (int32_t)bs.read_bits(kBits[0][mode]);
    if (kBits[1][mode] > 0)
        for (uint32_t j = 0; j < num_endpoints; j++) ep[j][3] = (int32_t)bs.read_bits(kBits[1][mode]);
    if (mode == 0 || mode == 1 || mode == 3 || mode == 6 || mode == 7) {
        for (uint32_t j = 0; j < num_endpoints; j++)
            for (int k = 0; k < 4; k++) ep[j][k] <<= 1;
        if (mode == 1) {
            int32_t i0 = (int32_t)bs.read_bits(1);
            int32_t j0 = (int32_t)bs.read_bits(1);
            for (int k = 0; k < 3; k++) {
                ep[0][k] |= i0;
                ep[1][k] |= i0;
                ep[2][k] |= j0;
                ep[3][k] |= j0;
            }
        } else if (has_pbits & (1u << mode)) {
            for (uint32_t j = 0; j < num_endpoints; j++) {
                int32_t pb = (int32_t)bs.read_bits(1);
                for (int k = 0; k < 4; k++) ep[j][k] |= pb;
            }
        }
    }
    for (uint32_t i = 0; i < num_endpoints; i++) {
        uint32_t j = kBits[0][mode] + ((has_pbits >> mode) & 1);
        for (int k = 0; k < 3; k++) {
            ep[i][k] <<= 8 - j;
            ep[i][k] |= ep[i][k] >> j;
        }
        j = kBits[1][mode] + ((has_pbits >> mode) & 1);
        ep[i][3] <<= 8 - j;
        ep[i][3] |= ep[i][3] >> j;
    }
    if (kBits[1][mode] == 0)
        for (uint32_t j = 0; j < num_endpoints; j++) ep[j][3] = 0xFF;
    uint32_t index_bits = (mode == 0 || mode == 1) ? 3 : (mode == 6 ? 4 : 2);
    uint32_t index_bits2 = mode == 4 ? 3 : (mode == 5 ? 2 : 0);
    const int32_t* weights = index_bits == 2 ? w2 : (index_bits == 3 ? w3 : w4);
    const int32_t* weights2 = index_bits2 == 2 ? w2 : w3;
    int32_t indices[4][4];
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            uint32_t ps = num_partitions == 1 ? ((i | j) == 0 ? 128u : 0u)
                                              : bc7_partition_set(num_partitions, partition, i * 4 + j);
            uint32_t ib = index_bits;
            if (ps & 0x80) ib -= 1;
            indices[i][j] = (int32_t)bs.read_bits(ib);
        }
    }
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            uint32_t ps = num_partitions == 1 ? ((i | j) == 0 ? 128u : 0u)
                                              : bc7_partition_set(num_partitions, partition, i * 4 + j);
            ps &= 3;
            int32_t index = indices[i][j];
            int32_t rr, gg, bb, aa;
            const int32_t* e0 = ep[ps * 2];
            const int32_t* e1 = ep[ps * 2 + 1];
            if (index_bits2 == 0) {
                rr = interpolate(e0[0], e1[0], weights, index);
                gg = interpolate(e0[1], e1[1], weights, index);
                bb = interpolate(e0[2], e1[2], weights, index);
                aa = interpolate(e0[3], e1[3], weights, index);
            } else {
                int32_t index2 = (int32_t)bs.read_bits((i | j) == 0 ? index_bits2 - 1 : index_bits2);
                if (isb == 0) {
                    rr = interpolate(e0[0], e1[0], weights, index);
                    gg = interpolate(e0[1], e1[1], weights, index);
                    bb = interpolate(e0[2], e1[2], weights, index);
                    aa = interpolate(e0[3], e1[3], weights2, index2);
                } else {
                    rr = interpolate(e0[0], e1[0], weights2, index2);
                    gg = interpolate(e0[1], e1[1], weights2, index2);
                    bb = interpolate(e0[2], e1[2], weights2, index2);
                    aa = interpolate(e0[3], e1[3], weights, index);
                }
            }
            int32_t t;
            switch (rotation) {
                case 1: t = aa; aa = rr; rr = t; break;
                case 2: t = aa; aa = gg; gg = t; break;
                case 3: t = aa; aa = bb; bb = t; break;
                default: break;
            }
            uint8_t* out = o + i * pitch + j * 4;
            out[0] = (uint8_t)rr;
            out[1] = (uint8_t)gg;
            out[2] = (uint8_t)bb;
            out[3] = (uint8_t)aa;
        }
    }
}

// decode.rs:151-159 (linear_to_srgb)
uint8_t linear_to_srgb(float linear) {
    float v = linear <= 0.0031308f ? linear * 12.92f : 1.055f * std::pow(linear, 1.0f / 2.4f) - 0.055f;
    float c = v;
    if (c < 0.0f) c = 0.0f;
    if (c > 1.0f) c = 1.0f;
    float r = std::round(c * 255.0f);
    if (std::isnan(r)) return 0;  // Rust `as u8` maps NaN to 0
    return (uint8_t)r;
}

// decode.rs:60-198: per-variant block -> RGBA8 conversions.
void decode_block_rgba8(int variant, const uint8_t* c, uint8_t* o, size_t pitch) {
    switch (variant) {
        case 0: decode_block_bc1(c, o, pitch); break;
        case 1: decode_block_bc2(c, o, pitch); break;
        case 2: decode_block_bc3(c, o, pitch); break;
        case 3: {
            uint8_t buf[16] = {0};
            decode_block_bc4(c, buf, 4);
            for (int y = 0; y < 4; y++)
                for (int x = 0; x < 4; x++) {
                    uint8_t* q = o + y * pitch + x * 4;
                    q[0] = buf[y * 4 + x];
                    q[1] = 0;
                    q[2] = 0;
                    q[3] = 0;
                }
            break;
        }
        case 4: {
            uint8_t buf[32] = {0};
            decode_block_bc5(c, buf, 8);
            for (int y = 0; y < 4; y++)
                for (int x = 0; x < 4; x++) {
                    uint8_t* q = o + y * pitch + x * 4;
                    q[0] = buf[y * 8 + x * 2];
                    q[1] = buf[y * 8 + x * 2 + 1];
                    q[2] = 0;
                    q[3] = 0;
                }
            break;
        }
        case 5: {
            float buf[48] = {0};
            decode_block_bc6h_float(c, buf, 12, false);
            for (int y = 0; y < 4; y++)
                for (int x = 0; x < 4; x++) {
                    uint8_t* q = o + y * pitch + x * 4;
                    q[0] = linear_to_srgb(buf[y * 12 + x * 3]);
                    q[1] = linear_to_srgb(buf[y * 12 + x * 3 + 1]);
                    q[2] = linear_to_srgb(buf[y * 12 + x * 3 + 2]);
                    q[3] = 0;
                }
            break;
        }
        case 6: decode_block_bc7(c, o, pitch); break;
        default: break;
    }
}

}  // namespace oracle

extern "C" float oracle_f16_to_f32(uint16_t h) { return oracle::half_to_float(h); }
