// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Image-level drivers restating src/encode.rs and src/decode.rs, plus the C
// entry points of oracle.h. The reference parallelises its block loops with
// rayon (src/encode.rs:267-287); here std::thread over block rows stands in.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle.h"
#include "oracle_common.h"
#include "oracle_decode.h"

namespace oracle {

namespace {

template <class F>
void parallel_rows(size_t rows, int threads, F fn) {
    if (threads <= 1 || rows < 2) {
        for (size_t r = 0; r < rows; r++) fn(r);
        return;
    }
    size_t n = std::min<size_t>((size_t)threads, rows);
    std::vector<std::thread> pool;
    pool.reserve(n);
    for (size_t t = 0; t < n; t++) {
        pool.emplace_back([=, &fn]() {
            for (size_t r = t; r < rows; r += n) fn(r);
        });
    }
    for (auto& th : pool) th.join();
}

size_t block_bytes(int variant) { return (variant == 0 || variant == 3) ? 8 : 16; }

// bc1_to_5.rs:14-40 / bc7.rs:38-63
void load_rgba(const uint8_t* src, size_t xx, size_t yy, size_t stride, float block[64]) {
    for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
            const uint8_t* p = src + (yy * 4 + y) * stride + (xx * 4 + x) * 4;
            int o = y * 4 + x;
            block[o] = (float)p[0];
            block[16 + o] = (float)p[1];
            block[32 + o] = (float)p[2];
            block[48 + o] = (float)p[3];
        }
}

// bc1_to_5.rs:42-82 (channel 0 = R, 1 = G into the alpha slot)
void load_channel(const uint8_t* src, size_t xx, size_t yy, size_t stride, int ch, float block[64]) {
    for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++)
            block[48 + y * 4 + x] = (float)src[(yy * 4 + y) * stride + (xx * 4 + x) * 4 + ch];
}

// bc1_to_5.rs:84-115
void load_alpha_4bit(const uint8_t* src, size_t xx, size_t yy, size_t stride, uint32_t bits[2]) {
    bits[0] = 0;
    bits[1] = 0;
    for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
            float alpha = (float)src[(yy * 4 + y) * stride + (xx * 4 + x) * 4 + 3] / 255.0f;
            uint32_t a4 = f2u(alpha * 15.0f);
            uint32_t pos = y * 16 + x * 4;
            if (pos < 32) bits[0] |= a4 << pos;
            else bits[1] |= a4 << (pos - 32);
        }
}

// bc6h.rs:20-27 (powf from the C library, as Rust std uses on Linux)
float srgb_to_linear(uint8_t s) {
    float v = (float)s / 255.0f;
    if (v <= 0.04045f) return v / 12.92f;
    return std::pow((v + 0.055f) / 1.055f, 2.4f);
}

void store_words(uint8_t* dst, const uint32_t* w, int n) {
    for (int i = 0; i < n; i++) {
        dst[i * 4 + 0] = (uint8_t)w[i];
        dst[i * 4 + 1] = (uint8_t)(w[i] >> 8);
        dst[i * 4 + 2] = (uint8_t)(w[i] >> 16);
        dst[i * 4 + 3] = (uint8_t)(w[i] >> 24);
    }
}

}  // namespace

// IEEE binary32 -> binary16, round to nearest even (half::f16::from_f32).
uint16_t f32_to_f16(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFF) return (uint16_t)(man ? (sign | 0x7E00u | (man >> 13)) : (sign | 0x7C00u));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t m = man | 0x800000u;
        int shift = 14 - e;
        uint32_t hm = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1);
        uint32_t halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (hm & 1))) hm++;
        return (uint16_t)(sign | hm);
    }
    uint32_t h = sign | ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1))) h++;
    return (uint16_t)h;
}

}  // namespace oracle

using namespace oracle;

extern "C" int oracle_compress_rgba8(int variant, const void* settings, const uint8_t* src, size_t src_len,
                                     uint8_t* dst, size_t dst_len, uint32_t width, uint32_t height,
                                     uint32_t stride, int threads) {
    if (height % 4 != 0 || width % 4 != 0) return ORACLE_ERR_DIMS;
    if (variant < 0 || variant > 6) return ORACLE_ERR_VARIANT;
    size_t bw = (width + 3) / 4, bh = (height + 3) / 4;
    size_t bb = block_bytes(variant);
    if (dst_len < bw * bh * bb) return ORACLE_ERR_DST;
    if (bh > 0 && bw > 0) {
        size_t need = (size_t)(height - 1) * stride + (size_t)width * 4;
        if (src_len < need) return ORACLE_ERR_SRC;
    }
    const BC6HSettings* s6 = (const BC6HSettings*)settings;
    const BC7Settings* s7 = (const BC7Settings*)settings;
    if ((variant == 5 || variant == 6) && settings == nullptr) return ORACLE_ERR_VARIANT;
    parallel_rows(bh, threads, [&](size_t yy) {
        for (size_t xx = 0; xx < bw; xx++) {
            uint8_t* out = dst + (yy * bw + xx) * bb;
            float block[64];
            std::memset(block, 0, sizeof(block));
            uint32_t w[4] = {0, 0, 0, 0};
            switch (variant) {
                case 0:  // encode.rs:260-299
                    load_rgba(src, xx, yy, stride, block);
                    bc1_core(block, w);
                    store_words(out, w, 2);
                    break;
                case 1: {  // encode.rs:302-361
                    uint32_t a[2];
                    load_alpha_4bit(src, xx, yy, stride, a);
                    w[0] = a[0];
                    w[1] = a[1];
                    load_rgba(src, xx, yy, stride, block);
                    bc1_core(block, w + 2);
                    store_words(out, w, 4);
                    break;
                }
                case 2:  // encode.rs:364-422
                    load_rgba(src, xx, yy, stride, block);
                    bc3_alpha(block, w);
                    bc1_core(block, w + 2);
                    store_words(out, w, 4);
                    break;
                case 3:  // encode.rs:425-475
                    load_channel(src, xx, yy, stride, 0, block);
                    bc3_alpha(block, w);
                    store_words(out, w, 2);
                    break;
                case 4:  // encode.rs:478-539
                    load_channel(src, xx, yy, stride, 0, block);
                    bc3_alpha(block, w);
                    load_channel(src, xx, yy, stride, 1, block);
                    bc3_alpha(block, w + 2);
                    store_words(out, w, 4);
                    break;
                case 5: {  // encode.rs:542-578, bc6h.rs:45-71
                    for (int y = 0; y < 4; y++)
                        for (int x = 0; x < 4; x++) {
                            const uint8_t* p = src + (yy * 4 + y) * stride + (xx * 4 + x) * 4;
                            int o = y * 4 + x;
                            block[o] = (float)f32_to_f16(srgb_to_linear(p[0]));
                            block[16 + o] = (float)f32_to_f16(srgb_to_linear(p[1]));
                            block[32 + o] = (float)f32_to_f16(srgb_to_linear(p[2]));
                            block[48 + o] = 0.0f;
                        }
                    bc6h_encode_block(block, s6, w);
                    store_words(out, w, 4);
                    break;
                }
                case 6:  // encode.rs:620-659
                    load_rgba(src, xx, yy, stride, block);
                    bc7_encode_block(block, s7, w);
                    store_words(out, w, 4);
                    break;
            }
        }
    });
    return ORACLE_OK;
}

extern "C" int oracle_compress_rgba16(const void* settings, const uint16_t* src, size_t src_len, uint8_t* dst,
                                      size_t dst_len, uint32_t width, uint32_t height, uint32_t stride,
                                      int threads) {
    if (height % 4 != 0 || width % 4 != 0) return ORACLE_ERR_DIMS;
    size_t bw = (width + 3) / 4, bh = (height + 3) / 4;
    if (dst_len < bw * bh * 16) return ORACLE_ERR_DST;
    if (settings == nullptr) return ORACLE_ERR_VARIANT;
    if (bh > 0 && bw > 0) {
        size_t need = (size_t)(height - 1) * stride + (size_t)width * 4;
        if (src_len < need) return ORACLE_ERR_SRC;
    }
    const BC6HSettings* s6 = (const BC6HSettings*)settings;
    parallel_rows(bh, threads, [&](size_t yy) {
        for (size_t xx = 0; xx < bw; xx++) {
            float block[64];
            // bc6h.rs:73-97: f16 bit patterns converted to f32, alpha slot 0.
            for (int y = 0; y < 4; y++)
                for (int x = 0; x < 4; x++) {
                    const uint16_t* p = src + (yy * 4 + y) * stride + (xx * 4 + x) * 4;
                    int o = y * 4 + x;
                    block[o] = (float)p[0];
                    block[16 + o] = (float)p[1];
                    block[32 + o] = (float)p[2];
                    block[48 + o] = 0.0f;
                }
            uint32_t w[4];
            bc6h_encode_block(block, s6, w);
            store_words(dst + (yy * bw + xx) * 16, w, 4);
        }
    });
    return ORACLE_OK;
}

// decode.rs:201-232 + 336-387
extern "C" int oracle_decompress_rgba8(int variant, uint32_t width, uint32_t height, const uint8_t* blocks,
                                       size_t blocks_len, uint8_t* out, size_t out_len, int threads) {
    if (variant < 0 || variant > 6) return ORACLE_ERR_VARIANT;
    size_t bw = (width + 3) / 4, bh = (height + 3) / 4;
    size_t bb = block_bytes(variant);
    if (blocks_len != bw * bh * bb) return ORACLE_ERR_SRC;
    if (out_len != (size_t)width * height * 4) return ORACLE_ERR_DST;
    // Any dimension that is not a multiple of 4 makes the reference write past
    // the output slice and panic.
    if (width % 4 != 0 || height % 4 != 0) return ORACLE_ERR_DIMS;
    size_t pitch = (size_t)width * 4;
    parallel_rows(bh, threads, [&](size_t by) {
        for (size_t bx = 0; bx < bw; bx++) {
            const uint8_t* c = blocks + (by * bw + bx) * bb;
            decode_block_rgba8(variant, c, out + by * 4 * pitch + bx * 16, pitch);
        }
    });
    return ORACLE_OK;
}

// decode.rs:247-278 + 397-428: RGB triplets written into an RGBA-pitched row.
extern "C" int oracle_decompress_rgba16f(uint32_t width, uint32_t height, const uint8_t* blocks,
                                         size_t blocks_len, uint16_t* out, size_t out_len) {
    size_t bw = (width + 3) / 4, bh = (height + 3) / 4;
    if (blocks_len != bw * bh * 16) return ORACLE_ERR_SRC;
    if (out_len != (size_t)width * height * 4) return ORACLE_ERR_DST;
    if (width % 4 != 0 || height % 4 != 0) return ORACLE_ERR_DIMS;
    size_t pitch = (size_t)width * 4;
    for (size_t by = 0; by < bh; by++)
        for (size_t bx = 0; bx < bw; bx++)
            decode_block_bc6h(blocks + (by * bw + bx) * 16, out + by * 4 * pitch + bx * 16, pitch, false);
    return ORACLE_OK;
}

// decode.rs:293-324 + 438-468
extern "C" int oracle_decompress_rgba32f(uint32_t width, uint32_t height, const uint8_t* blocks,
                                         size_t blocks_len, float* out, size_t out_len) {
    size_t bw = (width + 3) / 4, bh = (height + 3) / 4;
    if (blocks_len != bw * bh * 16) return ORACLE_ERR_SRC;
    if (out_len != (size_t)width * height * 4) return ORACLE_ERR_DST;
    if (width % 4 != 0 || height % 4 != 0) return ORACLE_ERR_DIMS;
    size_t pitch = (size_t)width * 4;
    for (size_t by = 0; by < bh; by++)
        for (size_t bx = 0; bx < bw; bx++)
            decode_block_bc6h_float(blocks + (by * bw + bx) * 16, out + by * 4 * pitch + bx * 16, pitch, false);
    return ORACLE_OK;
}

extern "C" void oracle_decode_block(int which, const uint8_t* block, void* out, size_t pitch, int is_signed) {
    switch (which) {
        case 0: decode_block_bc1(block, (uint8_t*)out, pitch); break;
        case 1: decode_block_bc2(block, (uint8_t*)out, pitch); break;
        case 2: decode_block_bc3(block, (uint8_t*)out, pitch); break;
        case 3: decode_block_bc4(block, (uint8_t*)out, pitch); break;
        case 4: decode_block_bc5(block, (uint8_t*)out, pitch); break;
        case 5: decode_block_bc6h(block, (uint16_t*)out, pitch, is_signed != 0); break;
        case 6: decode_block_bc6h_float(block, (float*)out, pitch, is_signed != 0); break;
        case 7: decode_block_bc7(block, (uint8_t*)out, pitch); break;
        default: break;
    }
}

extern "C" void oracle_encode_block_bc1(const float* block, uint32_t out[2]) { bc1_core(block, out); }
extern "C" void oracle_encode_block_bc3_alpha(const float* block, uint32_t out[2]) { bc3_alpha(block, out); }
extern "C" void oracle_encode_block_bc7(const float* block, const void* s, uint32_t out[4]) {
    bc7_encode_block(block, (const BC7Settings*)s, out);
}
extern "C" void oracle_encode_block_bc6h(const float* block, const void* s, uint32_t out[4]) {
    bc6h_encode_block(block, (const BC6HSettings*)s, out);
}
extern "C" float oracle_block_quant(uint32_t qblock[2], const float* block, uint32_t bits, const float* ep,
                                   uint32_t pattern, uint32_t channels) {
    return block_quant(qblock, block, bits, ep, pattern, channels);
}
extern "C" void oracle_opt_endpoints(float* ep, const float* block, uint32_t bits, const uint32_t qblock[2],
                                     uint32_t mask, uint32_t channels) {
    opt_endpoints(ep, block, bits, qblock, mask, channels);
}
extern "C" float oracle_block_pca_bound_split(const float* block, uint32_t mask, uint32_t channels) {
    float full[15] = {0};
    compute_stats_masked(full, block, 0xFFFFFFFFu, channels);
    return block_pca_bound_split(block, mask, full, channels);
}
extern "C" void oracle_block_segment_core(float* ep, const float* block, uint32_t mask, uint32_t channels) {
    block_segment_core(ep, block, mask, channels);
}
extern "C" void oracle_ep_quant_dequant(int32_t qep[24], float ep[24], uint32_t mode, uint32_t channels) {
    bc7_ep_quant_dequant(qep, ep, mode, channels);
}
extern "C" uint32_t oracle_get_pattern(int32_t part_id) { return get_pattern(part_id); }
extern "C" uint32_t oracle_get_pattern_mask(int32_t part_id, uint32_t j) { return get_pattern_mask(part_id, j); }
extern "C" uint32_t oracle_get_skip_packed(int32_t part_id) { return kSkipTable[part_id]; }
extern "C" uint32_t oracle_partition_set(uint32_t table_index, uint32_t k) { return bptc_partition_set(table_index, k); }
extern "C" uint16_t oracle_f32_to_f16(float f) { return f32_to_f16(f); }
extern "C" uint8_t oracle_linear_to_srgb(float linear) { return linear_to_srgb(linear); }
