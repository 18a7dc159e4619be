// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
//
// Relaxed (differentiable) BC1 / BC7 block decoding. The block layout is the
// one the reference decoders read (src/decode/block.rs:124-197 for BC1,
// :801-1258 for BC7); the endpoints become continuous values in 8-bit units
// and the interpolation drops the decoder's integer rounding:
//   BC7:  c = e0 + (e1 - e0) * w / 64, w = get_unquant_value(bits, index)
//         (src/encode/common.rs:6-21), rotation swap of block.rs:1238-1243;
//   BC1:  c = e0 + (e1 - e0) * t, t = 0, 1, 1/3, 2/3 for indices 0..3 in the
//         four-colour mode (block.rs:153-165); t = 0, 1, 1/2 and constant
//         transparent black for index 3 in the three-colour mode (:166-175).
// Mode, partition, rotation, index selector and indices stay fixed. The
// functions are templates so that the FD checks run them in double and the
// refinement restatement runs them in float, in the operation order the
// CUDA kernels use.
//
// Per-block metadata (shared layout with the CUDA kernels):
//   BC7 meta[8]: w0 = mode (8 = reserved encoding) | partition << 4 |
//                rotation << 10 | index selector << 12 | subsets << 13 |
//                colour index bits << 16 | alpha index bits << 20;
//                w1, w2 = colour index of pixel k at bits 4(k&7) (w1: k < 8);
//                w3, w4 = alpha index, same packing; w5 = subset of pixel k
//                at bits 2k; w6 = w7 = 0.
//   BC7 endpoints[24]: slot (2 * subset + end) * 4 + channel, decoder channel
//                order before the rotation swap (R, G, B, A).
//   BC1 meta[2]: w0 = colour0 | colour1 << 16 (RGB565), w1 = indices.
//   BC1 endpoints[6]: e0 R, G, B, e1 R, G, B, expanded from RGB565 the way
//                the decoder does ((v * 527 + 23) >> 6 for 5 bits, (v * 259 + 33) >> 6
//                for 6 bits).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle_decode.h"

namespace oracle {
namespace relaxed {

// LSB-first bit reader over the 16 block bytes.
struct ByteBits {
    const uint8_t* b;
    uint32_t pos;
    uint32_t get(uint32_t n) {
        uint32_t v = 0;
        for (uint32_t i = 0; i < n; i++, pos++) v |= (uint32_t)((b[pos >> 3] >> (pos & 7)) & 1) << i;
        return v;
    }
};

inline int bc7_weight(uint32_t bits, uint32_t index) {
    static const int w2[4] = {0, 21, 43, 64};
    static const int w3[8] = {0, 9, 18, 27, 37, 46, 55, 64};
    static const int w4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};
    return bits == 2 ? w2[index & 3] : (bits == 3 ? w3[index & 7] : w4[index & 15]);
}

// Parses one BC7 block into meta + endpoints (block.rs:801-1252 field order).
inline void bc7_parse(const uint8_t blk[16], uint32_t meta[8], float ep[24]) {
    static const uint32_t kColorBits[8] = {4, 6, 5, 7, 5, 7, 7, 5};
    static const uint32_t kAlphaBits[8] = {0, 0, 0, 0, 6, 8, 7, 5};
    static const uint32_t kSubsets[8] = {3, 2, 3, 2, 1, 1, 1, 2};
    static const uint32_t kIndexBits[8] = {3, 3, 2, 2, 2, 2, 4, 2};
    std::memset(meta, 0, 8 * sizeof(uint32_t));
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
    ByteBits bs{blk, 0};
    uint32_t mode = 0;
    while (mode < 8 && bs.get(1) == 0) mode++;
    if (mode == 8) {
        meta[0] = 8;
        return;
    }
    uint32_t subsets = kSubsets[mode], partition = 0, rotation = 0, isb = 0;
    if (subsets > 1) partition = bs.get(mode == 0 ? 4 : 6);
    if (mode == 4 || mode == 5) rotation = bs.get(2);
    if (mode == 4) isb = bs.get(1);
    uint32_t cb = kColorBits[mode], ab = kAlphaBits[mode], n = 2 * subsets;
    int e[6][4] = {{0}};
    for (int c = 0; c < 3; c++)
        for (uint32_t j = 0; j < n; j++) e[j][c] = (int)bs.get(cb);
    for (uint32_t j = 0; j < n && ab; j++) e[j][3] = (int)bs.get(ab);
    bool pbit = mode == 0 || mode == 1 || mode == 3 || mode == 6 || mode == 7;
    if (pbit) {
        int pb[6];
        if (mode == 1) {
            pb[0] = pb[1] = (int)bs.get(1);
            pb[2] = pb[3] = (int)bs.get(1);
        } else {
            for (uint32_t j = 0; j < n; j++) pb[j] = (int)bs.get(1);
        }
        for (uint32_t j = 0; j < n; j++)
            for (int c = 0; c < 4; c++)
                if (c < 3 || ab) e[j][c] = (e[j][c] << 1) | pb[j];
    }
    uint32_t pc = cb + (pbit ? 1 : 0), pa = ab + (pbit ? 1 : 0);
    for (uint32_t j = 0; j < n; j++) {
        for (int c = 0; c < 3; c++) {
            int v = e[j][c] << (8 - pc);
            ep[j * 4 + c] = (float)(v | (v >> pc));
        }
        if (ab) {
            int v = e[j][3] << (8 - pa);
            ep[j * 4 + 3] = (float)(v | (v >> pa));
        } else {
            ep[j * 4 + 3] = 255.0f;
        }
    }
    uint32_t table = subsets == 3 ? 64 + partition : partition;
    uint32_t ib = kIndexBits[mode], ib2 = mode == 4 ? 3 : (mode == 5 ? 2 : 0);
    uint32_t prim[16], sec[16], sub[16];
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t ps = subsets == 1 ? (k == 0 ? 0x80u : 0u) : bptc_partition_set(table, k);
        sub[k] = ps & 3;
        prim[k] = bs.get((ps & 0x80) ? ib - 1 : ib);
    }
    for (uint32_t k = 0; k < 16; k++) sec[k] = ib2 ? bs.get(k == 0 ? ib2 - 1 : ib2) : prim[k];
    uint32_t cbits = ib, abits = ib;
    const uint32_t* ci = prim;
    const uint32_t* ai = prim;
    if (ib2) {
        ai = isb ? prim : sec;
        ci = isb ? sec : prim;
        cbits = isb ? ib2 : ib;
        abits = isb ? ib : ib2;
    }
    if (ab == 0) abits = 0;
    meta[0] = mode | partition << 4 | rotation << 10 | isb << 12 | subsets << 13 | cbits << 16 | abits << 20;
    for (uint32_t k = 0; k < 16; k++) {
        meta[1 + (k >> 3)] |= ci[k] << (4 * (k & 7));
        meta[3 + (k >> 3)] |= ai[k] << (4 * (k & 7));
        meta[5] |= sub[k] << (2 * k);
    }
}

// Relaxed BC7 decode: out[k * 4 + c], k = y * 4 + x, RGBA after rotation.
template <class T>
void bc7_relaxed(const uint32_t meta[8], const T ep[24], T out[64]) {
    uint32_t mode = meta[0] & 15;
    if (mode >= 8) {
        for (int i = 0; i < 64; i++) out[i] = T(0);
        return;
    }
    uint32_t rot = (meta[0] >> 10) & 3, cbits = (meta[0] >> 16) & 7, abits = (meta[0] >> 20) & 7;
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t s = (meta[5] >> (2 * k)) & 3;
        uint32_t ci = (meta[1 + (k >> 3)] >> (4 * (k & 7))) & 15, ai = (meta[3 + (k >> 3)] >> (4 * (k & 7))) & 15;
        const T* e0 = ep + 8 * s;
        const T* e1 = ep + 8 * s + 4;
        T tc = T(bc7_weight(cbits, ci)) * T(0.015625);
        T px[4];
        for (int c = 0; c < 3; c++) px[c] = e0[c] + (e1[c] - e0[c]) * tc;
        if (abits) {
            T ta = T(bc7_weight(abits, ai)) * T(0.015625);
            px[3] = e0[3] + (e1[3] - e0[3]) * ta;
        } else {
            px[3] = T(255);
        }
        if (rot) {
            T t = px[3];
            px[3] = px[rot - 1];
            px[rot - 1] = t;
        }
        for (int c = 0; c < 4; c++) out[k * 4 + c] = px[c];
    }
}

// Adjoint of bc7_relaxed: gep = (d out / d ep)^T g, accumulated pixel by
// pixel, channel by channel (the order the CUDA kernels use).
template <class T>
void bc7_adjoint(const uint32_t meta[8], const T g[64], T gep[24]) {
    for (int i = 0; i < 24; i++) gep[i] = T(0);
    uint32_t mode = meta[0] & 15;
    if (mode >= 8) return;
    uint32_t rot = (meta[0] >> 10) & 3, cbits = (meta[0] >> 16) & 7, abits = (meta[0] >> 20) & 7;
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t s = (meta[5] >> (2 * k)) & 3;
        uint32_t ci = (meta[1 + (k >> 3)] >> (4 * (k & 7))) & 15, ai = (meta[3 + (k >> 3)] >> (4 * (k & 7))) & 15;
        T gp[4] = {g[k * 4], g[k * 4 + 1], g[k * 4 + 2], g[k * 4 + 3]};
        if (rot) {
            T t = gp[3];
            gp[3] = gp[rot - 1];
            gp[rot - 1] = t;
        }
        int wc = bc7_weight(cbits, ci);
        T tc = T(wc) * T(0.015625), uc = T(64 - wc) * T(0.015625);
        for (int c = 0; c < 3; c++) {
            gep[8 * s + c] += gp[c] * uc;
            gep[8 * s + 4 + c] += gp[c] * tc;
        }
        if (abits) {
            int wa = bc7_weight(abits, ai);
            T ta = T(wa) * T(0.015625), ua = T(64 - wa) * T(0.015625);
            gep[8 * s + 3] += gp[3] * ua;
            gep[8 * s + 7] += gp[3] * ta;
        }
    }
}

inline void bc1_parse(const uint8_t blk[8], uint32_t meta[2], float ep[6]) {
    uint32_t c0 = blk[0] | (uint32_t)blk[1] << 8, c1 = blk[2] | (uint32_t)blk[3] << 8;
    meta[0] = c0 | c1 << 16;
    meta[1] = blk[4] | (uint32_t)blk[5] << 8 | (uint32_t)blk[6] << 16 | (uint32_t)blk[7] << 24;
    const uint32_t cs[2] = {c0, c1};
    for (int i = 0; i < 2; i++) {
        uint32_t r = (cs[i] >> 11) & 31, g = (cs[i] >> 5) & 63, b = cs[i] & 31;
        ep[3 * i] = (float)((r * 527 + 23) >> 6);  // the decoder's expansion, block.rs:137-145
        ep[3 * i + 1] = (float)((g * 259 + 33) >> 6);
        ep[3 * i + 2] = (float)((b * 527 + 23) >> 6);
    }
}

// Interpolation weight of a BC1 index; -1 marks the constant black texel.
template <class T>
T bc1_t(bool four, uint32_t idx) {
    if (idx == 0) return T(0);
    if (idx == 1) return T(1);
    if (!four) return idx == 2 ? T(0.5) : T(-1);
    return idx == 2 ? T(1) / T(3) : T(2) / T(3);
}

template <class T>
void bc1_relaxed(const uint32_t meta[2], const T ep[6], T out[64]) {
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t idx = (meta[1] >> (2 * k)) & 3;
        T t = bc1_t<T>(four, idx);
        if (t < T(0)) {
            for (int c = 0; c < 4; c++) out[k * 4 + c] = T(0);
            continue;
        }
        for (int c = 0; c < 3; c++) out[k * 4 + c] = ep[c] + (ep[3 + c] - ep[c]) * t;
        out[k * 4 + 3] = T(255);
    }
}

template <class T>
void bc1_adjoint(const uint32_t meta[2], const T g[64], T gep[6]) {
    for (int i = 0; i < 6; i++) gep[i] = T(0);
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    for (uint32_t k = 0; k < 16; k++) {
        uint32_t idx = (meta[1] >> (2 * k)) & 3;
        T t = bc1_t<T>(four, idx);
        if (t < T(0)) continue;
        T u = T(1) - t;
        for (int c = 0; c < 3; c++) {
            gep[c] += g[k * 4 + c] * u;
            gep[3 + c] += g[k * 4 + c] * t;
        }
    }
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8 as the nearest floats) on
// n parameters; b1t / b2t hold beta^t after the caller's update.
inline void adam_step(float* theta, float* m, float* v, const float* g, int n, float lr, float b1t, float b2t) {
    for (int i = 0; i < n; i++) {
        m[i] = 0.9f * m[i] + 0.1f * g[i];
        v[i] = 0.999f * v[i] + 0.001f * g[i] * g[i];
        float mh = m[i] / (1.0f - b1t);
        float vh = v[i] / (1.0f - b2t);
        theta[i] = theta[i] - lr * mh / (std::sqrt(vh) + 1e-8f);
    }
}

}  // namespace relaxed
}  // namespace oracle
