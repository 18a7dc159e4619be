// Relaxed (differentiable) BC1 / BC7 decoding on the device: block parsing,
// the relaxed decode, its adjoint, and the Adam update. No reference
// counterpart; the block layouts are the ones the reference decoders read
// (src/decode/block.rs:124-197 for BC1, :801-1258 for BC7).
//
// Relaxation: endpoints become continuous values in 8-bit units and the
// interpolation drops the decoders' integer rounding,
//   BC7:  c = e0 + (e1 - e0) * w / 64, w = get_unquant_value(bits, index)
//         (src/encode/common.rs:6-21), rotation swap of block.rs:1238-1243;
//   BC1:  c = e0 + (e1 - e0) * t, t = 0, 1, 1/3, 2/3 for indices 0..3 in the
//         four-colour mode (block.rs:153-165); t = 0, 1, 1/2 and constant
//         transparent black for index 3 in the three-colour mode (:166-175).
// Mode, partition, rotation, index selector and indices stay fixed. With the
// parsed (integer) endpoints, floor(c + 0.5) is the decoder's output.
//
// Per-block metadata in memory:
//   BC7 meta[8]: w0 = mode (8 = reserved encoding) | partition << 4 |
//                rotation << 10 | index selector << 12 | subsets << 13 |
//                colour index bits << 16 | alpha index bits << 20;
//                w1, w2 = colour index of pixel k at bits 4(k&7) (w1: k < 8);
//                w3, w4 = alpha index, same packing; w5 = subset of pixel k
//                at bits 2k; w6 = w7 = 0.
//   BC7 endpoints[24]: slot (2 * subset + end) * 4 + channel, in the
//                decoder's channel order before the rotation swap.
//   BC1 meta[2]: w0 = colour0 | colour1 << 16 (RGB565), w1 = indices.
//   BC1 endpoints[6]: e0 R, G, B, e1 R, G, B, expanded from RGB565 the way
//                the decoder does ((v * 527 + 23) >> 6 for 5 bits, (v * 259 + 33) >> 6
//                for 6 bits).
// Relaxed outputs and their gradients are float[16][4] per block (pixel
// y * 4 + x, RGBA).
//
// Every sum runs pixel by pixel, channel by channel, without FMA contraction,
// so the results are reproducible bit for bit by a sequential CPU version.
#pragma once
#include "bc_common.cuh"
#include "bptc_decode.cuh"

namespace bcn {
namespace relax {

constexpr float kW64 = 0.015625f;  // 1/64

// ---- BC7 --------------------------------------------------------------------

BCN_DEV int bc7_weight(uint32_t bits, uint32_t index) { return w_of((int)bits, (int)index); }

BCN_DEV float sel_sub(const float* ep, uint32_t s, int slot) {
    return s == 0 ? ep[slot] : (s == 1 ? ep[8 + slot] : ep[16 + slot]);
}

// Parses one BC7 block (block.rs:801-1252 field order) into meta[0..5] and
// 8-bit endpoints.
BCN_DEV void bc7_parse(uint64_t lo, uint64_t hi, uint32_t meta[6], float ep[24]) {
#pragma unroll
    for (int i = 0; i < 6; i++) meta[i] = 0;
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
    Bits128 bs{lo, hi};
    uint32_t mode = 0;
    while (mode < 8 && bs.read(1) == 0) mode++;
    if (mode >= 8) {
        meta[0] = 8;
        return;
    }
    const uint32_t cbits_tab = 0x57757564u;  // colour endpoint bits per mode, 4 bits each
    const uint32_t abits_tab = 0x57860000u;  // alpha endpoint bits per mode
    uint32_t cb = (cbits_tab >> (4 * mode)) & 15, ab = (abits_tab >> (4 * mode)) & 15;
    uint32_t subsets = (mode == 0 || mode == 2) ? 3 : ((mode == 1 || mode == 3 || mode == 7) ? 2 : 1);
    uint32_t partition = 0, rotation = 0, isb = 0;
    if (subsets > 1) partition = bs.read(mode == 0 ? 4 : 6);
    if (mode == 4 || mode == 5) rotation = bs.read(2);
    if (mode == 4) isb = bs.read(1);
    uint32_t n = 2 * subsets;
    int e[6][4];
#pragma unroll
    for (int j = 0; j < 6; j++)
#pragma unroll
        for (int c = 0; c < 4; c++) e[j][c] = 0;
    for (int c = 0; c < 3; c++)
        for (uint32_t j = 0; j < n; j++) {
            int v = (int)bs.read(cb);
#pragma unroll
            for (int jj = 0; jj < 6; jj++)
                if (jj == (int)j) e[jj][c] = v;
        }
    if (ab)
        for (uint32_t j = 0; j < n; j++) {
            int v = (int)bs.read(ab);
#pragma unroll
            for (int jj = 0; jj < 6; jj++)
                if (jj == (int)j) e[jj][3] = v;
        }
    bool pbit = mode == 0 || mode == 1 || mode == 3 || mode == 6 || mode == 7;
    if (pbit) {
        int pb[6] = {0, 0, 0, 0, 0, 0};
        if (mode == 1) {
            pb[0] = pb[1] = (int)bs.read(1);
            pb[2] = pb[3] = (int)bs.read(1);
        } else {
            for (uint32_t j = 0; j < n; j++) {
                int b = (int)bs.read(1);
#pragma unroll
                for (int jj = 0; jj < 6; jj++)
                    if (jj == (int)j) pb[jj] = b;
            }
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
#pragma unroll
            for (int c = 0; c < 3; c++) e[j][c] = (e[j][c] << 1) | pb[j];
            if (ab) e[j][3] = (e[j][3] << 1) | pb[j];
        }
    }
    uint32_t pc = cb + (pbit ? 1 : 0), pa = ab + (pbit ? 1 : 0);
#pragma unroll
    for (int j = 0; j < 6; j++) {
        if (j >= (int)n) break;
#pragma unroll
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
    uint32_t ib = (mode == 0 || mode == 1) ? 3 : (mode == 6 ? 4 : 2);
    uint32_t ib2 = mode == 4 ? 3 : (mode == 5 ? 2 : 0);
    uint32_t prim0 = 0, prim1 = 0, sub = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t ps = subsets == 1 ? (k == 0 ? 0x80u : 0u) : partition_set(table, k);
        sub |= (ps & 3) << (2 * k);
        uint32_t q = bs.read((ps & 0x80) ? ib - 1 : ib);
        if (k < 8) prim0 |= q << (4 * k);
        else prim1 |= q << (4 * (k - 8));
    }
    uint32_t sec0 = prim0, sec1 = prim1;
    if (ib2) {
        sec0 = 0;
        sec1 = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            uint32_t q = bs.read(k == 0 ? ib2 - 1 : ib2);
            if (k < 8) sec0 |= q << (4 * k);
            else sec1 |= q << (4 * (k - 8));
        }
    }
    uint32_t cbits = ib, abits = ib;
    meta[1] = prim0;
    meta[2] = prim1;
    meta[3] = sec0;
    meta[4] = sec1;
    if (ib2 && isb) {  // colour reads the secondary (3-bit) indices, alpha the primary ones
        meta[1] = sec0;
        meta[2] = sec1;
        meta[3] = prim0;
        meta[4] = prim1;
        cbits = ib2;
        abits = ib;
    } else if (ib2) {
        abits = ib2;
    }
    if (ab == 0) {
        abits = 0;
        meta[3] = prim0;
        meta[4] = prim1;
    }
    meta[0] = mode | partition << 4 | rotation << 10 | isb << 12 | subsets << 13 | cbits << 16 | abits << 20;
    meta[5] = sub;
}

BCN_DEV uint32_t nib(uint32_t w0, uint32_t w1, int k) { return ((k < 8 ? w0 : w1) >> (4 * (k & 7))) & 15; }

// Relaxed value of pixel k (RGBA after the rotation swap).
BCN_DEV void bc7_relaxed_px(const uint32_t meta[6], const float ep[24], int k, float px[4]) {
    uint32_t mode = meta[0] & 15;
    if (mode >= 8) {
        px[0] = px[1] = px[2] = px[3] = 0.0f;
        return;
    }
    uint32_t rot = (meta[0] >> 10) & 3, cbits = (meta[0] >> 16) & 7, abits = (meta[0] >> 20) & 7;
    uint32_t s = (meta[5] >> (2 * k)) & 3;
    float tc = (float)bc7_weight(cbits, nib(meta[1], meta[2], k)) * kW64;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float e0 = sel_sub(ep, s, c), e1 = sel_sub(ep, s, 4 + c);
        px[c] = e0 + (e1 - e0) * tc;
    }
    if (abits) {
        float ta = (float)bc7_weight(abits, nib(meta[3], meta[4], k)) * kW64;
        float e0 = sel_sub(ep, s, 3), e1 = sel_sub(ep, s, 7);
        px[3] = e0 + (e1 - e0) * ta;
    } else {
        px[3] = 255.0f;
    }
    if (rot) {
        float t = px[3];
        px[3] = rot == 1 ? px[0] : (rot == 2 ? px[1] : px[2]);
        if (rot == 1) px[0] = t;
        else if (rot == 2) px[1] = t;
        else px[2] = t;
    }
}

// Adds pixel k's contribution g (d loss / d pixel, RGBA after rotation) to
// the endpoint gradient gep.
BCN_DEV void bc7_adjoint_px(const uint32_t meta[6], int k, const float g[4], float gep[24]) {
    uint32_t mode = meta[0] & 15;
    if (mode >= 8) return;
    uint32_t rot = (meta[0] >> 10) & 3, cbits = (meta[0] >> 16) & 7, abits = (meta[0] >> 20) & 7;
    uint32_t s = (meta[5] >> (2 * k)) & 3;
    float gp[4] = {g[0], g[1], g[2], g[3]};
    if (rot) {
        float t = gp[3];
        gp[3] = rot == 1 ? gp[0] : (rot == 2 ? gp[1] : gp[2]);
        if (rot == 1) gp[0] = t;
        else if (rot == 2) gp[1] = t;
        else gp[2] = t;
    }
    int wc = bc7_weight(cbits, nib(meta[1], meta[2], k));
    float tc = (float)wc * kW64, uc = (float)(64 - wc) * kW64;
    float ta = 0.0f, ua = 0.0f;
    if (abits) {
        int wa = bc7_weight(abits, nib(meta[3], meta[4], k));
        ta = (float)wa * kW64;
        ua = (float)(64 - wa) * kW64;
    }
#pragma unroll
    for (uint32_t j = 0; j < 3; j++) {
        if (j != s) continue;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            gep[8 * j + c] += gp[c] * uc;
            gep[8 * j + 4 + c] += gp[c] * tc;
        }
        if (abits) {
            gep[8 * j + 3] += gp[3] * ua;
            gep[8 * j + 7] += gp[3] * ta;
        }
    }
}

// ---- BC1 --------------------------------------------------------------------

BCN_DEV void bc1_parse(uint32_t w0, uint32_t w1, uint32_t meta[2], float ep[6]) {
    meta[0] = w0;
    meta[1] = w1;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        uint32_t c = i == 0 ? (w0 & 0xFFFF) : (w0 >> 16);
        uint32_t r = (c >> 11) & 31, g = (c >> 5) & 63, b = c & 31;
        ep[3 * i] = (float)((r * 527 + 23) >> 6);  // the decoder's expansion, block.rs:137-145
        ep[3 * i + 1] = (float)((g * 259 + 33) >> 6);
        ep[3 * i + 2] = (float)((b * 527 + 23) >> 6);
    }
}

// Interpolation weight of a BC1 index; -1 marks the constant black texel.
BCN_DEV float bc1_t(bool four, uint32_t idx) {
    if (idx == 0) return 0.0f;
    if (idx == 1) return 1.0f;
    if (!four) return idx == 2 ? 0.5f : -1.0f;
    return idx == 2 ? 1.0f / 3.0f : 2.0f / 3.0f;
}

BCN_DEV void bc1_relaxed_px(const uint32_t meta[2], const float ep[6], int k, float px[4]) {
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    float t = bc1_t(four, (meta[1] >> (2 * k)) & 3);
    if (t < 0.0f) {
        px[0] = px[1] = px[2] = px[3] = 0.0f;
        return;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) px[c] = ep[c] + (ep[3 + c] - ep[c]) * t;
    px[3] = 255.0f;
}

BCN_DEV void bc1_adjoint_px(const uint32_t meta[2], int k, const float g[4], float gep[6]) {
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    float t = bc1_t(four, (meta[1] >> (2 * k)) & 3);
    if (t < 0.0f) return;
    float u = 1.0f - t;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        gep[c] += g[c] * u;
        gep[3 + c] += g[c] * t;
    }
}

// ---- Adam (beta1 0.9, beta2 0.999, eps 1e-8 as the nearest floats) ----------

template <int N>
BCN_DEV void adam_step(float* theta, float* m, float* v, const float* g, float lr, float b1t, float b2t) {
#pragma unroll
    for (int i = 0; i < N; i++) {
        m[i] = 0.9f * m[i] + 0.1f * g[i];
        v[i] = 0.999f * v[i] + 0.001f * g[i] * g[i];
        float mh = m[i] / (1.0f - b1t);
        float vh = v[i] / (1.0f - b2t);
        theta[i] = theta[i] - lr * mh / (sqrtf(vh) + 1e-8f);
    }
}

}  // namespace relax
}  // namespace bcn
