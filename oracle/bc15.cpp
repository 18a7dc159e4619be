// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Restatement of src/encode/bc1_to_5.rs (BC1-BC5 block encoders).
#include "oracle_common.h"

namespace oracle {

// bc1_to_5.rs:157-192
static void compute_covar_dc(const real block[64], real covar[6], real dc[3]) {
    for (int p = 0; p < 3; p++) {
        real acc = 0.0f;
        for (int k = 0; k < 16; k++) acc += block[k + p * 16];
        dc[p] = acc / 16.0f;
    }
    real c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, c3 = 0.0f, c4 = 0.0f, c5 = 0.0f;
    for (int k = 0; k < 16; k++) {
        real rgb0 = block[k] - dc[0];
        real rgb1 = block[k + 16] - dc[1];
        real rgb2 = block[k + 32] - dc[2];
        c0 += rgb0 * rgb0;
        c1 += rgb0 * rgb1;
        c2 += rgb0 * rgb2;
        c3 += rgb1 * rgb1;
        c4 += rgb1 * rgb2;
        c5 += rgb2 * rgb2;
    }
    covar[0] = c0;
    covar[1] = c1;
    covar[2] = c2;
    covar[3] = c3;
    covar[4] = c4;
    covar[5] = c5;
}

// bc1_to_5.rs:194-198
static void ssymv(real r[3], const real covar[6], const real a[3]) {
    r[0] = covar[0] * a[0] + covar[1] * a[1] + covar[2] * a[2];
    r[1] = covar[1] * a[0] + covar[3] * a[1] + covar[4] * a[2];
    r[2] = covar[2] * a[0] + covar[4] * a[1] + covar[5] * a[2];
}

// bc1_to_5.rs:200-223
static void compute_axis3(real axis[3], const real covar[6], int power_iterations) {
    real a[3] = {1.0f, 1.0f, 1.0f};
    for (int i = 0; i < power_iterations; i++) {
        ssymv(axis, covar, a);
        a[0] = axis[0];
        a[1] = axis[1];
        a[2] = axis[2];
        if (i % 2 == 1) {
            real norm_sq = 0.0f;
            for (int p = 0; p < 3; p++) norm_sq += axis[p] * axis[p];
            real rnorm = 1.0f / sqrt_r(norm_sq);
            for (int p = 0; p < 3; p++) a[p] *= rnorm;
        }
    }
    axis[0] = a[0];
    axis[1] = a[1];
    axis[2] = a[2];
}

// bc1_to_5.rs:225-256
static void pick_endpoints(const real block[64], real c0[3], real c1[3], const real axis[3],
                           const real dc[3]) {
    real min_dot = 256.0f * 256.0f;
    real max_dot = 0.0f;
    for (int y = 0; y < 4; y++) {
        for (int x = 0; x < 4; x++) {
            real dot = 0.0f;
            for (int p = 0; p < 3; p++) dot += (block[p * 16 + y * 4 + x] - dc[p]) * axis[p];
            min_dot = fmin_r(min_dot, dot);
            max_dot = fmax_r(max_dot, dot);
        }
    }
    if (max_dot - min_dot < 1.0f) {
        min_dot -= 0.5f;
        max_dot += 0.5f;
    }
    real norm_sq = 0.0f;
    for (int p = 0; p < 3; p++) norm_sq += axis[p] * axis[p];
    real rnorm_sq = 1.0f / norm_sq;
    for (int p = 0; p < 3; p++) {
        c0[p] = clampf_r(dc[p] + min_dot * rnorm_sq * axis[p], 0.0f, 255.0f);
        c1[p] = clampf_r(dc[p] + max_dot * rnorm_sq * axis[p], 0.0f, 255.0f);
    }
}

// bc1_to_5.rs:258-266
static void dec_rgb565(real c[3], int32_t p) {
    int32_t b5 = p & 31;
    int32_t g6 = (p >> 5) & 63;
    int32_t r5 = (p >> 11) & 31;
    c[0] = (real)((r5 << 3) + (r5 >> 2));
    c[1] = (real)((g6 << 2) + (g6 >> 4));
    c[2] = (real)((b5 << 3) + (b5 >> 2));
}

// bc1_to_5.rs:268-278
static int32_t enc_rgb565(const real c[3]) {
    int32_t r = f2i(c[0]);
    int32_t g = f2i(c[1]);
    int32_t b = f2i(c[2]);
    int32_t r5 = (r * 31 + 128 + ((r * 31) >> 8)) >> 8;
    int32_t g6 = (g * 63 + 128 + ((g * 63) >> 8)) >> 8;
    int32_t b5 = (b * 31 + 128 + ((b * 31) >> 8)) >> 8;
    return (r5 << 11) + (g6 << 5) + b5;
}

// bc1_to_5.rs:280-321
static uint32_t fast_quant(const real block[64], int32_t p0, int32_t p1) {
    real c0[3], c1[3];
    dec_rgb565(c0, p0);
    dec_rgb565(c1, p1);
    real dir[3];
    for (int p = 0; p < 3; p++) dir[p] = c1[p] - c0[p];
    real sq_norm = 0.0f;
    for (int p = 0; p < 3; p++) sq_norm += dir[p] * dir[p];
    real rsq_norm = 1.0f / sq_norm;
    for (int p = 0; p < 3; p++) dir[p] *= rsq_norm * 3.0f;
    real bias = 0.5f;
    for (int p = 0; p < 3; p++) bias -= c0[p] * dir[p];
    uint32_t bits = 0;
    uint32_t scaler = 1;
    for (int k = 0; k < 16; k++) {
        real dot = 0.0f;
        for (int p = 0; p < 3; p++) dot += block[k + p * 16] * dir[p];
        int32_t q = clampi_r(f2i(dot + bias), 0, 3);
        bits += (uint32_t)q * scaler;
        scaler *= 4u;
    }
    return bits;
}

// bc1_to_5.rs:323-374
static void bc1_refine(const real block[64], int32_t pe[2], uint32_t bits, const real dc[3]) {
    real c0[3], c1[3];
    if ((bits ^ (bits * 4u)) < 4) {
        for (int p = 0; p < 3; p++) {
            c0[p] = dc[p];
            c1[p] = dc[p];
        }
    } else {
        real atb1[3] = {0.0f, 0.0f, 0.0f};
        real sum_q = 0.0f;
        real sum_qq = 0.0f;
        uint32_t shifted = bits;
        for (int k = 0; k < 16; k++) {
            real q = (real)(shifted & 3);
            shifted >>= 2;
            real x = 3.0f - q;
            sum_q += q;
            sum_qq += q * q;
            for (int p = 0; p < 3; p++) atb1[p] += x * block[k + p * 16];
        }
        real sum[3], atb2[3];
        for (int p = 0; p < 3; p++) {
            sum[p] = dc[p] * 16.0f;
            atb2[p] = 3.0f * sum[p] - atb1[p];
        }
        real cxx = 16.0f * 9.0f - 2.0f * 3.0f * sum_q + sum_qq;
        real cyy = sum_qq;
        real cxy = 3.0f * sum_q - sum_qq;
        real scale = 3.0f * (1.0f / (cxx * cyy - cxy * cxy));
        for (int p = 0; p < 3; p++) {
            c0[p] = (atb1[p] * cyy - atb2[p] * cxy) * scale;
            c1[p] = (atb2[p] * cxx - atb1[p] * cxy) * scale;
            c0[p] = clampf_r(c0[p], 0.0f, 255.0f);
            c1[p] = clampf_r(c1[p], 0.0f, 255.0f);
        }
    }
    pe[0] = enc_rgb565(c0);
    pe[1] = enc_rgb565(c1);
}

// bc1_to_5.rs:376-384
static uint32_t fix_qbits(uint32_t qbits) {
    const uint32_t mask_01b = 0x55555555u;
    const uint32_t mask_10b = 0xAAAAAAAAu;
    uint32_t qbits0 = qbits & mask_01b;
    uint32_t qbits1 = qbits & mask_10b;
    return (qbits1 >> 1) + (qbits1 ^ (qbits0 << 1));
}

// bc1_to_5.rs:386-429
void bc1_core(const real block[64], uint32_t data[2]) {
    const int power_iterations = 4;
    const int refine_iterations = 1;
    real covar[6], dc[3];
    compute_covar_dc(block, covar, dc);
    const real eps = 1.1920929e-7f;  // f32::EPSILON
    covar[0] += eps;
    covar[3] += eps;
    covar[5] += eps;
    real axis[3];
    compute_axis3(axis, covar, power_iterations);
    real c0[3], c1[3];
    pick_endpoints(block, c0, c1, axis, dc);
    int32_t p[2];
    p[0] = enc_rgb565(c0);
    p[1] = enc_rgb565(c1);
    if (p[0] < p[1]) {
        int32_t t = p[0];
        p[0] = p[1];
        p[1] = t;
    }
    data[0] = ((uint32_t)p[1] << 16) | (uint32_t)p[0];
    data[1] = fast_quant(block, p[0], p[1]);
    for (int it = 0; it < refine_iterations; it++) {
        bc1_refine(block, p, data[1], dc);
        if (p[0] < p[1]) {
            int32_t t = p[0];
            p[0] = p[1];
            p[1] = t;
        }
        data[0] = ((uint32_t)p[1] << 16) | (uint32_t)p[0];
        data[1] = fast_quant(block, p[0], p[1]);
    }
    data[1] = fix_qbits(data[1]);
}

// bc1_to_5.rs:431-472
void bc3_alpha(const real block[64], uint32_t data[2]) {
    real ep[2] = {255.0f, 0.0f};
    for (int k = 0; k < 16; k++) {
        ep[0] = fmin_r(ep[0], block[48 + k]);
        ep[1] = fmax_r(ep[1], block[48 + k]);
    }
    if (ep[0] == ep[1]) ep[1] = ep[0] + 0.1f;
    uint32_t qblock[2] = {0, 0};
    real scale = 7.0f / (ep[1] - ep[0]);
    for (int k = 0; k < 16; k++) {
        real v = block[48 + k];
        real proj = (v - ep[0]) * scale + 0.5f;
        int32_t q = clampi_r(f2i(proj), 0, 7);
        q = 7 - q;
        if (q > 0) q += 1;
        if (q == 8) q = 1;
        qblock[k / 8] |= ((uint32_t)q) << ((k % 8) * 3);
    }
    data[0] = (clampu_r(f2u(ep[0]), 0, 255) << 8) | clampu_r(f2u(ep[1]), 0, 255);
    data[0] |= qblock[0] << 16;
    data[1] = qblock[0] >> 16;
    data[1] |= qblock[1] << 8;
}

}  // namespace oracle

#ifndef ORACLE_COUNT_OPS
// ---- gradient endpoint refinement (no reference counterpart) -------------------
//
// BC1 counterpart of oracle_bc7_refine_block: Adam on the relaxed decode's RGB
// MSE, re-quantisation with enc_rgb565 (bc1_to_5.rs:268-278) and the block's
// fixed indices. A four-colour block whose endpoints come out in the wrong
// order is swapped with indices 0<->1, 2<->3 (as the encoder orders them,
// bc1_to_5.rs:406-409); equal endpoints would decode in the three-colour mode,
// so every index then points at endpoint 0. A three-colour block keeps
// colour0 <= colour1 (indices 0<->1 swapped). Kept only on a strictly lower
// exact RGB error.
#include "oracle_decode.h"
#include "oracle_relaxed.h"

namespace oracle {
static void bc1_requant_code(const uint32_t meta[2], const float theta[6], uint32_t out[2]) {
    real c0[3], c1[3];
    for (int c = 0; c < 3; c++) {
        c0[c] = clampf_r(theta[c], 0.0f, 255.0f);
        c1[c] = clampf_r(theta[3 + c], 0.0f, 255.0f);
    }
    int32_t p0 = enc_rgb565(c0), p1 = enc_rgb565(c1);
    uint32_t idx = meta[1];
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    if (four) {
        if (p0 < p1) {
            int32_t t = p0;
            p0 = p1;
            p1 = t;
            idx ^= 0x55555555u;
        } else if (p0 == p1) {
            idx = 0;
        }
    } else if (p0 > p1) {
        int32_t t = p0;
        p0 = p1;
        p1 = t;
        idx ^= ~(idx >> 1) & 0x55555555u;
    }
    out[0] = (uint32_t)p0 | (uint32_t)p1 << 16;
    out[1] = idx;
}

static uint32_t bc1_exact_err(const uint32_t words[2], const uint8_t src[64]) {
    uint8_t bytes[8], px[64];
    std::memcpy(bytes, words, 8);
    decode_block_bc1(bytes, px, 16);
    uint32_t err = 0;
    for (int k = 0; k < 16; k++)
        for (int c = 0; c < 3; c++) {
            int d = (int)px[k * 4 + c] - (int)src[k * 4 + c];
            err += (uint32_t)(d * d);
        }
    return err;
}
}  // namespace oracle

extern "C" void oracle_bc1_refine_block(uint8_t blk[8], const uint8_t src[64], uint32_t steps, float lr,
                                        float* theta_out, uint32_t errs[2]) {
    using namespace oracle;
    uint32_t meta[2], best[2];
    float theta[6], m[6] = {0}, v[6] = {0};
    relaxed::bc1_parse(blk, meta, theta);
    std::memcpy(best, blk, 8);
    uint32_t best_err = bc1_exact_err(best, src);
    errs[0] = best_err;
    float s[64], x[64], g[64], ge[6];
    for (int i = 0; i < 64; i++) s[i] = (float)src[i];
    float b1t = 1.0f, b2t = 1.0f;
    for (uint32_t it = 0; it < steps; it++) {
        relaxed::bc1_relaxed<float>(meta, theta, x);
        for (int k = 0; k < 16; k++)
            for (int c = 0; c < 4; c++) g[k * 4 + c] = c < 3 ? 2.0f * (x[k * 4 + c] - s[k * 4 + c]) : 0.0f;
        relaxed::bc1_adjoint<float>(meta, g, ge);
        b1t *= 0.9f;
        b2t *= 0.999f;
        relaxed::adam_step(theta, m, v, ge, 6, lr, b1t, b2t);
        uint32_t cand[2];
        bc1_requant_code(meta, theta, cand);
        uint32_t err = bc1_exact_err(cand, src);
        if (err < best_err) {
            best_err = err;
            std::memcpy(best, cand, 8);
        }
    }
    std::memcpy(blk, best, 8);
    errs[1] = best_err;
    if (theta_out) std::memcpy(theta_out, theta, sizeof(theta));
}
#endif
