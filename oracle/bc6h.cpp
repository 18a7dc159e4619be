// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Restatement of src/encode/bc6h.rs (BC6H unsigned-float block encoder).
#include "oracle_common.h"

namespace oracle {

namespace {

struct BC6H {  // bc6h.rs:4-17
    real block[64];
    uint32_t data[5];
    real best_err;
    real rgb_bounds[6];
    real max_span;
    uint32_t max_span_idx;
    uint32_t mode;
    uint32_t epb;
    int32_t qbounds[8];
    const BC6HSettings* settings;
};

// bc6h.rs:131-164
uint32_t get_mode_prefix(uint32_t mode) {
    static const uint32_t t[14] = {0, 1, 2, 6, 10, 14, 18, 22, 26, 30, 3, 7, 11, 15};
    return t[mode];
}

real get_span(uint32_t mode) {
    static const real t[14] = {
        0.9f * 65535.0f / 64.0f, 0.9f * 65535.0f / 4.0f, 0.8f * 65535.0f / 256.0f, -1.0f, -1.0f,
        0.9f * 65535.0f / 32.0f, 0.9f * 65535.0f / 16.0f, -1.0f, -1.0f, 65535.0f, 65535.0f,
        0.95f * 65535.0f / 8.0f, 0.95f * 65535.0f / 32.0f, 6.0f,
    };
    return t[mode];
}

uint32_t get_mode_bits(uint32_t mode) {
    static const uint32_t t[14] = {10, 7, 11, 0xFFFFFFFFu, 0xFFFFFFFFu, 9, 8, 0xFFFFFFFFu, 0xFFFFFFFFu, 6, 10, 11, 12, 16};
    return t[mode];
}

// bc6h.rs:166-173
void ep_quant_bc6h_8(BC6H& s, const real ep[8], uint32_t bits, uint32_t pairs) {
    int32_t levels = 1 << bits;
    for (uint32_t i = 0; i < 8 * pairs; i++) {
        int32_t v = f2i(ep[i] / (256.0f * 256.0f - 1.0f) * (real)(levels - 1) + 0.5f);
        s.qbounds[i] = clampi_r(v, 0, levels - 1);
    }
}

// bc6h.rs:175-197
void compute_qbounds_core(BC6H& s, const real rgb_span[3]) {
    real bounds[8] = {0};
    for (int p = 0; p < 3; p++) {
        real middle = (s.rgb_bounds[p] + s.rgb_bounds[3 + p]) / 2.0f;
        bounds[p] = middle - rgb_span[p] / 2.0f;
        bounds[4 + p] = middle + rgb_span[p] / 2.0f;
    }
    ep_quant_bc6h_8(s, bounds, s.epb, 1);
}

void compute_qbounds(BC6H& s, real span) {
    real r[3] = {span, span, span};
    compute_qbounds_core(s, r);
}

void compute_qbounds2(BC6H& s, real span, uint32_t max_span_idx) {
    real r[3] = {span, span, span};
    if (max_span_idx < 3) r[max_span_idx] *= 2.0f;
    compute_qbounds_core(s, r);
}

// bc6h.rs:199-211
uint32_t unpack_to_uf16(uint32_t v, uint32_t bits) {
    if (bits >= 15) return v;
    if (v == 0) return 0;
    if (v == (1u << bits) - 1) return 0xFFFF;
    return (v * 2 + 1) << (15 - bits);
}

// bc6h.rs:213-239
void ep_quant_dequant_bc6h(const BC6H& s, int32_t qep[24], real ep[24], uint32_t pairs) {
    uint32_t bits = s.epb;
    int32_t levels = 1 << bits;
    for (uint32_t i = 0; i < 8 * pairs; i++) {
        int32_t v = f2i(ep[i] / (256.0f * 256.0f - 1.0f) * (real)(levels - 1) + 0.5f);
        qep[i] = clampi_r(v, 0, levels - 1);
    }
    for (uint32_t i = 0; i < 2 * pairs; i++)
        for (int p = 0; p < 3; p++) qep[i * 4 + p] = clampi_r(qep[i * 4 + p], s.qbounds[p], s.qbounds[4 + p]);
    for (uint32_t i = 0; i < 8 * pairs; i++) ep[i] = (real)unpack_to_uf16((uint32_t)qep[i], bits);
}

inline uint32_t bit_at(int32_t v, uint32_t pos) { return (uint32_t)((v >> pos) & 1); }

// bc6h.rs:452-463
uint32_t reverse_bits(uint32_t v, uint32_t bits) {
    if (bits == 2) return (v >> 1) + (v & 1) * 2;
    // bits == 6
    uint32_t vv = (v & 0x5555) * 2 + ((v >> 1) & 0x5555);
    return (vv >> 4) + ((vv >> 2) & 3) * 4 + (vv & 3) * 16;
}

// bc6h.rs:465-791
void bc6h_pack(uint32_t packed[4], const int32_t qep[24], uint32_t mode) {
    if (mode == 0) {
        int32_t pq[16] = {0};
        for (int p = 0; p < 3; p++) {
            pq[p] = qep[p];
            pq[4 + p] = (qep[4 + p] - qep[p]) & 31;
            pq[8 + p] = (qep[8 + p] - qep[p]) & 31;
            pq[12 + p] = (qep[12 + p] - qep[p]) & 31;
        }
        uint32_t pqep[10] = {0};
        pqep[4] = (uint32_t)pq[4] + (uint32_t)(pq[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)pq[5] + (uint32_t)(pq[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)pq[6] + (uint32_t)(pq[8 + 2] & 15) * 64;
        pqep[4] += bit_at(pq[12 + 1], 4) << 5;
        pqep[5] += bit_at(pq[12 + 2], 0) << 5;
        pqep[6] += bit_at(pq[12 + 2], 1) << 5;
        pqep[8] = (uint32_t)pq[8] + bit_at(pq[12 + 2], 2) * 32;
        pqep[9] = (uint32_t)pq[12] + bit_at(pq[12 + 2], 3) * 32;
        packed[0] = get_mode_prefix(0);
        packed[0] += bit_at(pq[8 + 1], 4) << 2;
        packed[0] += bit_at(pq[8 + 2], 4) << 3;
        packed[0] += bit_at(pq[12 + 2], 4) << 4;
        packed[1] = ((uint32_t)pq[2] << 20) + ((uint32_t)pq[1] << 10) + (uint32_t)pq[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = (pqep[9] << 6) + pqep[8];
    } else if (mode == 1) {
        int32_t pq[16] = {0};
        for (int p = 0; p < 3; p++) {
            pq[p] = qep[p];
            pq[4 + p] = (qep[4 + p] - qep[p]) & 63;
            pq[8 + p] = (qep[8 + p] - qep[p]) & 63;
            pq[12 + p] = (qep[12 + p] - qep[p]) & 63;
        }
        uint32_t pqep[8] = {0};
        pqep[0] = (uint32_t)pq[0];
        pqep[0] += bit_at(pq[12 + 2], 0) << 7;
        pqep[0] += bit_at(pq[12 + 2], 1) << 8;
        pqep[0] += bit_at(pq[8 + 2], 4) << 9;
        pqep[1] = (uint32_t)pq[1];
        pqep[1] += bit_at(pq[8 + 2], 5) << 7;
        pqep[1] += bit_at(pq[12 + 2], 2) << 8;
        pqep[1] += bit_at(pq[8 + 1], 4) << 9;
        pqep[2] = (uint32_t)pq[2];
        pqep[2] += bit_at(pq[12 + 2], 3) << 7;
        pqep[2] += bit_at(pq[12 + 2], 5) << 8;
        pqep[2] += bit_at(pq[12 + 2], 4) << 9;
        pqep[4] = (uint32_t)pq[4] + (uint32_t)(pq[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)pq[5] + (uint32_t)(pq[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)pq[6] + (uint32_t)(pq[8 + 2] & 15) * 64;
        packed[0] = get_mode_prefix(1);
        packed[0] += bit_at(pq[8 + 1], 5) << 2;
        packed[0] += bit_at(pq[12 + 1], 4) << 3;
        packed[0] += bit_at(pq[12 + 1], 5) << 4;
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = ((uint32_t)pq[12] << 6) + (uint32_t)pq[8];
    } else if (mode == 2 || mode == 3 || mode == 4) {
        int32_t dq[16] = {0};
        for (uint32_t p = 0; p < 3; p++) {
            int32_t mask = (p == mode - 2) ? 31 : 15;
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & mask;
            dq[8 + p] = (qep[8 + p] - qep[p]) & mask;
            dq[12 + p] = (qep[12 + p] - qep[p]) & mask;
        }
        uint32_t pqep[10] = {0};
        pqep[0] = (uint32_t)(dq[0] & 1023);
        pqep[1] = (uint32_t)(dq[1] & 1023);
        pqep[2] = (uint32_t)(dq[2] & 1023);
        pqep[4] = (uint32_t)dq[4] + (uint32_t)(dq[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)dq[5] + (uint32_t)(dq[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)dq[6] + (uint32_t)(dq[8 + 2] & 15) * 64;
        pqep[8] = (uint32_t)dq[8];
        pqep[9] = (uint32_t)dq[12];
        if (mode == 2) {
            packed[0] = get_mode_prefix(2);
            pqep[5] += bit_at(dq[1], 10) << 4;
            pqep[6] += bit_at(dq[2], 10) << 4;
            pqep[4] += bit_at(dq[0], 10) << 5;
            pqep[5] += bit_at(dq[12 + 2], 0) << 5;
            pqep[6] += bit_at(dq[12 + 2], 1) << 5;
            pqep[8] += bit_at(dq[12 + 2], 2) << 5;
            pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        } else if (mode == 3) {
            packed[0] = get_mode_prefix(3);
            pqep[4] += bit_at(dq[0], 10) << 4;
            pqep[6] += bit_at(dq[2], 10) << 4;
            pqep[8] += bit_at(dq[12 + 2], 0) << 4;
            pqep[9] += bit_at(dq[8 + 1], 4) << 4;
            pqep[4] += bit_at(dq[12 + 1], 4) << 5;
            pqep[5] += bit_at(dq[1], 10) << 5;
            pqep[6] += bit_at(dq[12 + 2], 1) << 5;
            pqep[8] += bit_at(dq[12 + 2], 2) << 5;
            pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        } else {
            packed[0] = get_mode_prefix(4);
            pqep[4] += bit_at(dq[0], 10) << 4;
            pqep[5] += bit_at(dq[1], 10) << 4;
            pqep[8] += bit_at(dq[12 + 2], 1) << 4;
            pqep[9] += bit_at(dq[12 + 2], 4) << 4;
            pqep[4] += bit_at(dq[8 + 2], 4) << 5;
            pqep[5] += bit_at(dq[12 + 2], 0) << 5;
            pqep[6] += bit_at(dq[2], 10) << 5;
            pqep[8] += bit_at(dq[12 + 2], 2) << 5;
            pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        }
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = (pqep[9] << 6) + pqep[8];
    } else if (mode == 5) {
        int32_t dq[16] = {0};
        for (int p = 0; p < 3; p++) {
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & 31;
            dq[8 + p] = (qep[8 + p] - qep[p]) & 31;
            dq[12 + p] = (qep[12 + p] - qep[p]) & 31;
        }
        uint32_t pqep[10] = {0};
        pqep[0] = (uint32_t)dq[0];
        pqep[1] = (uint32_t)dq[1];
        pqep[2] = (uint32_t)dq[2];
        pqep[4] = (uint32_t)dq[4] + (uint32_t)(dq[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)dq[5] + (uint32_t)(dq[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)dq[6] + (uint32_t)(dq[8 + 2] & 15) * 64;
        pqep[8] = (uint32_t)dq[8];
        pqep[9] = (uint32_t)dq[12];
        pqep[0] += bit_at(dq[8 + 2], 4) << 9;
        pqep[1] += bit_at(dq[8 + 1], 4) << 9;
        pqep[2] += bit_at(dq[12 + 2], 4) << 9;
        pqep[4] += bit_at(dq[12 + 1], 4) << 5;
        pqep[5] += bit_at(dq[12 + 2], 0) << 5;
        pqep[6] += bit_at(dq[12 + 2], 1) << 5;
        pqep[8] += bit_at(dq[12 + 2], 2) << 5;
        pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        packed[0] = get_mode_prefix(5);
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = (pqep[9] << 6) + pqep[8];
    } else if (mode == 6 || mode == 7 || mode == 8) {
        int32_t dq[16] = {0};
        for (uint32_t p = 0; p < 3; p++) {
            int32_t mask = (p == mode - 6) ? 63 : 31;
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & mask;
            dq[8 + p] = (qep[8 + p] - qep[p]) & mask;
            dq[12 + p] = (qep[12 + p] - qep[p]) & mask;
        }
        uint32_t pqep[10] = {0};
        pqep[0] = (uint32_t)dq[0];
        pqep[0] += bit_at(dq[8 + 2], 4) << 9;
        pqep[1] = (uint32_t)dq[1];
        pqep[1] += bit_at(dq[8 + 1], 4) << 9;
        pqep[2] = (uint32_t)dq[2];
        pqep[2] += bit_at(dq[12 + 2], 4) << 9;
        pqep[4] = (uint32_t)dq[4] + (uint32_t)(dq[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)dq[5] + (uint32_t)(dq[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)dq[6] + (uint32_t)(dq[8 + 2] & 15) * 64;
        pqep[8] = (uint32_t)dq[8];
        pqep[9] = (uint32_t)dq[12];
        if (mode == 6) {
            packed[0] = get_mode_prefix(6);
            pqep[0] += bit_at(dq[12 + 1], 4) << 8;
            pqep[1] += bit_at(dq[12 + 2], 2) << 8;
            pqep[2] += bit_at(dq[12 + 2], 3) << 8;
            pqep[5] += bit_at(dq[12 + 2], 0) << 5;
            pqep[6] += bit_at(dq[12 + 2], 1) << 5;
        } else if (mode == 7) {
            packed[0] = get_mode_prefix(7);
            pqep[0] += bit_at(dq[12 + 2], 0) << 8;
            pqep[1] += bit_at(dq[8 + 1], 5) << 8;
            pqep[2] += bit_at(dq[12 + 1], 5) << 8;
            pqep[4] += bit_at(dq[12 + 1], 4) << 5;
            pqep[6] += bit_at(dq[12 + 2], 1) << 5;
            pqep[8] += bit_at(dq[12 + 2], 2) << 5;
            pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        } else {
            packed[0] = get_mode_prefix(8);
            pqep[0] += bit_at(dq[12 + 2], 1) << 8;
            pqep[1] += bit_at(dq[8 + 2], 5) << 8;
            pqep[2] += bit_at(dq[12 + 2], 5) << 8;
            pqep[4] += bit_at(dq[12 + 1], 4) << 5;
            pqep[5] += bit_at(dq[12 + 2], 0) << 5;
            pqep[8] += bit_at(dq[12 + 2], 2) << 5;
            pqep[9] += bit_at(dq[12 + 2], 3) << 5;
        }
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = (pqep[9] << 6) + pqep[8];
    } else if (mode == 9) {
        uint32_t pqep[10] = {0};
        pqep[0] = (uint32_t)qep[0];
        pqep[0] += bit_at(qep[12 + 1], 4) << 6;
        pqep[0] += bit_at(qep[12 + 2], 0) << 7;
        pqep[0] += bit_at(qep[12 + 2], 1) << 8;
        pqep[0] += bit_at(qep[8 + 2], 4) << 9;
        pqep[1] = (uint32_t)qep[1];
        pqep[1] += bit_at(qep[8 + 1], 5) << 6;
        pqep[1] += bit_at(qep[8 + 2], 5) << 7;
        pqep[1] += bit_at(qep[12 + 2], 2) << 8;
        pqep[1] += bit_at(qep[8 + 1], 4) << 9;
        pqep[2] = (uint32_t)qep[2];
        pqep[2] += bit_at(qep[12 + 1], 5) << 6;
        pqep[2] += bit_at(qep[12 + 2], 3) << 7;
        pqep[2] += bit_at(qep[12 + 2], 5) << 8;
        pqep[2] += bit_at(qep[12 + 2], 4) << 9;
        pqep[4] = (uint32_t)qep[4] + (uint32_t)(qep[8 + 1] & 15) * 64;
        pqep[5] = (uint32_t)qep[5] + (uint32_t)(qep[12 + 1] & 15) * 64;
        pqep[6] = (uint32_t)qep[6] + (uint32_t)(qep[8 + 2] & 15) * 64;
        packed[0] = get_mode_prefix(9);
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
        packed[3] = (uint32_t)(qep[12] << 6) + (uint32_t)qep[8];
    } else if (mode == 10) {
        packed[0] = get_mode_prefix(10);
        packed[1] = (uint32_t)(qep[2] << 20) + (uint32_t)(qep[1] << 10) + (uint32_t)qep[0];
        packed[2] = (uint32_t)(qep[6] << 20) + (uint32_t)(qep[5] << 10) + (uint32_t)qep[4];
    } else if (mode == 11) {
        int32_t dq[8] = {0};
        for (int p = 0; p < 3; p++) {
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & 511;
        }
        uint32_t pqep[10] = {0};
        pqep[0] = (uint32_t)(dq[0] & 1023);
        pqep[1] = (uint32_t)(dq[1] & 1023);
        pqep[2] = (uint32_t)(dq[2] & 1023);
        pqep[4] = (uint32_t)dq[4] + (uint32_t)(dq[0] >> 10) * 512;
        pqep[5] = (uint32_t)dq[5] + (uint32_t)(dq[1] >> 10) * 512;
        pqep[6] = (uint32_t)dq[6] + (uint32_t)(dq[2] >> 10) * 512;
        packed[0] = get_mode_prefix(11);
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
    } else if (mode == 12) {
        int32_t dq[8] = {0};
        for (int p = 0; p < 3; p++) {
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & 255;
        }
        uint32_t pqep[8] = {0};
        pqep[0] = (uint32_t)(dq[0] & 1023);
        pqep[1] = (uint32_t)(dq[1] & 1023);
        pqep[2] = (uint32_t)(dq[2] & 1023);
        pqep[4] = (uint32_t)dq[4] + reverse_bits((uint32_t)(dq[0] >> 10), 2) * 256;
        pqep[5] = (uint32_t)dq[5] + reverse_bits((uint32_t)(dq[1] >> 10), 2) * 256;
        pqep[6] = (uint32_t)dq[6] + reverse_bits((uint32_t)(dq[2] >> 10), 2) * 256;
        packed[0] = get_mode_prefix(12);
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
    } else if (mode == 13) {
        int32_t dq[8] = {0};
        for (int p = 0; p < 3; p++) {
            dq[p] = qep[p];
            dq[4 + p] = (qep[4 + p] - qep[p]) & 15;
        }
        uint32_t pqep[8] = {0};
        pqep[0] = (uint32_t)(dq[0] & 1023);
        pqep[1] = (uint32_t)(dq[1] & 1023);
        pqep[2] = (uint32_t)(dq[2] & 1023);
        pqep[4] = (uint32_t)dq[4] + reverse_bits((uint32_t)(dq[0] >> 10), 6) * 16;
        pqep[5] = (uint32_t)dq[5] + reverse_bits((uint32_t)(dq[1] >> 10), 6) * 16;
        pqep[6] = (uint32_t)dq[6] + reverse_bits((uint32_t)(dq[2] >> 10), 6) * 16;
        packed[0] = get_mode_prefix(13);
        packed[1] = (pqep[2] << 20) + (pqep[1] << 10) + pqep[0];
        packed[2] = (pqep[6] << 20) + (pqep[5] << 10) + pqep[4];
    }
}

// bc6h.rs:241-266
void bc6h_code_2p(BC6H& s, int32_t qep[24], const uint32_t qblock[2], int32_t part_id, uint32_t mode) {
    const uint32_t bits = 3;
    uint32_t flips = bc7_code_apply_swap_mode01237(qep, qblock, 1, part_id);
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t pos = 0;
    uint32_t packed[4] = {0, 0, 0, 0};
    bc6h_pack(packed, qep, mode);
    put_bits(s.data, &pos, 5, packed[0]);
    put_bits(s.data, &pos, 30, packed[1]);
    put_bits(s.data, &pos, 30, packed[2]);
    put_bits(s.data, &pos, 12, packed[3]);
    put_bits(s.data, &pos, 5, (uint32_t)part_id);
    bc7_code_qblock(s.data, &pos, qblock, bits, flips);
    bc7_code_adjust_skip_mode01237(s.data, 1, part_id);
}

// bc6h.rs:268-286
void bc6h_code_1p(BC6H& s, int32_t qep[24], uint32_t qblock[2], uint32_t mode) {
    bc7_code_apply_swap_mode456(qep, 4, qblock, 4);
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t pos = 0;
    uint32_t packed[4] = {0, 0, 0, 0};
    bc6h_pack(packed, qep, mode);
    put_bits(s.data, &pos, 5, packed[0]);
    put_bits(s.data, &pos, 30, packed[1]);
    put_bits(s.data, &pos, 30, packed[2]);
    bc7_code_qblock(s.data, &pos, qblock, 4, 0);
}

// bc6h.rs:304-324
real bc6h_enc_2p_part_fast(const BC6H& s, int32_t qep[24], uint32_t qblock[2], int32_t part_id) {
    uint32_t pattern = get_pattern(part_id);
    real ep[24] = {0};
    for (uint32_t j = 0; j < 2; j++) {
        uint32_t mask = get_pattern_mask(part_id, j);
        block_segment_core(ep + j * 8, s.block, mask, 3);
    }
    ep_quant_dequant_bc6h(s, qep, ep, 2);
    return block_quant(qblock, s.block, 3, ep, pattern, 3);
}

// bc6h.rs:326-388
void bc6h_enc_2p_list(BC6H& s, const int32_t part_list[32], uint32_t part_count) {
    if (part_count == 0) return;
    const uint32_t bits = 3, channels = 3;
    int32_t best_qep[24] = {0};
    uint32_t best_qblock[2] = {0, 0};
    int32_t best_part_id = -1;
    real best_err = INFINITY;
    for (uint32_t part = 0; part < part_count; part++) {
        int32_t part_id = part_list[part] & 31;
        int32_t qep[24] = {0};
        uint32_t qblock[2] = {0, 0};
        real err = bc6h_enc_2p_part_fast(s, qep, qblock, part_id);
        if (err < best_err) {
            std::memcpy(best_qep, qep, sizeof(int32_t) * 16);
            best_qblock[0] = qblock[0];
            best_qblock[1] = qblock[1];
            best_part_id = part_id;
            best_err = err;
        }
    }
    // Unreachable for finite inputs; avoids undefined behaviour where the
    // Rust code would panic on the -1 index.
    if (best_part_id < 0) return;
    for (uint32_t it = 0; it < s.settings->refine_iterations_2p; it++) {
        real ep[24] = {0};
        for (uint32_t j = 0; j < 2; j++) {
            uint32_t mask = get_pattern_mask(best_part_id, j);
            opt_endpoints(ep + j * 8, s.block, bits, best_qblock, mask, channels);
        }
        int32_t qep[24] = {0};
        uint32_t qblock[2] = {0, 0};
        ep_quant_dequant_bc6h(s, qep, ep, 2);
        uint32_t pattern = get_pattern(best_part_id);
        real err = block_quant(qblock, s.block, bits, ep, pattern, channels);
        if (err < best_err) {
            std::memcpy(best_qep, qep, sizeof(int32_t) * 16);
            best_qblock[0] = qblock[0];
            best_qblock[1] = qblock[1];
            best_err = err;
        }
    }
    if (best_err < s.best_err) {
        s.best_err = best_err;
        bc6h_code_2p(s, best_qep, best_qblock, best_part_id, s.mode);
    }
}

// bc6h.rs:288-302
void bc6h_enc_2p(BC6H& s) {
    real full_stats[15] = {0};
    compute_stats_masked(full_stats, s.block, 0xFFFFFFFFu, 3);
    int32_t part_list[32];
    for (int32_t part = 0; part < 32; part++) {
        uint32_t mask = get_pattern_mask(part, 0);
        real bound12 = block_pca_bound_split(s.block, mask, full_stats, 3);
        int32_t bound = f2i(bound12);
        part_list[part] = part + bound * 64;
    }
    partial_sort_list(part_list, 32, s.settings->fast_skip_threshold);
    bc6h_enc_2p_list(s, part_list, s.settings->fast_skip_threshold);
}

// bc6h.rs:390-412
void bc6h_enc_1p(BC6H& s) {
    real ep[24] = {0};
    block_segment_core(ep, s.block, 0xFFFFFFFFu, 3);
    int32_t qep[24] = {0};
    ep_quant_dequant_bc6h(s, qep, ep, 1);
    uint32_t qblock[2] = {0, 0};
    real err = block_quant(qblock, s.block, 4, ep, 0, 3);
    for (uint32_t it = 0; it < s.settings->refine_iterations_1p; it++) {
        opt_endpoints(ep, s.block, 4, qblock, 0xFFFFFFFFu, 3);
        ep_quant_dequant_bc6h(s, qep, ep, 1);
        err = block_quant(qblock, s.block, 4, ep, 0, 3);
    }
    if (err < s.best_err) {
        s.best_err = err;
        bc6h_code_1p(s, qep, qblock, s.mode);
    }
}

// bc6h.rs:414-446
void bc6h_test_mode(BC6H& s, uint32_t mode, bool enc, real margin) {
    uint32_t mode_bits = get_mode_bits(mode);
    real span = get_span(mode);
    real max_span = s.max_span;
    uint32_t max_span_idx = s.max_span_idx;
    if (max_span * margin > span) return;
    if (mode >= 10) {
        s.epb = mode_bits;
        s.mode = mode;
        compute_qbounds(s, span);
        if (enc) bc6h_enc_1p(s);
    } else if (mode <= 1 || mode == 5 || mode == 9) {
        s.epb = mode_bits;
        s.mode = mode;
        compute_qbounds(s, span);
        if (enc) bc6h_enc_2p(s);
    } else {
        s.epb = mode_bits;
        s.mode = mode + max_span_idx;
        compute_qbounds2(s, span, max_span_idx);
        if (enc) bc6h_enc_2p(s);
    }
}

// bc6h.rs:793-819
void bc6h_setup(BC6H& s) {
    for (int p = 0; p < 3; p++) {
        s.rgb_bounds[p] = (real)0xFFFF;
        s.rgb_bounds[3 + p] = 0.0f;
    }
    for (int p = 0; p < 3; p++) {
        for (int k = 0; k < 16; k++) {
            real value = (s.block[p * 16 + k] / 31.0f) * 64.0f;
            s.block[p * 16 + k] = value;
            s.rgb_bounds[p] = fmin_r(s.rgb_bounds[p], value);
            s.rgb_bounds[3 + p] = fmax_r(s.rgb_bounds[3 + p], value);
        }
    }
    s.max_span = 0.0f;
    s.max_span_idx = 0;
    for (uint32_t p = 0; p < 3; p++) {
        real span = s.rgb_bounds[3 + p] - s.rgb_bounds[p];
        if (span > s.max_span) {
            s.max_span_idx = p;
            s.max_span = span;
        }
    }
}

}  // namespace

// bc6h.rs:821-860 (compress_bc6h_core), fed by the planar block that
// load_block_interleaved_16bit (bc6h.rs:73-97) builds: f16 bit patterns as f32.
void bc6h_encode_block(const real block_in[64], const BC6HSettings* settings, uint32_t out[4]) {
    BC6H s;
    std::memcpy(s.block, block_in, sizeof(s.block));
    std::memset(s.data, 0, sizeof(s.data));
    s.best_err = INFINITY;
    for (int i = 0; i < 6; i++) s.rgb_bounds[i] = 0.0f;
    s.max_span = 0.0f;
    s.max_span_idx = 0;
    s.mode = 0;
    s.epb = 0;
    for (int i = 0; i < 8; i++) s.qbounds[i] = 0;
    s.settings = settings;

    bc6h_setup(s);
    if (settings->slow_mode != 0) {
        bc6h_test_mode(s, 0, true, 0.0f);
        bc6h_test_mode(s, 1, true, 0.0f);
        bc6h_test_mode(s, 2, true, 0.0f);
        bc6h_test_mode(s, 5, true, 0.0f);
        bc6h_test_mode(s, 6, true, 0.0f);
        bc6h_test_mode(s, 9, true, 0.0f);
        bc6h_test_mode(s, 10, true, 0.0f);
        bc6h_test_mode(s, 11, true, 0.0f);
        bc6h_test_mode(s, 12, true, 0.0f);
        bc6h_test_mode(s, 13, true, 0.0f);
    } else {
        if (settings->fast_skip_threshold > 0) {
            bc6h_test_mode(s, 9, false, 0.0f);
            if (settings->fast_mode != 0) bc6h_test_mode(s, 1, false, 1.0f);
            bc6h_test_mode(s, 6, false, 1.0f / 1.2f);
            bc6h_test_mode(s, 5, false, 1.0f / 1.2f);
            bc6h_test_mode(s, 0, false, 1.0f / 1.2f);
            bc6h_test_mode(s, 2, false, 1.0f);
            bc6h_enc_2p(s);
            if (settings->fast_mode == 0) bc6h_test_mode(s, 1, true, 0.0f);
        }
        bc6h_test_mode(s, 10, false, 0.0f);
        bc6h_test_mode(s, 11, false, 1.0f);
        bc6h_test_mode(s, 12, false, 1.0f);
        bc6h_test_mode(s, 13, false, 1.0f);
        bc6h_enc_1p(s);
    }
    for (int i = 0; i < 4; i++) out[i] = s.data[i];
}

}  // namespace oracle
