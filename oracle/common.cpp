// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Restatement of src/encode/common.rs (shared BC6H/BC7 math). Each function
// cites the reference line it follows.
#include "oracle_common.h"
#include "oracle_tables.h"

namespace oracle {

// common.rs:6-21
int32_t get_unquant_value(uint32_t bits, int32_t index) {
    static const int32_t w2[16] = {0, 21, 43, 64, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    static const int32_t w3[16] = {0, 9, 18, 27, 37, 46, 55, 64, 0, 0, 0, 0, 0, 0, 0, 0};
    static const int32_t w4[16] = {0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64};
    if (bits == 2) return w2[index];
    if (bits == 3) return w3[index];
    return w4[index];
}

// common.rs:23-47
uint32_t get_pattern(int32_t part_id) { return kPatternTable[part_id]; }

// common.rs:49-83
uint32_t get_pattern_mask(int32_t part_id, uint32_t j) {
    uint32_t packed = kPatternMaskTable[part_id];
    uint32_t mask0 = packed & 0xFFFF;
    uint32_t mask1 = packed >> 16;
    if (j == 2) return ~mask0 & ~mask1;
    if (j == 0) return mask0;
    return mask1;
}

// common.rs:85-101
void get_skips(int32_t part_id, uint32_t skips[3]) {
    uint32_t packed = kSkipTable[part_id];
    skips[0] = 0;
    skips[1] = packed >> 4;
    skips[2] = packed & 15;
}

// common.rs:103-109
void put_bits(uint32_t data[5], uint32_t* pos, uint32_t bits, uint32_t v) {
    data[*pos / 32] |= v << (*pos % 32);
    if (*pos % 32 + bits > 32) data[*pos / 32 + 1] |= v >> (32 - *pos % 32);
    *pos += bits;
}

// common.rs:111-124
void data_shl_1bit_from(uint32_t data[5], uint32_t from_bits) {
    if (from_bits < 96) {
        uint32_t shifted = (data[2] >> 1) | (data[3] << 31);
        uint32_t mask = ((1u << (from_bits - 64)) - 1) >> 1;
        data[2] = (mask & data[2]) | (~mask & shifted);
        data[3] = (data[3] >> 1) | (data[4] << 31);
        data[4] >>= 1;
    } else if (from_bits < 128) {
        uint32_t shifted = (data[3] >> 1) | (data[4] << 31);
        uint32_t mask = ((1u << (from_bits - 96)) - 1) >> 1;
        data[3] = (mask & data[3]) | (~mask & shifted);
        data[4] >>= 1;
    }
}

// common.rs:126-140
void partial_sort_list(int32_t* list, uint32_t length, uint32_t partial_count) {
    for (uint32_t k = 0; k < partial_count; k++) {
        uint32_t best_idx = k;
        int32_t best_value = list[k];
        for (uint32_t i = k + 1; i < length; i++) {
            if (best_value > list[i]) {
                best_value = list[i];
                best_idx = i;
            }
        }
        int32_t t = list[k];
        list[k] = list[best_idx];
        list[best_idx] = t;
    }
}

// common.rs:142-205
void opt_endpoints(real* ep, const real block[64], uint32_t bits, const uint32_t qblock[2],
                   uint32_t mask, uint32_t channels) {
    int32_t levels = 1 << bits;
    real atb1[4] = {0, 0, 0, 0};
    real sum_q = 0.0f;
    real sum_qq = 0.0f;
    real sum[5] = {0, 0, 0, 0, 0};
    uint32_t mask_shifted = mask << 1;
    for (int k1 = 0; k1 < 2; k1++) {
        uint32_t qbits_shifted = qblock[k1];
        for (int k2 = 0; k2 < 8; k2++) {
            int k = k1 * 8 + k2;
            real q = (real)(qbits_shifted & 15);
            qbits_shifted >>= 4;
            mask_shifted >>= 1;
            if ((mask_shifted & 1) == 0) continue;
            real x = (real)(levels - 1) - q;
            sum_q += q;
            sum_qq += q * q;
            sum[4] += 1.0f;
            for (uint32_t p = 0; p < channels; p++) {
                sum[p] += block[k + p * 16];
                atb1[p] += x * block[k + p * 16];
            }
        }
    }
    real atb2[4] = {0, 0, 0, 0};
    for (uint32_t p = 0; p < channels; p++) atb2[p] = (real)(levels - 1) * sum[p] - atb1[p];

    real lm1 = (real)(levels - 1);
    real cxx = sum[4] * sq(lm1) - 2.0f * lm1 * sum_q + sum_qq;
    real cyy = sum_qq;
    real cxy = lm1 * sum_q - sum_qq;
    real scale = lm1 / (cxx * cyy - cxy * cxy);
    for (uint32_t p = 0; p < channels; p++) {
        ep[p] = (atb1[p] * cyy - atb2[p] * cxy) * scale;
        ep[4 + p] = (atb2[p] * cxx - atb1[p] * cxy) * scale;
    }
    if (fabs_r(cxx * cyy - cxy * cxy) < 0.001f) {
        for (uint32_t p = 0; p < channels; p++) {
            ep[p] = sum[p] / sum[4];
            ep[4 + p] = ep[p];
        }
    }
}

static void ssymv3(real a[4], const real covar[10], const real b[4]) {
    a[0] = covar[0] * b[0] + covar[1] * b[1] + covar[2] * b[2];
    a[1] = covar[1] * b[0] + covar[4] * b[1] + covar[5] * b[2];
    a[2] = covar[2] * b[0] + covar[5] * b[1] + covar[7] * b[2];
}

static void ssymv4(real a[4], const real covar[10], const real b[4]) {
    a[0] = covar[0] * b[0] + covar[1] * b[1] + covar[2] * b[2] + covar[3] * b[3];
    a[1] = covar[1] * b[0] + covar[4] * b[1] + covar[5] * b[2] + covar[6] * b[3];
    a[2] = covar[2] * b[0] + covar[5] * b[1] + covar[7] * b[2] + covar[8] * b[3];
    a[3] = covar[3] * b[0] + covar[6] * b[1] + covar[8] * b[2] + covar[9] * b[3];
}

// common.rs:260-292
void compute_axis(real axis[4], const real covar[10], uint32_t power_iterations,
                  uint32_t channels) {
    real a_vec[4] = {1.0f, 1.0f, 1.0f, 1.0f};
    for (uint32_t i = 0; i < power_iterations; i++) {
        if (channels == 3) ssymv3(axis, covar, a_vec);
        else if (channels == 4) ssymv4(axis, covar, a_vec);
        for (uint32_t p = 0; p < channels; p++) a_vec[p] = axis[p];
        if (i % 2 == 1) {
            real norm_sq = 0.0f;
            for (uint32_t p = 0; p < channels; p++) norm_sq += sq(axis[p]);
            real rnorm = 1.0f / sqrt_r(norm_sq);
            for (uint32_t p = 0; p < channels; p++) a_vec[p] *= rnorm;
        }
    }
    for (uint32_t p = 0; p < channels; p++) axis[p] = a_vec[p];
}

// common.rs:208-245
real get_pca_bound(const real covar[10], uint32_t channels) {
    const uint32_t power_iterations = 4;
    real cs[10];
    const real inv_var = 1.0f / (256.0f * 256.0f);
    for (int i = 0; i < 10; i++) cs[i] = covar[i] * inv_var;
    const real eps = sq(0.001f);
    cs[0] += eps;
    cs[4] += eps;
    cs[7] += eps;
    real axis[4] = {0, 0, 0, 0};
    compute_axis(axis, cs, power_iterations, channels);
    real a_vec[4] = {0, 0, 0, 0};
    if (channels == 3) ssymv3(a_vec, cs, axis);
    else if (channels == 4) ssymv4(a_vec, cs, axis);
    real sq_sum = 0.0f;
    for (uint32_t p = 0; p < channels; p++) sq_sum += sq(a_vec[p]);
    real lambda = sqrt_r(sq_sum);
    real bound = cs[0] + cs[4] + cs[7];
    if (channels == 4) bound += cs[9];
    bound -= lambda;
    return fmax_r(bound, 0.0f);
}

// common.rs:294-332
void compute_stats_masked(real stats[15], const real block[64], uint32_t mask,
                          uint32_t channels) {
    uint32_t mask_shifted = mask << 1;
    for (int k = 0; k < 16; k++) {
        mask_shifted >>= 1;
        real flag = (real)(mask_shifted & 1);
        real rgba[4] = {0, 0, 0, 0};
        for (uint32_t p = 0; p < channels; p++) rgba[p] = block[k + p * 16] * flag;
        stats[14] += flag;
        stats[10] += rgba[0];
        stats[11] += rgba[1];
        stats[12] += rgba[2];
        stats[0] += rgba[0] * rgba[0];
        stats[1] += rgba[0] * rgba[1];
        stats[2] += rgba[0] * rgba[2];
        stats[4] += rgba[1] * rgba[1];
        stats[5] += rgba[1] * rgba[2];
        stats[7] += rgba[2] * rgba[2];
        if (channels == 4) {
            stats[13] += rgba[3];
            stats[3] += rgba[0] * rgba[3];
            stats[6] += rgba[1] * rgba[3];
            stats[8] += rgba[2] * rgba[3];
            stats[9] += rgba[3] * rgba[3];
        }
    }
}

// common.rs:334-350
void covar_from_stats(real covar[10], const real stats[15], uint32_t channels) {
    covar[0] = stats[0] - stats[10] * stats[10] / stats[14];
    covar[1] = stats[1] - stats[10] * stats[11] / stats[14];
    covar[2] = stats[2] - stats[10] * stats[12] / stats[14];
    covar[4] = stats[4] - stats[11] * stats[11] / stats[14];
    covar[5] = stats[5] - stats[11] * stats[12] / stats[14];
    covar[7] = stats[7] - stats[12] * stats[12] / stats[14];
    if (channels == 4) {
        covar[3] = stats[3] - stats[10] * stats[13] / stats[14];
        covar[6] = stats[6] - stats[11] * stats[13] / stats[14];
        covar[8] = stats[8] - stats[12] * stats[13] / stats[14];
        covar[9] = stats[9] - stats[13] * stats[13] / stats[14];
    }
}

// common.rs:352-368
void compute_covar_dc_masked(real covar[10], real dc[4], const real block[64], uint32_t mask,
                             uint32_t channels) {
    real stats[15] = {0};
    compute_stats_masked(stats, block, mask, channels);
    for (uint32_t p = 0; p < channels; p++) dc[p] = stats[10 + p] / stats[14];
    covar_from_stats(covar, stats, channels);
}

// common.rs:370-394
void block_pca_axis(real axis[4], real dc[4], const real block[64], uint32_t mask,
                    uint32_t channels) {
    const uint32_t power_iterations = 8;
    real covar[10] = {0};
    compute_covar_dc_masked(covar, dc, block, mask, channels);
    const real inv_var = 1.0f / (256.0f * 256.0f);
    for (int i = 0; i < 10; i++) covar[i] *= inv_var;
    const real eps = sq(0.001f);
    covar[0] += eps;
    covar[4] += eps;
    covar[7] += eps;
    covar[9] += eps;
    compute_axis(axis, covar, power_iterations, channels);
}

// common.rs:396-420
real block_pca_bound_split(const real block[64], uint32_t mask, const real full_stats[15],
                            uint32_t channels) {
    real stats[15] = {0};
    compute_stats_masked(stats, block, mask, channels);
    real covar1[10] = {0};
    covar_from_stats(covar1, stats, channels);
    for (int i = 0; i < 15; i++) stats[i] = full_stats[i] - stats[i];
    real covar2[10] = {0};
    covar_from_stats(covar2, stats, channels);
    real bound = 0.0f;
    bound += get_pca_bound(covar1, channels);
    bound += get_pca_bound(covar2, channels);
    return sqrt_r(bound) * 256.0f;
}

// common.rs:422-481
real block_quant(uint32_t qblock[2], const real block[64], uint32_t bits, const real* ep,
                  uint32_t pattern, uint32_t channels) {
    real total_err = 0.0f;
    int32_t levels = 1 << bits;
    qblock[0] = 0;
    qblock[1] = 0;
    uint32_t pattern_shifted = pattern;
    for (int k = 0; k < 16; k++) {
        uint32_t j = pattern_shifted & 3;
        pattern_shifted >>= 2;
        real proj = 0.0f;
        real div = 0.0f;
        for (uint32_t p = 0; p < channels; p++) {
            real ep_a = ep[8 * j + p];
            real ep_b = ep[8 * j + 4 + p];
            proj += (block[k + p * 16] - ep_a) * (ep_b - ep_a);
            div += sq(ep_b - ep_a);
        }
        proj /= div;
        int32_t q1 = f2i(proj * (real)levels + 0.5f);
        int32_t q1_clamped = clampi_r(q1, 1, levels - 1);
        real err0 = 0.0f;
        real err1 = 0.0f;
        int32_t w0 = get_unquant_value(bits, q1_clamped - 1);
        int32_t w1 = get_unquant_value(bits, q1_clamped);
        for (uint32_t p = 0; p < channels; p++) {
            real ep_a = ep[8 * j + p];
            real ep_b = ep[8 * j + 4 + p];
            real dec_v0 = (real)(((64 - w0) * f2i(ep_a) + w0 * f2i(ep_b) + 32) / 64);
            real dec_v1 = (real)(((64 - w1) * f2i(ep_a) + w1 * f2i(ep_b) + 32) / 64);
            err0 += sq(dec_v0 - block[k + p * 16]);
            err1 += sq(dec_v1 - block[k + p * 16]);
        }
        real best_err = err1;
        int32_t best_q = q1_clamped;
        if (err0 < err1) {
            best_err = err0;
            best_q = q1_clamped - 1;
        }
        qblock[k / 8] |= ((uint32_t)best_q) << (4 * (k % 8));
        total_err += best_err;
    }
    return total_err;
}

// common.rs:483-518
void block_segment_core(real* ep, const real block[64], uint32_t mask, uint32_t channels) {
    real axis[4] = {0, 0, 0, 0};
    real dc[4] = {0, 0, 0, 0};
    block_pca_axis(axis, dc, block, mask, channels);
    real ext[2] = {INFINITY, -INFINITY};
    uint32_t mask_shifted = mask << 1;
    for (int k = 0; k < 16; k++) {
        mask_shifted >>= 1;
        if ((mask_shifted & 1) == 0) continue;
        real dot = 0.0f;
        for (uint32_t p = 0; p < channels; p++) dot += axis[p] * (block[16 * p + k] - dc[p]);
        ext[0] = fmin_r(ext[0], dot);
        ext[1] = fmax_r(ext[1], dot);
    }
    if (ext[1] - ext[0] < 1.0f) {
        ext[0] -= 0.5f;
        ext[1] += 0.5f;
    }
    for (int i = 0; i < 2; i++)
        for (uint32_t p = 0; p < channels; p++) ep[4 * i + p] = ext[i] * axis[p] + dc[p];
}

// common.rs:520-547
void bc7_code_qblock(uint32_t data[5], uint32_t* qpos, const uint32_t qblock[2], uint32_t bits,
                     uint32_t flips) {
    uint32_t levels = 1u << bits;
    uint32_t flips_shifted = flips;
    for (int k1 = 0; k1 < 2; k1++) {
        uint32_t qbits_shifted = qblock[k1];
        for (int k2 = 0; k2 < 8; k2++) {
            uint32_t q = qbits_shifted & 15;
            if ((flips_shifted & 1) > 0) q = (levels - 1) - q;
            if (k1 == 0 && k2 == 0) put_bits(data, qpos, bits - 1, q);
            else put_bits(data, qpos, bits, q);
            qbits_shifted >>= 4;
            flips_shifted >>= 1;
        }
    }
}

// common.rs:549-562
void bc7_code_adjust_skip_mode01237(uint32_t data[5], uint32_t mode, int32_t part_id) {
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t skips[3];
    get_skips(part_id, skips);
    if (pairs > 2 && skips[1] < skips[2]) {
        uint32_t t = skips[1];
        skips[1] = skips[2];
        skips[2] = t;
    }
    for (uint32_t i = 1; i < pairs; i++) {
        uint32_t k = skips[i];
        data_shl_1bit_from(data, 128 + (pairs - 1) - (15 - k) * bits);
    }
}

// common.rs:564-581
void bc7_code_apply_swap_mode456(int32_t* qep, uint32_t channels, uint32_t qblock[2],
                                 uint32_t bits) {
    uint32_t levels = 1u << bits;
    if ((qblock[0] & 15) >= levels / 2) {
        for (uint32_t p = 0; p < channels; p++) {
            int32_t t = qep[p];
            qep[p] = qep[channels + p];
            qep[channels + p] = t;
        }
        for (int i = 0; i < 2; i++) qblock[i] = (0x11111111u * (levels - 1)) - qblock[i];
    }
}

// common.rs:583-613
uint32_t bc7_code_apply_swap_mode01237(int32_t qep[24], const uint32_t qblock[2], uint32_t mode,
                                       int32_t part_id) {
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t flips = 0;
    uint32_t levels = 1u << bits;
    uint32_t skips[3];
    get_skips(part_id, skips);
    for (uint32_t j = 0; j < pairs; j++) {
        uint32_t k0 = skips[j];
        uint32_t q = (qblock[k0 >> 3] << (28 - (k0 & 7) * 4)) >> 28;
        if (q >= levels / 2) {
            for (int p = 0; p < 4; p++) {
                int32_t t = qep[8 * j + p];
                qep[8 * j + p] = qep[8 * j + 4 + p];
                qep[8 * j + 4 + p] = t;
            }
            flips |= get_pattern_mask(part_id, j);
        }
    }
    return flips;
}

}  // namespace oracle
