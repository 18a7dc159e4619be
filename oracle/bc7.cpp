// CPU oracle — TEST INFRASTRUCTURE ONLY (see oracle_common.h).
// Restatement of src/encode/bc7.rs (BC7 block encoder).
#include "oracle_common.h"

namespace oracle {

namespace {

struct Mode45Parameters {  // bc7.rs:4-12
    int32_t qep[8] = {0};
    uint32_t qblock[2] = {0, 0};
    int32_t aqep[2] = {0, 0};
    uint32_t aqblock[2] = {0, 0};
    uint32_t rotation = 0;
    uint32_t swap = 0;
};

struct BC7 {  // bc7.rs:14-36
    real block[64];
    uint32_t data[5];
    real best_err;
    real opaque_err;
    const BC7Settings* settings;
};

const uint32_t kPairsTable[8] = {3, 2, 3, 2, 1, 1, 1, 2};

// bc7.rs:97-100
int32_t unpack_to_byte(int32_t v, uint32_t bits) {
    int32_t vv = v << (8 - bits);
    return vv + (vv >> bits);
}

// bc7.rs:102-148
void ep_quant0367(int32_t* qep, const real* ep, uint32_t mode, uint32_t channels) {
    int32_t bits = mode == 0 ? 4 : (mode == 7 ? 5 : 7);
    int32_t levels = 1 << bits;
    int32_t levels2 = levels * 2 - 1;
    for (int i = 0; i < 2; i++) {
        int32_t qep_b[8];
        for (int b = 0; b < 2; b++) {
            for (int p = 0; p < 4; p++) {
                int32_t v = f2i(((ep[i * 4 + p] / 255.0f * (real)levels2 - (real)b) / 2.0f + 0.5f)) * 2 + b;
                qep_b[b * 4 + p] = clampi_r(v, b, levels2 - 1 + b);
            }
        }
        real ep_b[8];
        for (int j = 0; j < 8; j++) ep_b[j] = (real)qep_b[j];
        if (mode == 0)
            for (int j = 0; j < 8; j++) ep_b[j] = (real)unpack_to_byte(qep_b[j], 5);
        real err0 = 0.0f, err1 = 0.0f;
        for (uint32_t p = 0; p < channels; p++) {
            err0 += sq(ep[i * 4 + p] - ep_b[p]);
            err1 += sq(ep[i * 4 + p] - ep_b[4 + p]);
        }
        for (int p = 0; p < 4; p++) qep[i * 4 + p] = err0 < err1 ? qep_b[p] : qep_b[4 + p];
    }
}

// bc7.rs:150-178
void ep_quant1(int32_t* qep, const real* ep) {
    int32_t qep_b[16];
    for (int b = 0; b < 2; b++) {
        for (int i = 0; i < 8; i++) {
            int32_t v = f2i(((ep[i] / 255.0f * 127.0f - (real)b) / 2.0f + 0.5f)) * 2 + b;
            qep_b[b * 8 + i] = clampi_r(v, b, 126 + b);
        }
    }
    real ep_b[16];
    for (int k = 0; k < 16; k++) ep_b[k] = (real)unpack_to_byte(qep_b[k], 7);
    real err0 = 0.0f, err1 = 0.0f;
    for (int j = 0; j < 2; j++) {
        for (int p = 0; p < 3; p++) {
            err0 += sq(ep[j * 4 + p] - ep_b[j * 4 + p]);
            err1 += sq(ep[j * 4 + p] - ep_b[8 + j * 4 + p]);
        }
    }
    for (int i = 0; i < 8; i++) qep[i] = err0 < err1 ? qep_b[i] : qep_b[8 + i];
}

// bc7.rs:180-189
void ep_quant245(int32_t* qep, const real* ep, uint32_t mode) {
    int32_t bits = mode == 5 ? 7 : 5;
    int32_t levels = 1 << bits;
    for (int i = 0; i < 8; i++) {
        int32_t v = f2i(ep[i] / 255.0f * (real)(levels - 1) + 0.5f);
        qep[i] = clampi_r(v, 0, levels - 1);
    }
}

// bc7.rs:191-208
void ep_quant(int32_t* qep, const real* ep, uint32_t mode, uint32_t channels) {
    uint32_t pairs = kPairsTable[mode];
    if (mode == 0 || mode == 3 || mode == 6 || mode == 7) {
        for (uint32_t i = 0; i < pairs; i++) ep_quant0367(qep + i * 8, ep + i * 8, mode, channels);
    } else if (mode == 1) {
        for (uint32_t i = 0; i < pairs; i++) ep_quant1(qep + i * 8, ep + i * 8);
    } else if (mode == 2 || mode == 4 || mode == 5) {
        for (uint32_t i = 0; i < pairs; i++) ep_quant245(qep + i * 8, ep + i * 8, mode);
    }
}

// bc7.rs:210-232
void ep_dequant(real* ep, const int32_t* qep, uint32_t mode) {
    uint32_t pairs = kPairsTable[mode];
    if (mode == 3 || mode == 6) {
        for (uint32_t i = 0; i < 8 * pairs; i++) ep[i] = (real)qep[i];
    } else if (mode == 1 || mode == 5) {
        for (uint32_t i = 0; i < 8 * pairs; i++) ep[i] = (real)unpack_to_byte(qep[i], 7);
    } else if (mode == 0 || mode == 2 || mode == 4) {
        for (uint32_t i = 0; i < 8 * pairs; i++) ep[i] = (real)unpack_to_byte(qep[i], 5);
    } else if (mode == 7) {
        for (uint32_t i = 0; i < 8 * pairs; i++) ep[i] = (real)unpack_to_byte(qep[i], 6);
    }
}

// bc7.rs:234-237
void ep_quant_dequant(int32_t* qep, real* ep, uint32_t mode, uint32_t channels) {
    ep_quant(qep, ep, mode, channels);
    ep_dequant(ep, qep, mode);
}

// bc7.rs:268-276
void channel_quant_dequant(int32_t qep[2], real ep[2], uint32_t epbits) {
    int32_t elevels = 1 << epbits;
    for (int i = 0; i < 2; i++) {
        int32_t v = f2i(ep[i] / 255.0f * (real)(elevels - 1) + 0.5f);
        qep[i] = clampi_r(v, 0, elevels - 1);
        ep[i] = (real)unpack_to_byte(qep[i], epbits);
    }
}

// bc7.rs:278-320
real channel_opt_quant(uint32_t qblock[2], const real cb[16], uint32_t bits, const real ep[2]) {
    int32_t levels = 1 << bits;
    qblock[0] = 0;
    qblock[1] = 0;
    real total_err = 0.0f;
    for (int k = 0; k < 16; k++) {
        real proj = (cb[k] - ep[0]) / (ep[1] - ep[0] + 0.001f);
        int32_t q1 = f2i(proj * (real)levels + 0.5f);
        int32_t q1c = clampi_r(q1, 1, levels - 1);
        real err0 = 0.0f, err1 = 0.0f;
        int32_t w0 = get_unquant_value(bits, q1c - 1);
        int32_t w1 = get_unquant_value(bits, q1c);
        real dec_v0 = (real)(((64 - w0) * f2i(ep[0]) + w0 * f2i(ep[1]) + 32) / 64);
        real dec_v1 = (real)(((64 - w1) * f2i(ep[0]) + w1 * f2i(ep[1]) + 32) / 64);
        err0 += sq(dec_v0 - cb[k]);
        err1 += sq(dec_v1 - cb[k]);
        real best_err = err0 < err1 ? err0 : err1;
        int32_t best_q = err0 < err1 ? q1c - 1 : q1c;
        qblock[k / 8] |= ((uint32_t)best_q) << (4 * (k % 8));
        total_err += best_err;
    }
    return total_err;
}

// bc7.rs:322-369
void channel_opt_endpoints(real ep[2], const real cb[16], uint32_t bits, const uint32_t qblock[2]) {
    int32_t levels = 1 << bits;
    real atb1 = 0.0f, sum_q = 0.0f, sum_qq = 0.0f, sum = 0.0f;
    for (int k1 = 0; k1 < 2; k1++) {
        uint32_t qbits_shifted = qblock[k1];
        for (int k2 = 0; k2 < 8; k2++) {
            int k = k1 * 8 + k2;
            real q = (real)(qbits_shifted & 15);
            qbits_shifted >>= 4;
            real x = (real)(levels - 1) - q;
            sum_q += q;
            sum_qq += q * q;
            sum += cb[k];
            atb1 += x * cb[k];
        }
    }
    real lm1 = (real)(levels - 1);
    real atb2 = lm1 * sum - atb1;
    real cxx = 16.0f * sq(lm1) - 2.0f * lm1 * sum_q + sum_qq;
    real cyy = sum_qq;
    real cxy = lm1 * sum_q - sum_qq;
    real scale = lm1 / (cxx * cyy - cxy * cxy);
    ep[0] = (atb1 * cyy - atb2 * cxy) * scale;
    ep[1] = (atb2 * cxx - atb1 * cxy) * scale;
    ep[0] = clampf_r(ep[0], 0.0f, 255.0f);
    ep[1] = clampf_r(ep[1], 0.0f, 255.0f);
    if (fabs_r(cxx * cyy - cxy * cxy) < 0.001f) {
        ep[0] = sum / 16.0f;
        ep[1] = ep[0];
    }
}

// bc7.rs:239-266
real opt_channel(const BC7& s, uint32_t qblock[2], int32_t qep[2], const real cb[16], uint32_t bits,
                  uint32_t epbits) {
    real ep[2] = {255.0f, 0.0f};
    for (int k = 0; k < 16; k++) {
        ep[0] = fmin_r(ep[0], cb[k]);
        ep[1] = fmax_r(ep[1], cb[k]);
    }
    channel_quant_dequant(qep, ep, epbits);
    real err = channel_opt_quant(qblock, cb, bits, ep);
    for (uint32_t it = 0; it < s.settings->refine_iterations_channel; it++) {
        channel_opt_endpoints(ep, cb, bits, qblock);
        channel_quant_dequant(qep, ep, epbits);
        err = channel_opt_quant(qblock, cb, bits, ep);
    }
    return err;
}

// bc7.rs:371-379
void block_segment(real* ep, const real block[64], uint32_t mask, uint32_t channels) {
    block_segment_core(ep, block, mask, channels);
    for (int i = 0; i < 2; i++)
        for (uint32_t p = 0; p < channels; p++) ep[4 * i + p] = clampf_r(ep[4 * i + p], 0.0f, 255.0f);
}

// bc7.rs:381-440
void bc7_code_mode01237(BC7& s, int32_t qep[24], const uint32_t qblock[2], int32_t part_id,
                        uint32_t mode) {
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t channels = mode == 7 ? 4 : 3;
    uint32_t flips = bc7_code_apply_swap_mode01237(qep, qblock, mode, part_id);
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t pos = 0;
    put_bits(s.data, &pos, mode + 1, 1u << mode);
    if (mode == 0) put_bits(s.data, &pos, 4, (uint32_t)(part_id & 15));
    else put_bits(s.data, &pos, 6, (uint32_t)(part_id & 63));
    for (uint32_t p = 0; p < channels; p++) {
        for (uint32_t j = 0; j < pairs * 2; j++) {
            uint32_t v = (uint32_t)qep[j * 4 + p];
            if (mode == 0) put_bits(s.data, &pos, 4, v >> 1);
            else if (mode == 1) put_bits(s.data, &pos, 6, v >> 1);
            else if (mode == 2) put_bits(s.data, &pos, 5, v);
            else if (mode == 3) put_bits(s.data, &pos, 7, v >> 1);
            else if (mode == 7) put_bits(s.data, &pos, 5, v >> 1);
        }
    }
    if (mode == 1)
        for (int j = 0; j < 2; j++) put_bits(s.data, &pos, 1, (uint32_t)qep[j * 8] & 1);
    if (mode == 0 || mode == 3 || mode == 7)
        for (uint32_t j = 0; j < pairs * 2; j++) put_bits(s.data, &pos, 1, (uint32_t)qep[j * 4] & 1);
    bc7_code_qblock(s.data, &pos, qblock, bits, flips);
    bc7_code_adjust_skip_mode01237(s.data, mode, part_id);
}

// bc7.rs:442-492
void bc7_code_mode45(BC7& s, const Mode45Parameters& params, uint32_t mode) {
    int32_t qep[8];
    std::memcpy(qep, params.qep, sizeof(qep));
    uint32_t qblock[2] = {params.qblock[0], params.qblock[1]};
    int32_t aqep[2] = {params.aqep[0], params.aqep[1]};
    uint32_t aqblock[2] = {params.aqblock[0], params.aqblock[1]};
    uint32_t rotation = params.rotation;
    uint32_t swap = params.swap;
    uint32_t bits = 2;
    uint32_t abits = mode == 4 ? 3 : 2;
    uint32_t epbits = mode == 4 ? 5 : 7;
    uint32_t aepbits = mode == 4 ? 6 : 8;
    if (swap == 0) {
        bc7_code_apply_swap_mode456(qep, 4, qblock, bits);
        bc7_code_apply_swap_mode456(aqep, 1, aqblock, abits);
    } else {
        uint32_t t0 = qblock[0], t1 = qblock[1];
        qblock[0] = aqblock[0];
        qblock[1] = aqblock[1];
        aqblock[0] = t0;
        aqblock[1] = t1;
        bc7_code_apply_swap_mode456(aqep, 1, qblock, bits);
        bc7_code_apply_swap_mode456(qep, 4, aqblock, abits);
    }
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t pos = 0;
    put_bits(s.data, &pos, mode + 1, 1u << mode);
    put_bits(s.data, &pos, 2, (rotation + 1) & 3);
    if (mode == 4) put_bits(s.data, &pos, 1, swap);
    for (int p = 0; p < 3; p++) {
        put_bits(s.data, &pos, epbits, (uint32_t)qep[p]);
        put_bits(s.data, &pos, epbits, (uint32_t)qep[4 + p]);
    }
    put_bits(s.data, &pos, aepbits, (uint32_t)aqep[0]);
    put_bits(s.data, &pos, aepbits, (uint32_t)aqep[1]);
    bc7_code_qblock(s.data, &pos, qblock, bits, 0);
    bc7_code_qblock(s.data, &pos, aqblock, abits, 0);
}

// bc7.rs:494-515
void bc7_code_mode6(BC7& s, int32_t* qep, uint32_t qblock[2]) {
    bc7_code_apply_swap_mode456(qep, 4, qblock, 4);
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t pos = 0;
    put_bits(s.data, &pos, 7, 64);
    for (int p = 0; p < 4; p++) {
        put_bits(s.data, &pos, 7, (uint32_t)qep[p] >> 1);
        put_bits(s.data, &pos, 7, (uint32_t)qep[4 + p] >> 1);
    }
    put_bits(s.data, &pos, 1, (uint32_t)qep[0] & 1);
    put_bits(s.data, &pos, 1, (uint32_t)qep[4] & 1);
    bc7_code_qblock(s.data, &pos, qblock, 4, 0);
}

// bc7.rs:517-538
real bc7_enc_mode01237_part_fast(const BC7& s, int32_t qep[24], uint32_t qblock[2], int32_t part_id,
                                  uint32_t mode) {
    uint32_t pattern = get_pattern(part_id);
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t channels = mode == 7 ? 4 : 3;
    real ep[24] = {0};
    for (uint32_t j = 0; j < pairs; j++) {
        uint32_t mask = get_pattern_mask(part_id, j);
        block_segment(ep + j * 8, s.block, mask, channels);
    }
    ep_quant_dequant(qep, ep, mode, channels);
    return block_quant(qblock, s.block, bits, ep, pattern, channels);
}

// bc7.rs:540-610
void bc7_enc_mode01237(BC7& s, uint32_t mode, const int32_t part_list[64], uint32_t part_count) {
    if (part_count == 0) return;
    uint32_t bits = (mode == 0 || mode == 1) ? 3 : 2;
    uint32_t pairs = (mode == 0 || mode == 2) ? 3 : 2;
    uint32_t channels = mode == 7 ? 4 : 3;
    int32_t best_qep[24] = {0};
    uint32_t best_qblock[2] = {0, 0};
    int32_t best_part_id = -1;
    real best_err = INFINITY;
    for (uint32_t i = 0; i < part_count; i++) {
        int32_t part_id = part_list[i] & 63;
        part_id = pairs == 3 ? part_id + 64 : part_id;
        int32_t qep[24] = {0};
        uint32_t qblock[2] = {0, 0};
        real err = bc7_enc_mode01237_part_fast(s, qep, qblock, part_id, mode);
        if (err < best_err) {
            std::memcpy(best_qep, qep, sizeof(int32_t) * 8 * pairs);
            best_qblock[0] = qblock[0];
            best_qblock[1] = qblock[1];
            best_part_id = part_id;
            best_err = err;
        }
    }
    // Unreachable for finite inputs (every candidate error is finite); the
    // Rust code would panic on the -1 index, this guard avoids undefined behaviour.
    if (best_part_id < 0) return;
    uint32_t refine_iterations = s.settings->refine_iterations[mode];
    for (uint32_t it = 0; it < refine_iterations; it++) {
        real ep[24] = {0};
        for (uint32_t j = 0; j < pairs; j++) {
            uint32_t mask = get_pattern_mask(best_part_id, j);
            opt_endpoints(ep + j * 8, s.block, bits, best_qblock, mask, channels);
        }
        int32_t qep[24] = {0};
        uint32_t qblock[2] = {0, 0};
        ep_quant_dequant(qep, ep, mode, channels);
        uint32_t pattern = get_pattern(best_part_id);
        real err = block_quant(qblock, s.block, bits, ep, pattern, channels);
        if (err < best_err) {
            std::memcpy(best_qep, qep, sizeof(int32_t) * 8 * pairs);
            best_qblock[0] = qblock[0];
            best_qblock[1] = qblock[1];
            best_err = err;
        }
    }
    if (mode != 7) best_err += s.opaque_err;
    if (best_err < s.best_err) {
        s.best_err = best_err;
        bc7_code_mode01237(s, best_qep, best_qblock, best_part_id, mode);
    }
}

// bc7.rs:612-620
void bc7_enc_mode02(BC7& s) {
    int32_t part_list[64];
    for (int i = 0; i < 64; i++) part_list[i] = i;
    bc7_enc_mode01237(s, 0, part_list, 16);
    if (s.settings->skip_mode2 == 0) bc7_enc_mode01237(s, 2, part_list, 64);
}

// bc7.rs:622-655
void bc7_enc_mode13(BC7& s) {
    if (s.settings->fast_skip_threshold_mode1 == 0 && s.settings->fast_skip_threshold_mode3 == 0) return;
    real full_stats[15] = {0};
    compute_stats_masked(full_stats, s.block, 0xFFFFFFFFu, 3);
    int32_t part_list[64];
    for (int32_t part = 0; part < 64; part++) {
        uint32_t mask = get_pattern_mask(part, 0);
        real bound12 = block_pca_bound_split(s.block, mask, full_stats, 3);
        int32_t bound = f2i(bound12);
        part_list[part] = part + bound * 64;
    }
    uint32_t partial_count = s.settings->fast_skip_threshold_mode1 > s.settings->fast_skip_threshold_mode3
                                 ? s.settings->fast_skip_threshold_mode1
                                 : s.settings->fast_skip_threshold_mode3;
    partial_sort_list(part_list, 64, partial_count);
    bc7_enc_mode01237(s, 1, part_list, s.settings->fast_skip_threshold_mode1);
    bc7_enc_mode01237(s, 3, part_list, s.settings->fast_skip_threshold_mode3);
}

// bc7.rs:657-733
void bc7_enc_mode45_candidate(const BC7& s, Mode45Parameters& best_candidate, real* best_err, uint32_t mode,
                              uint32_t rotation, uint32_t swap) {
    uint32_t bits = 2;
    uint32_t abits = 2;
    uint32_t aepbits = 8;
    if (mode == 4) {
        abits = 3;
        aepbits = 6;
    }
    if (swap == 1) {
        bits = 3;
        abits = 2;
    }
    real candidate_block[64] = {0};
    for (int k = 0; k < 16; k++) {
        for (int p = 0; p < 3; p++) candidate_block[k + p * 16] = s.block[k + p * 16];
        if (rotation < 3) {
            if (s.settings->channels == 4) candidate_block[k + rotation * 16] = s.block[k + 3 * 16];
            if (s.settings->channels == 3) candidate_block[k + rotation * 16] = 255.0f;
        }
    }
    real ep[8] = {0};
    block_segment(ep, candidate_block, 0xFFFFFFFFu, 3);
    int32_t qep[8] = {0};
    ep_quant_dequant(qep, ep, mode, 3);
    uint32_t qblock[2] = {0, 0};
    real err = block_quant(qblock, candidate_block, bits, ep, 0, 3);
    uint32_t refine_iterations = s.settings->refine_iterations[mode];
    for (uint32_t it = 0; it < refine_iterations; it++) {
        opt_endpoints(ep, candidate_block, bits, qblock, 0xFFFFFFFFu, 3);
        ep_quant_dequant(qep, ep, mode, 3);
        err = block_quant(qblock, candidate_block, bits, ep, 0, 3);
    }
    real channel_data[16];
    for (int k = 0; k < 16; k++) channel_data[k] = s.block[k + rotation * 16];
    int32_t aqep[2] = {0, 0};
    uint32_t aqblock[2] = {0, 0};
    err += opt_channel(s, aqblock, aqep, channel_data, abits, aepbits);
    if (err < *best_err) {
        std::memcpy(best_candidate.qep, qep, sizeof(qep));
        best_candidate.qblock[0] = qblock[0];
        best_candidate.qblock[1] = qblock[1];
        best_candidate.aqblock[0] = aqblock[0];
        best_candidate.aqblock[1] = aqblock[1];
        best_candidate.aqep[0] = aqep[0];
        best_candidate.aqep[1] = aqep[1];
        best_candidate.rotation = rotation;
        best_candidate.swap = swap;
        *best_err = err;
    }
}

// bc7.rs:735-760
void bc7_enc_mode45(BC7& s) {
    Mode45Parameters best_candidate;
    real best_err = s.best_err;
    uint32_t channel0 = s.settings->mode45_channel0;
    for (uint32_t p = channel0; p < s.settings->channels; p++) {
        bc7_enc_mode45_candidate(s, best_candidate, &best_err, 4, p, 0);
        bc7_enc_mode45_candidate(s, best_candidate, &best_err, 4, p, 1);
    }
    if (best_err < s.best_err) {
        s.best_err = best_err;
        bc7_code_mode45(s, best_candidate, 4);
    }
    for (uint32_t p = channel0; p < s.settings->channels; p++)
        bc7_enc_mode45_candidate(s, best_candidate, &best_err, 5, p, 0);
    if (best_err < s.best_err) {
        s.best_err = best_err;
        bc7_code_mode45(s, best_candidate, 5);
    }
}

// bc7.rs:762-817
void bc7_enc_mode6(BC7& s) {
    const uint32_t mode = 6;
    const uint32_t bits = 4;
    uint32_t channels = s.settings->channels;
    real ep[8] = {0};
    block_segment(ep, s.block, 0xFFFFFFFFu, channels);
    if (channels == 3) {
        ep[3] = 255.0f;
        ep[7] = 255.0f;
    }
    int32_t qep[8] = {0};
    ep_quant_dequant(qep, ep, mode, channels);
    uint32_t qblock[2] = {0, 0};
    real err = block_quant(qblock, s.block, bits, ep, 0, channels);
    uint32_t refine_iterations = s.settings->refine_iterations[mode];
    for (uint32_t it = 0; it < refine_iterations; it++) {
        opt_endpoints(ep, s.block, bits, qblock, 0xFFFFFFFFu, channels);
        ep_quant_dequant(qep, ep, mode, channels);
        err = block_quant(qblock, s.block, bits, ep, 0, channels);
    }
    if (err < s.best_err) {
        s.best_err = err;
        bc7_code_mode6(s, qep, qblock);
    }
}

// bc7.rs:819-851
void bc7_enc_mode7(BC7& s) {
    if (s.settings->fast_skip_threshold_mode7 == 0) return;
    real full_stats[15] = {0};
    compute_stats_masked(full_stats, s.block, 0xFFFFFFFFu, s.settings->channels);
    int32_t part_list[64];
    for (int32_t part = 0; part < 64; part++) {
        uint32_t mask = get_pattern_mask(part, 0);
        real bound12 = block_pca_bound_split(s.block, mask, full_stats, s.settings->channels);
        int32_t bound = f2i(bound12);
        part_list[part] = part + bound * 64;
    }
    partial_sort_list(part_list, 64, s.settings->fast_skip_threshold_mode7);
    bc7_enc_mode01237(s, 7, part_list, s.settings->fast_skip_threshold_mode7);
}

}  // namespace

// bc7.rs:853-879 (compress_block_bc7_core + compute_opaque_err), fed by the
// planar block of load_block_interleaved_rgba (bc7.rs:38-63).
void bc7_encode_block(const real block[64], const BC7Settings* settings, uint32_t out[4]) {
    BC7 s;
    std::memcpy(s.block, block, sizeof(s.block));
    std::memset(s.data, 0, sizeof(s.data));
    s.best_err = INFINITY;
    s.settings = settings;
    if (settings->channels == 3) {
        s.opaque_err = 0.0f;
    } else {
        real err = 0.0f;
        for (int k = 0; k < 16; k++) err += sq(s.block[48 + k] - 255.0f);
        s.opaque_err = err;
    }
    if (settings->mode_selection[0] != 0) bc7_enc_mode02(s);
    if (settings->mode_selection[1] != 0) {
        bc7_enc_mode13(s);
        bc7_enc_mode7(s);
    }
    if (settings->mode_selection[2] != 0) bc7_enc_mode45(s);
    if (settings->mode_selection[3] != 0) bc7_enc_mode6(s);
    for (int i = 0; i < 4; i++) out[i] = s.data[i];
}

// bc7.rs:234-237, exported for the differential tests.
void bc7_ep_quant_dequant(int32_t* qep, real* ep, uint32_t mode, uint32_t channels) {
    ep_quant_dequant(qep, ep, mode, channels);
}

}  // namespace oracle

#ifndef ORACLE_COUNT_OPS
// ---- gradient endpoint refinement (no reference counterpart) -------------------
//
// Restatement, for the parity tests, of the BC7 refinement the CUDA kernels
// run: Adam on the relaxed decode's MSE (oracle_relaxed.h), then after every
// step the endpoints are re-quantised with the encoder's own ep_quant /
// channel_quant_dequant (bc7.rs:97-276) and coded with the block's fixed mode,
// partition, rotation, index selector and indices through bc7_code_*
// (bc7.rs:381-515, anchor swaps included). A coded block replaces the best so
// far only if its exact squared error (decoded bytes against the source) is
// strictly lower.
#include "oracle_relaxed.h"

namespace oracle {
namespace {

void bc7_requant_code(const uint32_t meta[8], const float theta[24], uint32_t channels, uint32_t out[4]) {
    uint32_t mode = meta[0] & 15, partition = (meta[0] >> 4) & 63, rotation = (meta[0] >> 10) & 3;
    uint32_t isb = (meta[0] >> 12) & 1, subsets = (meta[0] >> 13) & 3;
    real ep[24];
    for (int i = 0; i < 24; i++) ep[i] = clampf_r(theta[i], 0.0f, 255.0f);
    BC7 s;
    std::memset(s.data, 0, sizeof(s.data));
    uint32_t qblock[2] = {meta[1], meta[2]};
    if (mode == 4 || mode == 5) {
        Mode45Parameters p;
        ep_quant245(p.qep, ep, mode);
        real aep[2] = {ep[3], ep[7]};
        channel_quant_dequant(p.aqep, aep, mode == 4 ? 6 : 8);
        p.qblock[0] = meta[1];
        p.qblock[1] = meta[2];
        p.aqblock[0] = meta[3];
        p.aqblock[1] = meta[4];
        p.rotation = (rotation + 3) & 3;  // the stored field is the encoder's rotation + 1
        p.swap = isb;
        bc7_code_mode45(s, p, mode);
    } else if (mode == 6) {
        int32_t qep[8] = {0};
        ep_quant(qep, ep, 6, channels);
        bc7_code_mode6(s, qep, qblock);
    } else {
        int32_t qep[24] = {0};
        ep_quant(qep, ep, mode, mode == 7 ? 4 : 3);
        int32_t part_id = (int32_t)(subsets == 3 ? 64 + partition : partition);
        bc7_code_mode01237(s, qep, qblock, part_id, mode);
    }
    for (int i = 0; i < 4; i++) out[i] = s.data[i];
}

uint32_t bc7_exact_err(const uint32_t words[4], const uint8_t src[64], uint32_t channels) {
    uint8_t bytes[16], px[64];
    std::memcpy(bytes, words, 16);
    decode_block_bc7(bytes, px, 16);
    uint32_t err = 0;
    for (int k = 0; k < 16; k++)
        for (uint32_t c = 0; c < channels; c++) {
            int d = (int)px[k * 4 + c] - (int)src[k * 4 + c];
            err += (uint32_t)(d * d);
        }
    return err;
}

}  // namespace
}  // namespace oracle

// blk: 16 bytes, refined in place. src: the block's 16 RGBA8 source pixels
// (row-major). channels: 3 (RGB error) or 4 (RGBA). theta_out: the final
// continuous endpoints (may be NULL). errs: {error before, error after}.
extern "C" void oracle_bc7_refine_block(uint8_t blk[16], const uint8_t src[64], uint32_t channels, uint32_t steps,
                                        float lr, float* theta_out, uint32_t errs[2]) {
    using namespace oracle;
    uint32_t meta[8], best[4];
    float theta[24], m[24] = {0}, v[24] = {0};
    relaxed::bc7_parse(blk, meta, theta);
    std::memcpy(best, blk, 16);
    uint32_t best_err = bc7_exact_err(best, src, channels);
    errs[0] = best_err;
    if ((meta[0] & 15) < 8) {
        float s[64], x[64], g[64], ge[24];
        for (int i = 0; i < 64; i++) s[i] = (float)src[i];
        float b1t = 1.0f, b2t = 1.0f;
        for (uint32_t it = 0; it < steps; it++) {
            relaxed::bc7_relaxed<float>(meta, theta, x);
            for (int k = 0; k < 16; k++)
                for (uint32_t c = 0; c < 4; c++) g[k * 4 + c] = c < channels ? 2.0f * (x[k * 4 + c] - s[k * 4 + c]) : 0.0f;
            relaxed::bc7_adjoint<float>(meta, g, ge);
            b1t *= 0.9f;
            b2t *= 0.999f;
            relaxed::adam_step(theta, m, v, ge, 24, lr, b1t, b2t);
            uint32_t cand[4];
            bc7_requant_code(meta, theta, channels, cand);
            uint32_t err = bc7_exact_err(cand, src, channels);
            if (err < best_err) {
                best_err = err;
                std::memcpy(best, cand, 16);
            }
        }
    }
    std::memcpy(blk, best, 16);
    errs[1] = best_err;
    if (theta_out) std::memcpy(theta_out, theta, sizeof(theta));
}
#endif
