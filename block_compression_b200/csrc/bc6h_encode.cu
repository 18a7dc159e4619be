// BC6H (unsigned float) encoder for sm_100a.
//
// Same tiling as the BC7 kernel: a CTA owns 32 consecutive blocks, lane l of
// every warp works on block l. The reference's per-block search
// (src/encode/bc6h.rs:288-860) is a sequence of "encodes", each run with a
// per-block quantisation state (mode, endpoint bits, quantisation bounds)
// chosen by bc6h_test_mode's span checks:
//   fast/basic settings: one 2-region encode in the mode the tests settle on,
//                        one 2-region encode in mode 1 (not in fast mode), and
//                        one 1-region encode;
//   slow settings:       2-region encodes in modes 0,1,2,5,6,9 and 1-region
//                        encodes in modes 10..13.
// Phases:
//   1. load + setup    f16 bit patterns -> f32, scaled by 64/31, block bounds,
//                      per-block states of every encode
//   2. bounds          32 PCA split bounds per block (mode independent, so one
//                      pass serves every 2-region encode)
//   3. top-k           ascending partial sort of the 32 bounds
//   4. search          (encode, partition) candidates spread over warps; each
//                      warp keeps a first minimum per encode
//   5. chains          refinement + coding of each 2-region encode's winner,
//                      and each 1-region encode
//   6. select          the reference's sequential strict comparisons
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <climits>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bptc_math.cuh"

namespace bcn {

// u8 sRGB -> f16 bit pattern of the linear value (bc6h.rs:20-27 then
// half::f16::from_f32), filled from the host.
__device__ uint16_t g_srgb_to_half[256];

cudaError_t set_srgb_to_half_table(const uint16_t* host) {
    return cudaMemcpyToSymbol(g_srgb_to_half, host, sizeof(g_srgb_to_half));
}

namespace bc6h {

using namespace bptc;

// Minimum resident CTAs per SM requested from the register allocator.
#ifndef BCN_BC6H_MINB
#define BCN_BC6H_MINB 3
#endif

constexpr int MAXJ = 10;  // encodes per block (slow settings)
constexpr int NW = 4;

struct Job {  // per-block quantisation state of one encode
    int mode;
    int epb;
    int qb[6];  // qbounds[0..3) and qbounds[4..7)
};

struct Smem {
    float px[48][NB];
    int keys[32][NB];
    uint8_t list[32][NB];
    int jmode[MAXJ][NB];
    int jepb[MAXJ][NB];
    int jqb[MAXJ][6][NB];
    float werr[6][NW][NB];
    int wcand[6][NW][NB];
    int winner[6][NB];
    float slot_err[MAXJ][NB];
    uint4 slot_data[MAXJ][NB];
};

// bc6h.rs:137-164
BCN_DEV float get_span(int mode) {
    switch (mode) {
        case 0: return 0.9f * 65535.0f / 64.0f;
        case 1: return 0.9f * 65535.0f / 4.0f;
        case 2: return 0.8f * 65535.0f / 256.0f;
        case 5: return 0.9f * 65535.0f / 32.0f;
        case 6: return 0.9f * 65535.0f / 16.0f;
        case 9: return 65535.0f;
        case 10: return 65535.0f;
        case 11: return 0.95f * 65535.0f / 8.0f;
        case 12: return 0.95f * 65535.0f / 32.0f;
        case 13: return 6.0f;
        default: return -1.0f;
    }
}

BCN_DEV int get_mode_bits(int mode) {
    switch (mode) {
        case 0: return 10;
        case 1: return 7;
        case 2: return 11;
        case 5: return 9;
        case 6: return 8;
        case 9: return 6;
        case 10: return 10;
        case 11: return 11;
        case 12: return 12;
        default: return 16;  // 13
    }
}

struct Setup {
    float bounds[6];
    float max_span;
    int max_span_idx;
};

// bc6h.rs:175-197 (compute_qbounds_core + ep_quant_bc6h_8 for one pair)
BCN_DEV void compute_qbounds(const Setup& su, float span, int max_span_idx_or_3, int epb, int qb[6]) {
    int levels = 1 << epb;
#pragma unroll
    for (int p = 0; p < 3; p++) {
        float s = span;
        if (p == max_span_idx_or_3) s *= 2.0f;
        float middle = (su.bounds[p] + su.bounds[3 + p]) / 2.0f;
        float lo = middle - s / 2.0f, hi = middle + s / 2.0f;
        qb[p] = clampi((int)(div_const<65535>(lo) * (float)(levels - 1) + 0.5f), 0, levels - 1);
        qb[3 + p] = clampi((int)(div_const<65535>(hi) * (float)(levels - 1) + 0.5f), 0, levels - 1);
    }
}

// bc6h_test_mode (bc6h.rs:414-446) without the encode call: returns whether
// the mode passed and updates the state.
BCN_DEV bool test_mode(const Setup& su, int mode, float margin, Job& st) {
    float span = get_span(mode);
    if (su.max_span * margin > span) return false;
    st.epb = get_mode_bits(mode);
    if (mode >= 10 || mode <= 1 || mode == 5 || mode == 9) {
        st.mode = mode;
        compute_qbounds(su, span, 3, st.epb, st.qb);
    } else {
        st.mode = mode + su.max_span_idx;
        compute_qbounds(su, span, su.max_span_idx, st.epb, st.qb);
    }
    return true;
}

// bc6h.rs:199-211
BCN_DEV int unpack_to_uf16(int v, int bits) {
    if (bits >= 15) return v;
    if (v == 0) return 0;
    if (v == (1 << bits) - 1) return 0xFFFF;
    return (v * 2 + 1) << (15 - bits);
}

// bc6h.rs:213-239 over PAIRS pairs (channel 3 is never coded nor in an error).
template <int PAIRS>
BCN_DEV void quant_dequant(int qep[24], float ep[24], int epb, const int qb[6]) {
    int levels = 1 << epb;
#pragma unroll
    for (int i = 0; i < 2 * PAIRS; i++)
#pragma unroll
        for (int p = 0; p < 3; p++) {
            int q = clampi((int)(div_const<65535>(ep[i * 4 + p]) * (float)(levels - 1) + 0.5f), 0, levels - 1);
            q = clampi(q, qb[p], qb[3 + p]);
            qep[i * 4 + p] = q;
            ep[i * 4 + p] = (float)unpack_to_uf16(q, epb);
        }
}

BCN_DEV uint32_t bit_at(int v, int pos) { return (uint32_t)((v >> pos) & 1); }

BCN_DEV uint32_t reverse_bits(uint32_t v, int bits) {
    if (bits == 2) return (v >> 1) + (v & 1) * 2;
    uint32_t vv = (v & 0x5555) * 2 + ((v >> 1) & 0x5555);
    return (vv >> 4) + ((vv >> 2) & 3) * 4 + (vv & 3) * 16;
}

// bc6h.rs:465-791: endpoint packing per mode.
BCN_DEV void bc6h_pack(uint32_t packed[4], const int* qep, int mode) {
    packed[0] = packed[1] = packed[2] = packed[3] = 0;
    const uint32_t prefix[14] = {0, 1, 2, 6, 10, 14, 18, 22, 26, 30, 3, 7, 11, 15};
    // prefix[mode] without indexing the table at run time
    const uint32_t prefix_m = mode < 2 ? (uint32_t)mode : (mode < 10 ? (uint32_t)(4 * mode - 6) : (uint32_t)(4 * mode - 37));
    if (mode <= 8) {
        // Delta-coded two-region modes share the skeleton below; the masks
        // and bit placements differ per mode exactly as in the reference.
        int d[16];
        int mask_r, mask_g, mask_b;
        if (mode == 0) mask_r = mask_g = mask_b = 31;
        else if (mode == 1) mask_r = mask_g = mask_b = 63;
        else if (mode == 5) mask_r = mask_g = mask_b = 31;
        else if (mode <= 4) {
            mask_r = mode == 2 ? 31 : 15;
            mask_g = mode == 3 ? 31 : 15;
            mask_b = mode == 4 ? 31 : 15;
        } else {
            mask_r = mode == 6 ? 63 : 31;
            mask_g = mode == 7 ? 63 : 31;
            mask_b = mode == 8 ? 63 : 31;
        }
        const int mk[3] = {mask_r, mask_g, mask_b};
#pragma unroll
        for (int p = 0; p < 3; p++) {
            d[p] = qep[p];
            d[4 + p] = (qep[4 + p] - qep[p]) & mk[p];
            d[8 + p] = (qep[8 + p] - qep[p]) & mk[p];
            d[12 + p] = (qep[12 + p] - qep[p]) & mk[p];
        }
        uint32_t pq[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (mode == 0) {
            pq[4] = (uint32_t)d[4] + (uint32_t)(d[9] & 15) * 64;
            pq[5] = (uint32_t)d[5] + (uint32_t)(d[13] & 15) * 64;
            pq[6] = (uint32_t)d[6] + (uint32_t)(d[10] & 15) * 64;
            pq[4] += bit_at(d[13], 4) << 5;
            pq[5] += bit_at(d[14], 0) << 5;
            pq[6] += bit_at(d[14], 1) << 5;
            pq[8] = (uint32_t)d[8] + bit_at(d[14], 2) * 32;
            pq[9] = (uint32_t)d[12] + bit_at(d[14], 3) * 32;
            packed[0] = prefix[0] + (bit_at(d[9], 4) << 2) + (bit_at(d[10], 4) << 3) + (bit_at(d[14], 4) << 4);
            packed[1] = ((uint32_t)d[2] << 20) + ((uint32_t)d[1] << 10) + (uint32_t)d[0];
            packed[2] = (pq[6] << 20) + (pq[5] << 10) + pq[4];
            packed[3] = (pq[9] << 6) + pq[8];
        } else if (mode == 1) {
            pq[0] = (uint32_t)d[0] + (bit_at(d[14], 0) << 7) + (bit_at(d[14], 1) << 8) + (bit_at(d[10], 4) << 9);
            pq[1] = (uint32_t)d[1] + (bit_at(d[10], 5) << 7) + (bit_at(d[14], 2) << 8) + (bit_at(d[9], 4) << 9);
            pq[2] = (uint32_t)d[2] + (bit_at(d[14], 3) << 7) + (bit_at(d[14], 5) << 8) + (bit_at(d[14], 4) << 9);
            pq[4] = (uint32_t)d[4] + (uint32_t)(d[9] & 15) * 64;
            pq[5] = (uint32_t)d[5] + (uint32_t)(d[13] & 15) * 64;
            pq[6] = (uint32_t)d[6] + (uint32_t)(d[10] & 15) * 64;
            packed[0] = prefix[1] + (bit_at(d[9], 5) << 2) + (bit_at(d[13], 4) << 3) + (bit_at(d[13], 5) << 4);
            packed[1] = (pq[2] << 20) + (pq[1] << 10) + pq[0];
            packed[2] = (pq[6] << 20) + (pq[5] << 10) + pq[4];
            packed[3] = ((uint32_t)d[12] << 6) + (uint32_t)d[8];
        } else if (mode <= 4) {
            pq[0] = (uint32_t)(d[0] & 1023);
            pq[1] = (uint32_t)(d[1] & 1023);
            pq[2] = (uint32_t)(d[2] & 1023);
            pq[4] = (uint32_t)d[4] + (uint32_t)(d[9] & 15) * 64;
            pq[5] = (uint32_t)d[5] + (uint32_t)(d[13] & 15) * 64;
            pq[6] = (uint32_t)d[6] + (uint32_t)(d[10] & 15) * 64;
            pq[8] = (uint32_t)d[8];
            pq[9] = (uint32_t)d[12];
            if (mode == 2) {
                packed[0] = prefix[2];
                pq[5] += bit_at(d[1], 10) << 4;
                pq[6] += bit_at(d[2], 10) << 4;
                pq[4] += bit_at(d[0], 10) << 5;
                pq[5] += bit_at(d[14], 0) << 5;
                pq[6] += bit_at(d[14], 1) << 5;
                pq[8] += bit_at(d[14], 2) << 5;
                pq[9] += bit_at(d[14], 3) << 5;
            } else if (mode == 3) {
                packed[0] = prefix[3];
                pq[4] += bit_at(d[0], 10) << 4;
                pq[6] += bit_at(d[2], 10) << 4;
                pq[8] += bit_at(d[14], 0) << 4;
                pq[9] += bit_at(d[9], 4) << 4;
                pq[4] += bit_at(d[13], 4) << 5;
                pq[5] += bit_at(d[1], 10) << 5;
                pq[6] += bit_at(d[14], 1) << 5;
                pq[8] += bit_at(d[14], 2) << 5;
                pq[9] += bit_at(d[14], 3) << 5;
            } else {
                packed[0] = prefix[4];
                pq[4] += bit_at(d[0], 10) << 4;
                pq[5] += bit_at(d[1], 10) << 4;
                pq[8] += bit_at(d[14], 1) << 4;
                pq[9] += bit_at(d[14], 4) << 4;
                pq[4] += bit_at(d[10], 4) << 5;
                pq[5] += bit_at(d[14], 0) << 5;
                pq[6] += bit_at(d[2], 10) << 5;
                pq[8] += bit_at(d[14], 2) << 5;
                pq[9] += bit_at(d[14], 3) << 5;
            }
            packed[1] = (pq[2] << 20) + (pq[1] << 10) + pq[0];
            packed[2] = (pq[6] << 20) + (pq[5] << 10) + pq[4];
            packed[3] = (pq[9] << 6) + pq[8];
        } else if (mode == 5) {
            pq[0] = (uint32_t)d[0] + (bit_at(d[10], 4) << 9);
            pq[1] = (uint32_t)d[1] + (bit_at(d[9], 4) << 9);
            pq[2] = (uint32_t)d[2] + (bit_at(d[14], 4) << 9);
            pq[4] = (uint32_t)d[4] + (uint32_t)(d[9] & 15) * 64 + (bit_at(d[13], 4) << 5);
            pq[5] = (uint32_t)d[5] + (uint32_t)(d[13] & 15) * 64 + (bit_at(d[14], 0) << 5);
            pq[6] = (uint32_t)d[6] + (uint32_t)(d[10] & 15) * 64 + (bit_at(d[14], 1) << 5);
            pq[8] = (uint32_t)d[8] + (bit_at(d[14], 2) << 5);
            pq[9] = (uint32_t)d[12] + (bit_at(d[14], 3) << 5);
            packed[0] = prefix[5];
            packed[1] = (pq[2] << 20) + (pq[1] << 10) + pq[0];
            packed[2] = (pq[6] << 20) + (pq[5] << 10) + pq[4];
            packed[3] = (pq[9] << 6) + pq[8];
        } else {  // 6, 7, 8
            pq[0] = (uint32_t)d[0] + (bit_at(d[10], 4) << 9);
            pq[1] = (uint32_t)d[1] + (bit_at(d[9], 4) << 9);
            pq[2] = (uint32_t)d[2] + (bit_at(d[14], 4) << 9);
            pq[4] = (uint32_t)d[4] + (uint32_t)(d[9] & 15) * 64;
            pq[5] = (uint32_t)d[5] + (uint32_t)(d[13] & 15) * 64;
            pq[6] = (uint32_t)d[6] + (uint32_t)(d[10] & 15) * 64;
            pq[8] = (uint32_t)d[8];
            pq[9] = (uint32_t)d[12];
            if (mode == 6) {
                packed[0] = prefix[6];
                pq[0] += bit_at(d[13], 4) << 8;
                pq[1] += bit_at(d[14], 2) << 8;
                pq[2] += bit_at(d[14], 3) << 8;
                pq[5] += bit_at(d[14], 0) << 5;
                pq[6] += bit_at(d[14], 1) << 5;
            } else if (mode == 7) {
                packed[0] = prefix[7];
                pq[0] += bit_at(d[14], 0) << 8;
                pq[1] += bit_at(d[9], 5) << 8;
                pq[2] += bit_at(d[13], 5) << 8;
                pq[4] += bit_at(d[13], 4) << 5;
                pq[6] += bit_at(d[14], 1) << 5;
                pq[8] += bit_at(d[14], 2) << 5;
                pq[9] += bit_at(d[14], 3) << 5;
            } else {
                packed[0] = prefix[8];
                pq[0] += bit_at(d[14], 1) << 8;
                pq[1] += bit_at(d[10], 5) << 8;
                pq[2] += bit_at(d[14], 5) << 8;
                pq[4] += bit_at(d[13], 4) << 5;
                pq[5] += bit_at(d[14], 0) << 5;
                pq[8] += bit_at(d[14], 2) << 5;
                pq[9] += bit_at(d[14], 3) << 5;
            }
            packed[1] = (pq[2] << 20) + (pq[1] << 10) + pq[0];
            packed[2] = (pq[6] << 20) + (pq[5] << 10) + pq[4];
            packed[3] = (pq[9] << 6) + pq[8];
        }
    } else if (mode == 9) {
        uint32_t p0 = (uint32_t)qep[0] + (bit_at(qep[13], 4) << 6) + (bit_at(qep[14], 0) << 7) + (bit_at(qep[14], 1) << 8) +
                      (bit_at(qep[10], 4) << 9);
        uint32_t p1 = (uint32_t)qep[1] + (bit_at(qep[9], 5) << 6) + (bit_at(qep[10], 5) << 7) + (bit_at(qep[14], 2) << 8) +
                      (bit_at(qep[9], 4) << 9);
        uint32_t p2 = (uint32_t)qep[2] + (bit_at(qep[13], 5) << 6) + (bit_at(qep[14], 3) << 7) + (bit_at(qep[14], 5) << 8) +
                      (bit_at(qep[14], 4) << 9);
        uint32_t p4 = (uint32_t)qep[4] + (uint32_t)(qep[9] & 15) * 64;
        uint32_t p5 = (uint32_t)qep[5] + (uint32_t)(qep[13] & 15) * 64;
        uint32_t p6 = (uint32_t)qep[6] + (uint32_t)(qep[10] & 15) * 64;
        packed[0] = prefix[9];
        packed[1] = (p2 << 20) + (p1 << 10) + p0;
        packed[2] = (p6 << 20) + (p5 << 10) + p4;
        packed[3] = (uint32_t)(qep[12] << 6) + (uint32_t)qep[8];
    } else if (mode == 10) {
        packed[0] = prefix[10];
        packed[1] = (uint32_t)(qep[2] << 20) + (uint32_t)(qep[1] << 10) + (uint32_t)qep[0];
        packed[2] = (uint32_t)(qep[6] << 20) + (uint32_t)(qep[5] << 10) + (uint32_t)qep[4];
    } else {
        // 11, 12, 13: one region, delta-coded second endpoint
        int dm = mode == 11 ? 511 : (mode == 12 ? 255 : 15);
        uint32_t p[3], q[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            int d0 = qep[c];
            int d1 = (qep[4 + c] - qep[c]) & dm;
            p[c] = (uint32_t)(d0 & 1023);
            if (mode == 11) q[c] = (uint32_t)d1 + (uint32_t)(d0 >> 10) * 512;
            else if (mode == 12) q[c] = (uint32_t)d1 + reverse_bits((uint32_t)(d0 >> 10), 2) * 256;
            else q[c] = (uint32_t)d1 + reverse_bits((uint32_t)(d0 >> 10), 6) * 16;
        }
        packed[0] = prefix_m;
        packed[1] = (p[2] << 20) + (p[1] << 10) + p[0];
        packed[2] = (q[2] << 20) + (q[1] << 10) + q[0];
    }
}

// 2-region candidate (bc6h.rs:304-324)
BCN_DEV float eval_2p(const Blk& blk, int part_id, int epb, const int qb[6], int qep[24], uint32_t& q0, uint32_t& q1) {
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) {
        ep[i] = 0.0f;
        qep[i] = 0;
    }
    uint32_t pattern = kPartitionMap[part_id];
#pragma unroll
    for (int j = 0; j < 2; j++) block_segment<3, false>(blk, subset_mask_from_map(pattern, j), ep + 8 * j);
    quant_dequant<2>(qep, ep, epb, qb);
    return block_quant<3, 3, 2>(blk, ep, pattern, q0, q1);
}

// bc6h.rs:355-387 (refine) + bc6h_code_2p (bc6h.rs:241-266)
BCN_DEV float refine_code_2p(const Blk& blk, int part_id, const Job& st, float best_err, uint32_t iters, uint4& out) {
    int best_qep[24];
    uint32_t bq0, bq1;
    eval_2p(blk, part_id, st.epb, st.qb, best_qep, bq0, bq1);
    uint32_t pattern = kPartitionMap[part_id];
    for (uint32_t it = 0; it < iters; it++) {
        float ep[24];
#pragma unroll
        for (int i = 0; i < 24; i++) ep[i] = 0.0f;
#pragma unroll
        for (int j = 0; j < 2; j++) opt_endpoints<3, 3>(ep + 8 * j, blk, bq0, bq1, subset_mask_from_map(pattern, j));
        int qep[24];
        uint32_t q0, q1;
        quant_dequant<2>(qep, ep, st.epb, st.qb);
        float err = block_quant<3, 3, 2>(blk, ep, pattern, q0, q1);
        if (err < best_err) {
#pragma unroll
            for (int i = 0; i < 16; i++) best_qep[i] = qep[i];
            bq0 = q0;
            bq1 = q1;
            best_err = err;
        }
    }
    uint32_t flips = apply_swap_mode01237(best_qep, bq0, bq1, 1, part_id);
    uint32_t packed[4];
    bc6h_pack(packed, best_qep, st.mode);
    BitWriter bw;
    bw.clear();
    bw.put(5, packed[0]);
    bw.put(30, packed[1]);
    bw.put(30, packed[2]);
    bw.put(12, packed[3]);
    bw.put(5, (uint32_t)part_id);
    code_qblock(bw, bq0, bq1, 3, flips);
    adjust_skip_mode01237(bw.d, 1, part_id);
    out = make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
    return best_err;
}

// bc6h_enc_1p (bc6h.rs:390-412) + bc6h_code_1p (bc6h.rs:268-286)
BCN_DEV float encode_1p(const Blk& blk, const Job& st, uint32_t iters, uint4& out) {
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
    block_segment<3, false>(blk, 0xFFFFu, ep);
    int qep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) qep[i] = 0;
    quant_dequant<1>(qep, ep, st.epb, st.qb);
    uint32_t q0, q1;
    float err = block_quant<3, 4, 1>(blk, ep, 0, q0, q1);
    for (uint32_t it = 0; it < iters; it++) {
        opt_endpoints<3, 4>(ep, blk, q0, q1, 0xFFFFu);
        quant_dequant<1>(qep, ep, st.epb, st.qb);
        err = block_quant<3, 4, 1>(blk, ep, 0, q0, q1);
    }
    apply_swap_mode456(qep, 4, q0, q1, 4);
    uint32_t packed[4];
    bc6h_pack(packed, qep, st.mode);
    BitWriter bw;
    bw.clear();
    bw.put(5, packed[0]);
    bw.put(30, packed[1]);
    bw.put(30, packed[2]);
    code_qblock(bw, q0, q1, 4, 0);
    out = make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
    return err;
}

// Encode list of a settings value: kind (2 = two-region, 1 = one-region) per
// encode, in the reference's order. Uniform over the launch.
struct Plan {
    int n;
    int kind[MAXJ];
    int n2;  // number of two-region encodes (they come first)
    int k;   // partitions tried per two-region encode
};

BCN_DEV Plan make_plan(const BC6HSettingsDev& s) {
    Plan p;
    p.n = 0;
    if (s.slow_mode != 0) {
        for (int i = 0; i < 6; i++) p.kind[p.n++] = 2;
        for (int i = 0; i < 4; i++) p.kind[p.n++] = 1;
    } else {
        if (s.fast_skip_threshold > 0) {
            p.kind[p.n++] = 2;
            if (s.fast_mode == 0) p.kind[p.n++] = 2;
        }
        p.kind[p.n++] = 1;
    }
    p.n2 = 0;
    for (int i = 0; i < p.n; i++) p.n2 += p.kind[i] == 2;
    p.k = (int)s.fast_skip_threshold;
    return p;
}

__global__ void __launch_bounds__(NW * 32, BCN_BC6H_MINB) bc6h_encode_kernel(const uint8_t* __restrict__ src, size_t stride,
                                                               int source_format, uint32_t bw, uint32_t nblocks,
                                                               uint8_t* __restrict__ dst, BC6HSettingsDev S) {
    __shared__ Smem sm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile0 = blockIdx.x * NB;
    const Plan P = make_plan(S);

    // 1. load: f16 bit patterns as f32 (bc6h.rs:73-97 / 45-71)
    for (int t = threadIdx.x; t < NB * 4; t += blockDim.x) {
        int b = t & 31, y = t >> 5;
        uint32_t gi = tile0 + b;
        float v[12];
#pragma unroll
        for (int i = 0; i < 12; i++) v[i] = 0.0f;
        if (gi < nblocks) {
            uint32_t by = gi / bw, bx = gi - by * bw;
            const uint8_t* row = src + (size_t)(by * 4 + y) * stride;
            if (source_format == BC6H_SRC_RGBA16F) {
                const uint16_t* r16 = reinterpret_cast<const uint16_t*>(row) + (size_t)bx * 16;
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int c = 0; c < 3; c++) v[x * 3 + c] = (float)r16[x * 4 + c];
            } else {
                const uint8_t* r8 = row + (size_t)bx * 16;
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int c = 0; c < 3; c++) v[x * 3 + c] = (float)g_srgb_to_half[r8[x * 4 + c]];
            }
        }
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int c = 0; c < 3; c++) sm.px[c * 16 + y * 4 + x][b] = div_const<31>(v[x * 3 + c]) * 64.0f;
    }
    __syncthreads();
    const Blk blk{&sm.px[0][lane]};

    // per-block setup (bc6h.rs:793-819) and encode states (warp 0)
    if (warp == 0) {
        Setup su;
        for (int p = 0; p < 3; p++) {
            su.bounds[p] = 65535.0f;
            su.bounds[3 + p] = 0.0f;
        }
        for (int p = 0; p < 3; p++)
            for (int k = 0; k < 16; k++) {
                float value = blk(p, k);
                su.bounds[p] = fminf(su.bounds[p], value);
                su.bounds[3 + p] = fmaxf(su.bounds[3 + p], value);
            }
        su.max_span = 0.0f;
        su.max_span_idx = 0;
        for (int p = 0; p < 3; p++) {
            float span = su.bounds[3 + p] - su.bounds[p];
            if (span > su.max_span) {
                su.max_span_idx = p;
                su.max_span = span;
            }
        }
        // each encode's state goes straight to shared memory (a local array
        // indexed by the running count would live in local memory)
        int n = 0;
        auto keep = [&](const Job& j) {
            sm.jmode[n][lane] = j.mode;
            sm.jepb[n][lane] = j.epb;
#pragma unroll
            for (int i = 0; i < 6; i++) sm.jqb[n][i][lane] = j.qb[i];
            n++;
        };
        Job st;
        st.mode = 0;
        st.epb = 0;
        for (int i = 0; i < 6; i++) st.qb[i] = 0;
        if (S.slow_mode != 0) {
            // modes 0, 1, 2, 5, 6, 9 (two regions), 10..13 (one region)
            const uint64_t modes = 0xDCBA965210ull;
            for (int i = 0; i < 10; i++) {
                test_mode(su, (int)((modes >> (4 * i)) & 15), 0.0f, st);  // margin 0: always passes
                keep(st);
            }
        } else {
            if (S.fast_skip_threshold > 0) {
                test_mode(su, 9, 0.0f, st);
                if (S.fast_mode != 0) test_mode(su, 1, 1.0f, st);
                test_mode(su, 6, 1.0f / 1.2f, st);
                test_mode(su, 5, 1.0f / 1.2f, st);
                test_mode(su, 0, 1.0f / 1.2f, st);
                test_mode(su, 2, 1.0f, st);
                keep(st);
                if (S.fast_mode == 0) {
                    test_mode(su, 1, 0.0f, st);
                    keep(st);
                }
            }
            test_mode(su, 10, 0.0f, st);
            test_mode(su, 11, 1.0f, st);
            test_mode(su, 12, 1.0f, st);
            test_mode(su, 13, 1.0f, st);
            keep(st);
        }
    }

    // 2. bounds over the 32 two-region partitions (bc6h.rs:288-302)
    const bool any2 = P.n2 > 0 && P.k > 0;
    if (any2) {
        float full[15];
        stats_masked<3>(blk, 0xFFFFu, full);
        for (int part = warp; part < 32; part += NW) {
            float b12 = pca_bound_split<3>(blk, subset_mask_from_map(kPartitionMap[part], 0), full);
            sm.keys[part][lane] = part + (int)b12 * 64;
        }
    }
    __syncthreads();

    // 3. partial sort (common.rs:126-140)
    if (any2 && warp == 0) {
        for (int k = 0; k < P.k; k++) {
            int best = INT_MAX, bi = 0;
            for (int q = 0; q < 32; q++) {
                int v = sm.keys[q][lane];
                if (v < best) {
                    best = v;
                    bi = q;
                }
            }
            sm.list[k][lane] = (uint8_t)bi;
            sm.keys[bi][lane] = INT_MAX;
        }
    }
    __syncthreads();

    // 4. candidates of every two-region encode
    {
        float berr[6];
        int bc[6];
#pragma unroll
        for (int j = 0; j < 6; j++) {
            berr[j] = __int_as_float(0x7f800000);
            bc[j] = -1;
        }
        const int total = any2 ? P.n2 * P.k : 0;
        for (int item = warp; item < total; item += NW) {
            int j = item / P.k, c = item - j * P.k;
            Job st;
            st.epb = sm.jepb[j][lane];
#pragma unroll
            for (int i = 0; i < 6; i++) st.qb[i] = sm.jqb[j][i][lane];
            int qep[24];
            uint32_t q0, q1;
            float err = eval_2p(blk, sm.list[c][lane] & 31, st.epb, st.qb, qep, q0, q1);
#pragma unroll
            for (int m = 0; m < 6; m++)
                if (m == j && err < berr[m]) {
                    berr[m] = err;
                    bc[m] = c;
                }
        }
#pragma unroll
        for (int j = 0; j < 6; j++) {
            sm.werr[j][warp][lane] = berr[j];
            sm.wcand[j][warp][lane] = bc[j];
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int j = 0; j < P.n2; j++) {
            float be = __int_as_float(0x7f800000);
            int bc = -1;
            for (int w = 0; w < NW; w++) {
                float e = sm.werr[j][w][lane];
                int c = sm.wcand[j][w][lane];
                if (c >= 0 && (bc < 0 || e < be || (e == be && c < bc))) {
                    be = e;
                    bc = c;
                }
            }
            sm.winner[j][lane] = bc;
            sm.slot_err[j][lane] = be;
        }
    }
    __syncthreads();

    // 5. chains
    for (int j = warp; j < P.n; j += NW) {
        Job st;
        st.mode = sm.jmode[j][lane];
        st.epb = sm.jepb[j][lane];
#pragma unroll
        for (int i = 0; i < 6; i++) st.qb[i] = sm.jqb[j][i][lane];
        float err = __int_as_float(0x7f800000);
        uint4 data = make_uint4(0, 0, 0, 0);
        if (P.kind[j] == 2) {
            int wc = any2 ? sm.winner[j][lane] : -1;
            if (wc >= 0) err = refine_code_2p(blk, sm.list[wc][lane] & 31, st, sm.slot_err[j][lane], S.refine_iterations_2p, data);
        } else {
            err = encode_1p(blk, st, S.refine_iterations_1p, data);
        }
        sm.slot_err[j][lane] = err;
        sm.slot_data[j][lane] = data;
    }
    __syncthreads();

    // 6. select + store
    if (warp == 0) {
        float best = __int_as_float(0x7f800000);
        uint4 data = make_uint4(0, 0, 0, 0);
        for (int j = 0; j < P.n; j++) {
            float e = sm.slot_err[j][lane];
            if (e < best) {
                best = e;
                data = sm.slot_data[j][lane];
            }
        }
        uint32_t gi = tile0 + lane;
        if (gi < nblocks) {
            uint8_t* o = dst + (size_t)gi * 16;
            if (((uintptr_t)dst & 15) == 0) {
                *reinterpret_cast<uint4*>(o) = data;
            } else {
                uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
                o32[0] = data.x;
                o32[1] = data.y;
                o32[2] = data.z;
                o32[3] = data.w;
            }
        }
    }
}

}  // namespace bc6h

void launch_bc6h_encode(const void* src, size_t stride_bytes, int source_format, uint32_t bw, uint32_t bh,
                        uint8_t* dst, const BC6HSettingsDev& settings, cudaStream_t s) {
    uint32_t n = bw * bh;
    if (n == 0) return;
    uint32_t grid = (n + bptc::NB - 1) / bptc::NB;
    bc6h::bc6h_encode_kernel<<<grid, bc6h::NW * 32, 0, s>>>((const uint8_t*)src, stride_bytes, source_format, bw, n,
                                                            dst, settings);
}

}  // namespace bcn
