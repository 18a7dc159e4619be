// BC6H (unsigned float) encoder for sm_100a.
//
// Work decomposition as in the BC7 encoder: tiles of 32 consecutive blocks,
// lane l of a warp always works on block l of its tile. The reference's
// per-block search (src/encode/bc6h.rs:288-860) is a sequence of "encodes",
// each run with a per-block quantisation state (mode, endpoint bits,
// quantisation bounds) chosen by bc6h_test_mode's span checks:
//   fast/basic settings: one 2-region encode in the mode the tests settle on,
//                        one 2-region encode in mode 1 (not in fast mode), and
//                        one 1-region encode;
//   slow settings:       2-region encodes in modes 0,1,2,5,6,9 and 1-region
//                        encodes in modes 10..13.
// It runs as a pipeline of launches, each one code path (a single fused
// kernel ran at 42% issue: 164 registers, local-memory arrays, warps idle at
// the barriers between unequal phases):
//   prep     setup (bc6h.rs:793-819) and the encode states of every block,
//            the 32 PCA split bounds and the ascending top-k partition list
//   search   grid (tile, candidate group): a warp evaluates one (2-region
//            encode, partition) candidate for 32 blocks; the first minimum
//            per block and encode is kept with a 64-bit atomicMin on
//            (error bits << 32 | candidate)
//   refine2  one warp per (tile, 2-region encode): refinement of the winner
//            and coding
//   enc1     one warp per (tile, 1-region encode)
//   select   the reference's sequential strict comparisons -> 128-bit store
// Per-block state between launches lives in scratch device memory
// (bc6h_scratch_bytes), indexed [row * npad + block] so a warp's lanes touch
// consecutive entries.
#include <cuda_runtime.h>
#include <cuda_fp16.h>

#include <climits>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bptc_math.cuh"
#include "bc_check.cuh"

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
#ifndef BCN_BC6H_PREP_MINB
#define BCN_BC6H_PREP_MINB 4
#endif
#ifndef BCN_BC6H_SEARCH_MINB
#define BCN_BC6H_SEARCH_MINB 6  // 80 registers: 0.242 ms at 1024x1024, 96 (5) 0.246, 64 (8) 0.246
#endif
#ifndef BCN_BC6H_REFINE_MINB
#define BCN_BC6H_REFINE_MINB 4
#endif
#ifndef BCN_BC6H_ENC1_MINB
#define BCN_BC6H_ENC1_MINB 4
#endif

constexpr int NW = 4;     // warps per CTA

struct Job {  // per-block quantisation state of one encode
    int mode;
    int epb;
    int qb[6];  // qbounds[0..3) and qbounds[4..7)
};

// A job in 16 bytes: mode | epb << 8, then the six bounds as 16-bit pairs
// (a bound is at most 2^16 - 1).
BCN_DEV uint4 pack_job(const Job& j) {
    return make_uint4((uint32_t)j.mode | ((uint32_t)j.epb << 8), (uint32_t)j.qb[0] | ((uint32_t)j.qb[1] << 16),
                      (uint32_t)j.qb[2] | ((uint32_t)j.qb[3] << 16), (uint32_t)j.qb[4] | ((uint32_t)j.qb[5] << 16));
}
BCN_DEV Job unpack_job(uint4 v) {
    Job j;
    j.mode = (int)(v.x & 0xFFu);
    j.epb = (int)(v.x >> 8);
    j.qb[0] = (int)(v.y & 0xFFFFu);
    j.qb[1] = (int)(v.y >> 16);
    j.qb[2] = (int)(v.z & 0xFFFFu);
    j.qb[3] = (int)(v.z >> 16);
    j.qb[4] = (int)(v.w & 0xFFFFu);
    j.qb[5] = (int)(v.w >> 16);
    return j;
}

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
// ep0: the partition's unquantised endpoints (block_segment of both
// subsets), as the search computed and kept them.
BCN_DEV float eval_2p(const Blk& blk, int part_id, const float ep0[16], int epb, const int qb[6], int qep[24],
                      uint32_t& q0, uint32_t& q1) {
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) {
        ep[i] = i < 16 ? ep0[i] : 0.0f;
        qep[i] = 0;
    }
    uint32_t pattern = kPartitionMap[part_id];
    quant_dequant<2>(qep, ep, epb, qb);
    return block_quant<3, 3, 2>(blk, ep, pattern, q0, q1);
}

// The refinement of a two-region encode's winner (bc6h.rs:355-387): the
// best endpoints (qep[0..16), channel 3 unused) and indices.
BCN_DEV float refine_2p(const Blk& blk, int part_id, const float ep0[16], const Job& st, float best_err,
                        uint32_t iters, int best_qep[16], uint32_t& bq0, uint32_t& bq1) {
    int qe[24];
    eval_2p(blk, part_id, ep0, st.epb, st.qb, qe, bq0, bq1);
#pragma unroll
    for (int i = 0; i < 16; i++) best_qep[i] = qe[i];
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
    return best_err;
}

// bc6h_code_2p (bc6h.rs:241-266).
BCN_DEV uint4 code_2p(int qep[24], uint32_t q0, uint32_t q1, int part_id, int mode) {
    uint32_t flips = apply_swap_mode01237(qep, q0, q1, 1, part_id);
    uint32_t packed[4];
    bc6h_pack(packed, qep, mode);
    BitWriter bw;
    bw.clear();
    bw.put(5, packed[0]);
    bw.put(30, packed[1]);
    bw.put(30, packed[2]);
    bw.put(12, packed[3]);
    bw.put(5, (uint32_t)part_id);
    code_qblock(bw, q0, q1, 3, flips);
    adjust_skip_mode01237(bw.d, 1, part_id);
    return make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
}

// bc6h_enc_1p (bc6h.rs:390-412): the endpoints (qep[0..8)) and indices.
BCN_DEV float encode_1p(const Blk& blk, const Job& st, uint32_t iters, int out_qep[8], uint32_t& q0, uint32_t& q1) {
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
    block_segment<3, false>(blk, 0xFFFFu, ep);
    int qep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) qep[i] = 0;
    quant_dequant<1>(qep, ep, st.epb, st.qb);
    float err = block_quant<3, 4, 1>(blk, ep, 0, q0, q1);
    for (uint32_t it = 0; it < iters; it++) {
        opt_endpoints<3, 4>(ep, blk, q0, q1, 0xFFFFu);
        quant_dequant<1>(qep, ep, st.epb, st.qb);
        err = block_quant<3, 4, 1>(blk, ep, 0, q0, q1);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) out_qep[i] = qep[i];
    return err;
}

// bc6h_code_1p (bc6h.rs:268-286).
BCN_DEV uint4 code_1p(int qep[24], uint32_t q0, uint32_t q1, int mode) {
    apply_swap_mode456(qep, 4, q0, q1, 4);
    uint32_t packed[4];
    bc6h_pack(packed, qep, mode);
    BitWriter bw;
    bw.clear();
    bw.put(5, packed[0]);
    bw.put(30, packed[1]);
    bw.put(30, packed[2]);
    code_qblock(bw, q0, q1, 4, 0);
    return make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
}

// Encode list of a settings value: kind (2 = two-region, 1 = one-region) per
// encode, in the reference's order (the two-region encodes come first).
// Uniform over the launch.
struct Plan {
    int n;
    int n2;  // number of two-region encodes
    int k;   // partitions tried per two-region encode
};

static __host__ __device__ Plan make_plan(const BC6HSettingsDev& s) {
    Plan p;
    if (s.slow_mode != 0) {
        p.n2 = 6;
        p.n = 10;
    } else {
        p.n2 = s.fast_skip_threshold > 0 ? (s.fast_mode == 0 ? 2 : 1) : 0;
        p.n = p.n2 + 1;
    }
    p.k = (int)s.fast_skip_threshold;
    if (p.k == 0) {  // no partition is tried: the 2-region encodes do nothing (bc6h.rs:327-329)
        p.n2 = 0;
        p.n = s.slow_mode != 0 ? 4 : 1;
    }
    return p;
}

// Arguments shared by every kernel of one encode.
struct Work {
    const uint8_t* src;
    size_t stride;
    int source_format;
    bool aligned;  // 16-byte loads of RGBA16F rows
    uint32_t bw, nblocks, npad;
    uint8_t* dst;
    uint4* jobs;               // [j * npad + block]
    uint8_t* lists;            // [c * npad + block]: top-k partitions, ascending bound
    unsigned long long* keys;  // [j * npad + block], 2-region encodes: (error bits << 32) | candidate
    float* slot_err;           // [j * npad + block]
    uint4* slot_pay;           // [(j * 3 + r) * npad + block]: the encode's result, coded by select only if it wins
    float4* seg;               // [(c * 4 + q) * npad + block]: list entry c's unquantised endpoints (16 floats)
    BC6HSettingsDev S;
};

// Row `row` of a scratch array with `rows` rows, at block gi: whether the
// guarded index is inside the array (always true outside check builds).
BCN_DEV bool scratch_ok(const Work& w, int row, int rows, uint32_t gi) {
    return BCN_GUARD(row, rows, CHECK_BC6H_SCRATCH) && BCN_GUARD(gi, w.npad, CHECK_BC6H_SCRATCH);
}

// An encode's result in three 16-byte rows: the 16 endpoint values as 16-bit
// pairs (BC6H endpoints are below 2^16), then the indices and the partition.
BCN_DEV void store_pay(const Work& w, int j, uint32_t gi, const int qep[16], uint32_t q0, uint32_t q1, int part) {
    uint32_t v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = (uint32_t)qep[2 * i] | ((uint32_t)qep[2 * i + 1] << 16);
    w.slot_pay[((size_t)j * 3 + 0) * w.npad + gi] = make_uint4(v[0], v[1], v[2], v[3]);
    w.slot_pay[((size_t)j * 3 + 1) * w.npad + gi] = make_uint4(v[4], v[5], v[6], v[7]);
    w.slot_pay[((size_t)j * 3 + 2) * w.npad + gi] = make_uint4(q0, q1, (uint32_t)part, 0u);
}
BCN_DEV void load_pay(const Work& w, int j, uint32_t gi, int qep[24], uint32_t& q0, uint32_t& q1, int& part) {
    const uint4 a = w.slot_pay[((size_t)j * 3 + 0) * w.npad + gi], b = w.slot_pay[((size_t)j * 3 + 1) * w.npad + gi],
                c = w.slot_pay[((size_t)j * 3 + 2) * w.npad + gi];
    const uint32_t v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int i = 0; i < 8; i++) {
        qep[2 * i] = (int)(v[i] & 0xFFFFu);
        qep[2 * i + 1] = (int)(v[i] >> 16);
    }
#pragma unroll
    for (int i = 16; i < 24; i++) qep[i] = 0;
    q0 = c.x;
    q1 = c.y;
    part = (int)c.z;
}

// Stages the 32 blocks of `tile` as planar f32 (the f16 bit pattern of
// every channel value, scaled by 64/31 as bc6h_setup does, bc6h.rs:801-804)
// with threads tid = 0..nt-1 of the caller; px rows are c * 16 + k.
BCN_DEV void stage_tile(float (*px)[NB], const Work& w, uint32_t tile, int tid, int nt) {
    for (int t = tid; t < NB * 4; t += nt) {
        const int b = t & 31, y = t >> 5;
        const uint32_t gi = tile * NB + b;
        float v[12];
#pragma unroll
        for (int i = 0; i < 12; i++) v[i] = 0.0f;
        if (gi < w.nblocks && BCN_GUARD(gi / w.bw * 4 + y, (w.nblocks + w.bw - 1) / w.bw * 4, CHECK_BC6H_STAGE)) {
            const uint32_t by = gi / w.bw, bx = gi - by * w.bw;
            const uint8_t* row = w.src + (size_t)(by * 4 + y) * w.stride;
            if (w.source_format == BC6H_SRC_RGBA16F) {
                if (w.aligned) {  // the row's 4 pixels: 32 bytes
                    const uint4* r = reinterpret_cast<const uint4*>(row + (size_t)bx * 32);
                    const uint4 a = __ldg(r), c = __ldg(r + 1);
                    const uint32_t wd[8] = {a.x, a.y, a.z, a.w, c.x, c.y, c.z, c.w};
#pragma unroll
                    for (int x = 0; x < 4; x++) {
                        v[x * 3 + 0] = (float)(wd[2 * x] & 0xFFFFu);
                        v[x * 3 + 1] = (float)(wd[2 * x] >> 16);
                        v[x * 3 + 2] = (float)(wd[2 * x + 1] & 0xFFFFu);
                    }
                } else {
                    const uint16_t* r16 = reinterpret_cast<const uint16_t*>(row) + (size_t)bx * 16;
#pragma unroll
                    for (int x = 0; x < 4; x++)
#pragma unroll
                        for (int c = 0; c < 3; c++) v[x * 3 + c] = (float)r16[x * 4 + c];
                }
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
            for (int c = 0; c < 3; c++) px[c * 16 + y * 4 + x][b] = div_const<31>(v[x * 3 + c]) * 64.0f;
    }
}

// bc6h_setup (bc6h.rs:793-819) and the state of every encode of the block
// (compress_bc6h_core's bc6h_test_mode sequence, bc6h.rs:821-860), written
// to the job rows.
BCN_DEV void setup_jobs(const Blk& blk, const Work& w, uint32_t gi) {
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
    int n = 0;
    const int njobs = make_plan(w.S).n;
    auto keep = [&](const Job& j) {
        if (scratch_ok(w, n, njobs, gi)) w.jobs[(size_t)n * w.npad + gi] = pack_job(j);
        n++;
    };
    Job st;
    st.mode = 0;
    st.epb = 0;
    for (int i = 0; i < 6; i++) st.qb[i] = 0;
    const BC6HSettingsDev& S = w.S;
    if (S.slow_mode != 0) {
        // modes 0, 1, 2, 5, 6, 9 (two regions), 10..13 (one region); margin 0 always passes
        const uint64_t modes = 0xDCBA965210ull;
        for (int i = 0; i < 10; i++) {
            test_mode(su, (int)((modes >> (4 * i)) & 15), 0.0f, st);
            if (S.fast_skip_threshold > 0 || i >= 6) keep(st);
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

// K1: setup + encode states (warp 0), the 32 PCA split bounds of the
// two-region partitions (bc6h.rs:288-302) over all warps, and the ascending
// top-k list (partial_sort_list, common.rs:126-140; keys are unique) by the
// last warp. Also clears the search's argmin keys.
__global__ void __launch_bounds__(NW * 32, BCN_BC6H_PREP_MINB) bc6h_prep_kernel(Work w) {
    __shared__ float px[48][NB];
    __shared__ int keys[32][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile(px, w, tile, threadIdx.x, NW * 32);
    __syncthreads();
    const Blk blk{&px[0][lane]};
    if (warp == 0) {
        setup_jobs(blk, w, gi);
        for (int j = 0; j < P.n2; j++)
            if (scratch_ok(w, j, P.n2, gi)) w.keys[(size_t)j * w.npad + gi] = ~0ull;
    }
    if (P.n2 == 0) return;
    float full[15];
    stats_masked<3>(blk, 0xFFFFu, full);
    for (int part = warp; part < 32; part += NW) {
        float b12 = pca_bound_split<3>(blk, subset_mask_from_map(kPartitionMap[part], 0), full);
        keys[part][lane] = part + (int)b12 * 64;
    }
    __syncthreads();
    if (warp == NW - 1) {
        for (int k = 0; k < P.k; k++) {
            int best = INT_MAX, bi = 0;
            for (int q = 0; q < 32; q++) {
                int v = keys[q][lane];
                if (v < best) {
                    best = v;
                    bi = q;
                }
            }
            if (scratch_ok(w, k, P.k, gi)) w.lists[(size_t)k * w.npad + gi] = (uint8_t)bi;
            keys[bi][lane] = INT_MAX;
        }
    }
}

// K2: list entry c = `blockIdx.y * NW + warp` for the 32 blocks of the tile,
// for every two-region encode j (bc6h_enc_2p_part_fast, bc6h.rs:304-324).
// Entry c is the same partition for every j (one list per block), and its
// unquantised endpoints (block_segment of both subsets) depend only on the
// pixels, so they are computed once and each encode quantises its own copy
// with its endpoint precision and bounds. A candidate counts only with an
// error below +inf (the reference's running best starts there,
// bc6h.rs:337); errors are non-negative, so the argmin key's high word
// orders like the error and the low word keeps the earliest candidate among
// equal errors, the reference's strict "<" scan.
__global__ void __launch_bounds__(NW * 32, BCN_BC6H_SEARCH_MINB) bc6h_search_kernel(Work w) {
    __shared__ float px[48][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x, gi = tile * NB + lane;
    const Plan P = make_plan(w.S);
    stage_tile(px, w, tile, threadIdx.x, NW * 32);
    __syncthreads();
    const int c = blockIdx.y * NW + warp;
    if (c >= P.k || gi >= w.nblocks || !scratch_ok(w, c, P.k, gi)) return;
    const Blk blk{&px[0][lane]};
    const uint32_t pattern = kPartitionMap[w.lists[(size_t)c * w.npad + gi] & 31];
    float ep0[16];
#pragma unroll
    for (int i = 0; i < 16; i++) ep0[i] = 0.0f;
#pragma unroll
    for (int h = 0; h < 2; h++) block_segment<3, false>(blk, subset_mask_from_map(pattern, h), ep0 + 8 * h);
    // kept for the refinement of whichever encode picks this entry
#pragma unroll
    for (int q = 0; q < 4; q++)
        w.seg[((size_t)c * 4 + q) * w.npad + gi] = make_float4(ep0[4 * q], ep0[4 * q + 1], ep0[4 * q + 2], ep0[4 * q + 3]);
#pragma unroll 1
    for (int j = 0; j < P.n2; j++) {
        if (!scratch_ok(w, j, P.n2, gi)) continue;
        const Job st = unpack_job(w.jobs[(size_t)j * w.npad + gi]);
        float ep[24];
        int qep[24];
#pragma unroll
        for (int i = 0; i < 24; i++) {
            ep[i] = i < 16 ? ep0[i] : 0.0f;
            qep[i] = 0;
        }
        uint32_t q0, q1;
        quant_dequant<2>(qep, ep, st.epb, st.qb);
        const float err = block_quant<3, 3, 2>(blk, ep, pattern, q0, q1);
        if (err < __int_as_float(0x7f800000))
            atomicMin(&w.keys[(size_t)j * w.npad + gi], ((unsigned long long)__float_as_uint(err) << 32) | (uint32_t)c);
    }
}

// K3: the winner of two-region encode blockIdx.y, refined (bc6h.rs:355-387);
// one warp per tile, a private staged tile per warp. The winner's
// unquantised endpoints come from the search's scratch (`seg`) instead of a
// second endpoint fit of the same pixels.
__global__ void __launch_bounds__(NW * 32, BCN_BC6H_REFINE_MINB) bc6h_refine2_kernel(Work w, uint32_t ntiles) {
    __shared__ float px[NW][48][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x * NW + warp, gi = tile * NB + lane;
    if (tile >= ntiles) return;
    stage_tile(px[warp], w, tile, lane, 32);
    __syncwarp();
    const int j = blockIdx.y;
    const Plan P = make_plan(w.S);
    if (!scratch_ok(w, j, P.n2, gi)) return;
    float err = __int_as_float(0x7f800000);
    const unsigned long long key = w.keys[(size_t)j * w.npad + gi];
    if (gi < w.nblocks && key != ~0ull && scratch_ok(w, (int)(key & 0xFFFFFFFFull), P.k, gi)) {
        const Job st = unpack_job(w.jobs[(size_t)j * w.npad + gi]);
        const int c = (int)(key & 0xFFFFFFFFull);
        const int part = w.lists[(size_t)c * w.npad + gi] & 31;
        float ep0[16];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float4 v = w.seg[((size_t)c * 4 + q) * w.npad + gi];
            ep0[4 * q] = v.x;
            ep0[4 * q + 1] = v.y;
            ep0[4 * q + 2] = v.z;
            ep0[4 * q + 3] = v.w;
        }
        int qep[16];
        uint32_t q0, q1;
        err = refine_2p(Blk{&px[warp][0][lane]}, part, ep0, st, __uint_as_float((uint32_t)(key >> 32)),
                        w.S.refine_iterations_2p, qep, q0, q1);
        store_pay(w, j, gi, qep, q0, q1, part);
    }
    w.slot_err[(size_t)j * w.npad + gi] = err;
}

// K4: one-region encode n2 + blockIdx.y (bc6h_enc_1p, bc6h.rs:390-412).
__global__ void __launch_bounds__(NW * 32, BCN_BC6H_ENC1_MINB) bc6h_enc1_kernel(Work w, uint32_t ntiles, int n2) {
    __shared__ float px[NW][48][NB];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile = blockIdx.x * NW + warp, gi = tile * NB + lane;
    if (tile >= ntiles) return;
    stage_tile(px[warp], w, tile, lane, 32);
    __syncwarp();
    const int j = n2 + blockIdx.y;
    if (!scratch_ok(w, j, make_plan(w.S).n, gi)) return;
    float err = __int_as_float(0x7f800000);
    if (gi < w.nblocks) {
        const Job st = unpack_job(w.jobs[(size_t)j * w.npad + gi]);
        int qep[16];
        uint32_t q0, q1;
        err = encode_1p(Blk{&px[warp][0][lane]}, st, w.S.refine_iterations_1p, qep, q0, q1);
#pragma unroll
        for (int i = 8; i < 16; i++) qep[i] = 0;
        store_pay(w, j, gi, qep, q0, q1, 0);
    }
    w.slot_err[(size_t)j * w.npad + gi] = err;
}

// K5: the reference's sequential strict comparisons over the encodes, in
// order (self.best_err starts at +inf), then the coding of the winner alone
// (coding depends only on the winner's endpoints, indices, partition and
// mode; the reference codes on every improvement, bc6h.rs:383-386, 407-411,
// and keeps the last) and the block's 128-bit store. A block no encode
// improved stays all zero, as the reference's data array.
__global__ void __launch_bounds__(128) bc6h_select_kernel(Work w, int n, int n2) {
    const uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= w.nblocks) return;
    float best = __int_as_float(0x7f800000);
    int win = -1;
    for (int j = 0; j < n; j++) {
        const float e = scratch_ok(w, j, n, gi) ? w.slot_err[(size_t)j * w.npad + gi] : __int_as_float(0x7f800000);
        if (e < best) {
            best = e;
            win = j;
        }
    }
    uint4 data = make_uint4(0, 0, 0, 0);
    if (win >= 0) {
        int qep[24];
        uint32_t q0, q1;
        int part;
        load_pay(w, win, gi, qep, q0, q1, part);
        const int mode = (int)(w.jobs[(size_t)win * w.npad + gi].x & 0xFFu);
        data = win < n2 ? code_2p(qep, q0, q1, part, mode) : code_1p(qep, q0, q1, mode);
    }
    if (!BCN_GUARD(gi, w.nblocks, CHECK_BC6H_STORE)) return;
    uint8_t* o = w.dst + (size_t)gi * 16;
    if (((uintptr_t)w.dst & 15) == 0) {
        *reinterpret_cast<uint4*>(o) = data;
    } else {
        uint32_t* o32 = reinterpret_cast<uint32_t*>(o);
        o32[0] = data.x;
        o32[1] = data.y;
        o32[2] = data.z;
        o32[3] = data.w;
    }
}

// Scratch layout, each array 256-byte aligned.
struct Layout {
    size_t jobs, lists, keys, slot_err, slot_pay, seg, total;
};
static Layout layout(uint32_t npad, const Plan& P) {
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    Layout L;
    L.jobs = 0;
    L.lists = up(L.jobs + (size_t)P.n * npad * sizeof(uint4));
    L.keys = up(L.lists + (size_t)(P.k > 0 ? P.k : 1) * npad);
    L.slot_err = up(L.keys + (size_t)(P.n2 > 0 ? P.n2 : 1) * npad * sizeof(unsigned long long));
    L.slot_pay = up(L.slot_err + (size_t)P.n * npad * sizeof(float));
    L.seg = up(L.slot_pay + (size_t)P.n * 3 * npad * sizeof(uint4));
    L.total = up(L.seg + (size_t)(P.k > 0 ? P.k : 1) * 4 * npad * sizeof(float4));
    return L;
}

}  // namespace bc6h

cudaError_t check_take_bc6h(unsigned long long out[3]) { return check_record_take(out); }

size_t bc6h_scratch_bytes(uint32_t nblocks, const BC6HSettingsDev& settings) {
    const uint32_t npad = (nblocks + bptc::NB - 1) / bptc::NB * bptc::NB;
    return bc6h::layout(npad, bc6h::make_plan(settings)).total;
}

namespace bc6h {
// The side stream of launch_bc6h_encode with its fork and join events, per
// host thread, created on first use for the current device.
struct SideStream {
    cudaStream_t st = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    int device = -1;
    void release() {
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (st) cudaStreamDestroy(st);
        fork = join = nullptr;
        st = nullptr;
        device = -1;
    }
    ~SideStream() { release(); }
    cudaError_t get() {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess || dev == device) return e;
        release();
        if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming)) != cudaSuccess) return e;
        device = dev;
        return cudaSuccess;
    }
};
static thread_local SideStream t_side;
}  // namespace bc6h

// prep on `s`; then the one-region encodes (they need only the encode
// states) on a side stream forked from `s`, while `s` runs the two-region
// search and refinement; joined before the selection. While `s` captures a
// graph, the side stream is used only if this thread made it earlier for
// the device (a stream is not created during a capture); otherwise every
// launch stays on `s`.
cudaError_t launch_bc6h_encode(const void* src, size_t stride_bytes, int source_format, uint32_t bw, uint32_t bh,
                               uint8_t* dst, const BC6HSettingsDev& settings, void* scratch, cudaStream_t s) {
    using namespace bc6h;
    const uint32_t n = bw * bh;
    if (n == 0) return cudaSuccess;
    const uint32_t ntiles = (n + NB - 1) / NB, npad = ntiles * NB;
    const Plan P = make_plan(settings);
    const Layout L = layout(npad, P);
    uint8_t* base = (uint8_t*)scratch;
    Work w;
    w.src = (const uint8_t*)src;
    w.stride = stride_bytes;
    w.source_format = source_format;
    w.aligned = ((uintptr_t)src % 16 == 0) && (stride_bytes % 16 == 0);
    w.bw = bw;
    w.nblocks = n;
    w.npad = npad;
    w.dst = dst;
    w.jobs = (uint4*)(base + L.jobs);
    w.lists = base + L.lists;
    w.keys = (unsigned long long*)(base + L.keys);
    w.slot_err = (float*)(base + L.slot_err);
    w.slot_pay = (uint4*)(base + L.slot_pay);
    w.seg = (float4*)(base + L.seg);
    w.S = settings;
    cudaError_t e;
    bc6h_prep_kernel<<<ntiles, NW * 32, 0, s>>>(w);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaStream_t s1 = s;
    if (P.n2 > 0 && P.n > P.n2) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if ((e = cudaStreamIsCapturing(s, &cs)) != cudaSuccess) return e;
        int dev = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if (cs == cudaStreamCaptureStatusNone || t_side.device == dev) {
            if ((e = t_side.get()) != cudaSuccess) return e;
            if ((e = cudaEventRecord(t_side.fork, s)) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(t_side.st, t_side.fork, 0)) != cudaSuccess) return e;
            s1 = t_side.st;
        }
    }
    if (P.n > P.n2)
        bc6h_enc1_kernel<<<dim3((ntiles + NW - 1) / NW, (uint32_t)(P.n - P.n2)), NW * 32, 0, s1>>>(w, ntiles, P.n2);
    if (P.n2 > 0) {
        const uint32_t groups = (uint32_t)(P.k + NW - 1) / NW;
        bc6h_search_kernel<<<dim3(ntiles, groups), NW * 32, 0, s>>>(w);
        bc6h_refine2_kernel<<<dim3((ntiles + NW - 1) / NW, (uint32_t)P.n2), NW * 32, 0, s>>>(w, ntiles);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (s1 != s) {
        if ((e = cudaEventRecord(t_side.join, s1)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, t_side.join, 0)) != cudaSuccess) return e;
    }
    bc6h_select_kernel<<<(n + 127) / 128, 128, 0, s>>>(w, P.n, P.n2);
    return cudaGetLastError();
}

}  // namespace bcn
