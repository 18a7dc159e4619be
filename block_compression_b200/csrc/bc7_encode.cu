// BC7 encoder for sm_100a.
//
// Work decomposition. A CTA owns a tile of 32 consecutive 4x4 blocks; lane l
// of every warp works on block l of the tile, so all 32 lanes of a warp always
// run the same mode and candidate (no intra-warp divergence apart from the
// per-block partition lists). The candidate space of the reference search
// (src/encode/bc7.rs:540-879) is swept by the CTA's warps in phases:
//
//   1. load     32 blocks -> shared memory, planar f32 (128-bit coalesced loads)
//   2. bounds   64 (or 128) PCA split bounds per block, spread over warps
//   3. top-k    per-block ascending selection of the best partitions (modes 1/3/7)
//   4. search   every partition candidate of modes 0/2/1/3/7, spread over
//               warps; each warp keeps a first-minimum per mode, merged in
//               shared memory (smallest error, then earliest candidate)
//   5. chains   refinement of each mode's winner, every mode-4/5
//               rotation/index-swap candidate, and mode 6 -- one chain per warp
//               item; each chain leaves (error, coded 128-bit block) in a slot
//   6. select   per block, the reference's sequential "strictly better"
//               comparisons over the slots in the reference mode order
//   7. store    one 128-bit store per block
//
// Every per-candidate computation keeps the reference's operation order, so
// the chosen mode, endpoints and indices are bit-identical to the reference
// CPU encoder (see bc_common.cuh for the float rules).
#include <cuda_runtime.h>

#include <climits>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bptc_math.cuh"
namespace bcn {
namespace bc7 {

using namespace bptc;
constexpr int NSLOT = 18;   // 5 mode-0/2/1/3/7 results + 12 mode-4/5 candidates + mode 6

// Mode 4/5 candidate block (bc7.rs:680-696): channel `rot` replaced by alpha
// (4-channel settings) or by 255 (3-channel settings).
struct BlkRot {
    const float* p;
    int rot;
    int channels;
    BCN_DEV float operator()(int c, int k) const {
        if (c == rot) return channels == 4 ? p[(48 + k) * NB] : 255.0f;
        return p[(c * 16 + k) * NB];
    }
};

struct Smem {
    float px[64][NB];
    uint32_t map[128];
    uint8_t anchors[128];
    float opaque_err[NB];
    union {
        int keys[2][64][NB];                // phase 2-3
        struct {
            float err[5][8][NB];            // phase 4 per-warp first minima
            int cand[5][8][NB];
        } c;
    } u;
    uint8_t list[2][64][NB];                // sorted partitions: [0] modes 1/3, [1] mode 7
    int winner[5][NB];
    float slot_err[NSLOT][NB];
    uint4 slot_data[NSLOT][NB];
};

// ---- endpoint quantisation (bc7.rs:97-237) ----------------------------------

// ep_quant0367 for one endpoint pair (8 values). QCH = channels quantised
// (the error uses the first CH); EPB_MODE0 unpacks the trial values to bytes
// as the reference does for mode 0 only.
template <int BITS, int CH, int QCH, bool MODE0>
BCN_DEV void quant0367_pair(int* qep, const float* ep) {
    constexpr int levels2 = (1 << BITS) * 2 - 1;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        int qb[2][4];
        float eb[2][4];
#pragma unroll
        for (int b = 0; b < 2; b++) {
#pragma unroll
            for (int p = 0; p < QCH; p++) {
                int v = (int)((ep[i * 4 + p] / 255.0f * (float)levels2 - (float)b) / 2.0f + 0.5f) * 2 + b;
                qb[b][p] = clampi(v, b, levels2 - 1 + b);
                eb[b][p] = MODE0 ? (float)unpack_to_byte(qb[b][p], 5) : (float)qb[b][p];
            }
        }
        float err0 = 0.0f, err1 = 0.0f;
#pragma unroll
        for (int p = 0; p < CH; p++) {
            err0 += sqf(ep[i * 4 + p] - eb[0][p]);
            err1 += sqf(ep[i * 4 + p] - eb[1][p]);
        }
#pragma unroll
        for (int p = 0; p < QCH; p++) qep[i * 4 + p] = err0 < err1 ? qb[0][p] : qb[1][p];
    }
}

// ep_quant1 for one pair (shared p-bit)
BCN_DEV void quant1_pair(int* qep, const float* ep) {
    int qb[2][8];
    float eb[2][8];
#pragma unroll
    for (int b = 0; b < 2; b++) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if ((i & 3) == 3) continue;  // channel 3 is neither coded nor in the error
            int v = (int)((ep[i] / 255.0f * 127.0f - (float)b) / 2.0f + 0.5f) * 2 + b;
            qb[b][i] = clampi(v, b, 126 + b);
            eb[b][i] = (float)unpack_to_byte(qb[b][i], 7);
        }
    }
    float err0 = 0.0f, err1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
        for (int p = 0; p < 3; p++) {
            err0 += sqf(ep[j * 4 + p] - eb[0][j * 4 + p]);
            err1 += sqf(ep[j * 4 + p] - eb[1][j * 4 + p]);
        }
#pragma unroll
    for (int i = 0; i < 8; i++)
        if ((i & 3) != 3) qep[i] = err0 < err1 ? qb[0][i] : qb[1][i];
}

template <int BITS, int N>
BCN_DEV void quant245(int* qep, const float* ep) {
    constexpr int levels = 1 << BITS;
#pragma unroll
    for (int i = 0; i < N; i++) qep[i] = clampi((int)(ep[i] / 255.0f * (float)(levels - 1) + 0.5f), 0, levels - 1);
}

// ep_quant_dequant for the partitioned modes over PAIRS pairs; channel 3 is
// handled only for mode 7 (4 channels).
template <int MODE>
BCN_DEV void quant_dequant_part(int qep[24], float ep[24]) {
    constexpr int pairs = (MODE == 0 || MODE == 2) ? 3 : 2;
#pragma unroll
    for (int j = 0; j < pairs; j++) {
        int* q = qep + 8 * j;
        float* e = ep + 8 * j;
        if (MODE == 0) quant0367_pair<4, 3, 3, true>(q, e);
        else if (MODE == 3) quant0367_pair<7, 3, 3, false>(q, e);
        else if (MODE == 7) quant0367_pair<5, 4, 4, false>(q, e);
        else if (MODE == 1) quant1_pair(q, e);
        else {
#pragma unroll
            for (int i = 0; i < 8; i++)
                if ((i & 3) != 3) q[i] = clampi((int)(e[i] / 255.0f * 31.0f + 0.5f), 0, 31);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (MODE != 7 && (i & 3) == 3) continue;
            if (MODE == 3) e[i] = (float)q[i];
            else if (MODE == 1) e[i] = (float)unpack_to_byte(q[i], 7);
            else if (MODE == 7) e[i] = (float)unpack_to_byte(q[i], 6);
            else e[i] = (float)unpack_to_byte(q[i], 5);
        }
    }
}

// ---- candidate evaluation of modes 0/1/2/3/7 (bc7.rs:517-538) -----------------

template <int MODE>
struct ModeTraits {
    static constexpr int bits = (MODE == 0 || MODE == 1) ? 3 : 2;
    static constexpr int pairs = (MODE == 0 || MODE == 2) ? 3 : 2;
    static constexpr int ch = MODE == 7 ? 4 : 3;
};

template <int MODE>
BCN_DEV float eval_part(const Blk& blk, const uint32_t* map, int part_id, int qep[24], uint32_t& q0, uint32_t& q1) {
    using T = ModeTraits<MODE>;
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
    uint32_t pattern = map[part_id];
#pragma unroll
    for (int j = 0; j < T::pairs; j++)
        block_segment<T::ch, true>(blk, subset_mask_from_map(pattern, j), ep + 8 * j);
    quant_dequant_part<MODE>(qep, ep);
    return block_quant<T::ch, T::bits, T::pairs>(blk, ep, pattern, q0, q1);
}

// bc7.rs:381-440
template <int MODE>
BCN_DEV uint4 code_mode01237(int qep[24], uint32_t q0, uint32_t q1, int part_id) {
    using T = ModeTraits<MODE>;
    uint32_t flips = apply_swap_mode01237(qep, q0, q1, MODE, part_id);
    BitWriter bw;
    bw.clear();
    bw.put(MODE + 1, 1u << MODE);
    if (MODE == 0) bw.put(4, (uint32_t)(part_id & 15));
    else bw.put(6, (uint32_t)(part_id & 63));
#pragma unroll
    for (int p = 0; p < T::ch; p++)
#pragma unroll
        for (int j = 0; j < T::pairs * 2; j++) {
            uint32_t v = (uint32_t)qep[j * 4 + p];
            if (MODE == 0) bw.put(4, v >> 1);
            else if (MODE == 1) bw.put(6, v >> 1);
            else if (MODE == 2) bw.put(5, v);
            else if (MODE == 3) bw.put(7, v >> 1);
            else bw.put(5, v >> 1);
        }
    if (MODE == 1)
        for (int j = 0; j < 2; j++) bw.put(1, (uint32_t)qep[j * 8] & 1);
    if (MODE == 0 || MODE == 3 || MODE == 7)
#pragma unroll
        for (int j = 0; j < T::pairs * 2; j++) bw.put(1, (uint32_t)qep[j * 4] & 1);
    code_qblock(bw, q0, q1, T::bits, flips);
    adjust_skip_mode01237(bw.d, MODE, part_id);
    return make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
}

// Refinement of a mode's winning partition (bc7.rs:571-609), then coding.
template <int MODE>
BCN_DEV float refine_and_code(const Blk& blk, const uint32_t* map, int part_id, float best_err, uint32_t iters,
                              float opaque_err, uint4& out) {
    using T = ModeTraits<MODE>;
    int best_qep[24];
    uint32_t bq0, bq1;
    eval_part<MODE>(blk, map, part_id, best_qep, bq0, bq1);  // re-creates the winner's state
    uint32_t pattern = map[part_id];
    for (uint32_t it = 0; it < iters; it++) {
        float ep[24];
#pragma unroll
        for (int i = 0; i < 24; i++) ep[i] = 0.0f;
#pragma unroll
        for (int j = 0; j < T::pairs; j++)
            opt_endpoints<T::ch, T::bits>(ep + 8 * j, blk, bq0, bq1, subset_mask_from_map(pattern, j));
        int qep[24];
        uint32_t q0, q1;
        quant_dequant_part<MODE>(qep, ep);
        float err = block_quant<T::ch, T::bits, T::pairs>(blk, ep, pattern, q0, q1);
        if (err < best_err) {
#pragma unroll
            for (int i = 0; i < 24; i++) best_qep[i] = qep[i];
            bq0 = q0;
            bq1 = q1;
            best_err = err;
        }
    }
    if (MODE != 7) best_err += opaque_err;
    out = code_mode01237<MODE>(best_qep, bq0, bq1, part_id);
    return best_err;
}

// ---- mode 4/5 (bc7.rs:239-369, 442-492, 657-733) ---------------------------------

BCN_DEV void channel_quant_dequant(int qep[2], float ep[2], int epbits) {
    int elevels = 1 << epbits;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        qep[i] = clampi((int)(ep[i] / 255.0f * (float)(elevels - 1) + 0.5f), 0, elevels - 1);
        ep[i] = (float)unpack_to_byte(qep[i], epbits);
    }
}

BCN_DEV float channel_opt_quant(uint32_t& q0, uint32_t& q1, const float cb[16], int bits, const float ep[2]) {
    int levels = 1 << bits;
    q0 = 0;
    q1 = 0;
    float total = 0.0f;
    int ia = (int)ep[0], ib = (int)ep[1];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float proj = (cb[k] - ep[0]) / (ep[1] - ep[0] + 0.001f);
        int q1i = clampi((int)(proj * (float)levels + 0.5f), 1, levels - 1);
        int w0 = unquant_w(bits, q1i - 1), w1 = unquant_w(bits, q1i);
        float d0 = (float)(((64 - w0) * ia + w0 * ib + 32) / 64);
        float d1 = (float)(((64 - w1) * ia + w1 * ib + 32) / 64);
        float err0 = 0.0f, err1 = 0.0f;
        err0 += sqf(d0 - cb[k]);
        err1 += sqf(d1 - cb[k]);
        float be = err0 < err1 ? err0 : err1;
        int bq = err0 < err1 ? q1i - 1 : q1i;
        if (k < 8) q0 |= (uint32_t)bq << (4 * k);
        else q1 |= (uint32_t)bq << (4 * (k - 8));
        total += be;
    }
    return total;
}

BCN_DEV void channel_opt_endpoints(float ep[2], const float cb[16], int bits, uint32_t q0, uint32_t q1) {
    int levels = 1 << bits;
    float lm1 = (float)(levels - 1);
    float atb1 = 0.0f, sum_q = 0.0f, sum_qq = 0.0f, sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float q = (float)(((k < 8 ? q0 : q1) >> (4 * (k & 7))) & 15);
        float x = lm1 - q;
        sum_q += q;
        sum_qq += q * q;
        sum += cb[k];
        atb1 += x * cb[k];
    }
    float atb2 = lm1 * sum - atb1;
    float cxx = 16.0f * sqf(lm1) - 2.0f * lm1 * sum_q + sum_qq;
    float cyy = sum_qq;
    float cxy = lm1 * sum_q - sum_qq;
    float det = cxx * cyy - cxy * cxy;
    float scale = lm1 / det;
    ep[0] = clampf_r((atb1 * cyy - atb2 * cxy) * scale, 0.0f, 255.0f);
    ep[1] = clampf_r((atb2 * cxx - atb1 * cxy) * scale, 0.0f, 255.0f);
    if (fabsf(det) < 0.001f) {
        ep[0] = sum / 16.0f;
        ep[1] = ep[0];
    }
}

// One mode-4/5 candidate: rotation `rot`, index swap `swap`. Returns its
// error and its coded block (bc7_code_mode45 for MODE).
template <int MODE>
BCN_DEV float mode45_candidate(const float* pxlane, int channels, uint32_t refine, uint32_t refine_channel, int rot,
                               int swap, uint4& out) {
    int bits = 2, abits = MODE == 4 ? 3 : 2, aepbits = MODE == 4 ? 6 : 8;
    if (swap == 1) {
        bits = 3;
        abits = 2;
    }
    BlkRot cb{pxlane, rot < 3 ? rot : -1, channels};
    float ep[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    block_segment<3, true>(cb, 0xFFFFu, ep);
    int qep[8];
    constexpr int EPB = MODE == 4 ? 5 : 7;
    quant245<EPB, 8>(qep, ep);
#pragma unroll
    for (int i = 0; i < 8; i++) ep[i] = (float)unpack_to_byte(qep[i], EPB);
    uint32_t q0, q1;
    float err = bits == 2 ? block_quant<3, 2, 1>(cb, ep, 0, q0, q1) : block_quant<3, 3, 1>(cb, ep, 0, q0, q1);
    for (uint32_t it = 0; it < refine; it++) {
        if (bits == 2) opt_endpoints<3, 2>(ep, cb, q0, q1, 0xFFFFu);
        else opt_endpoints<3, 3>(ep, cb, q0, q1, 0xFFFFu);
        quant245<EPB, 8>(qep, ep);
#pragma unroll
        for (int i = 0; i < 8; i++) ep[i] = (float)unpack_to_byte(qep[i], EPB);
        err = bits == 2 ? block_quant<3, 2, 1>(cb, ep, 0, q0, q1) : block_quant<3, 3, 1>(cb, ep, 0, q0, q1);
    }
    // scalar channel (opt_channel, bc7.rs:239-266)
    float chan[16];
#pragma unroll
    for (int k = 0; k < 16; k++) chan[k] = pxlane[(rot * 16 + k) * NB];
    float aep[2] = {255.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 16; k++) {
        aep[0] = fminf(aep[0], chan[k]);
        aep[1] = fmaxf(aep[1], chan[k]);
    }
    int aqep[2];
    uint32_t a0, a1;
    channel_quant_dequant(aqep, aep, aepbits);
    float aerr = channel_opt_quant(a0, a1, chan, abits, aep);
    for (uint32_t it = 0; it < refine_channel; it++) {
        channel_opt_endpoints(aep, chan, abits, a0, a1);
        channel_quant_dequant(aqep, aep, aepbits);
        aerr = channel_opt_quant(a0, a1, chan, abits, aep);
    }
    err += aerr;

    // bc7_code_mode45 (bc7.rs:442-492)
    const int cbits = 2, cabits = MODE == 4 ? 3 : 2, cepbits = MODE == 4 ? 5 : 7, caepbits = MODE == 4 ? 6 : 8;
    uint32_t c0 = q0, c1 = q1, d0 = a0, d1 = a1;
    if (swap == 0) {
        apply_swap_mode456(qep, 4, c0, c1, cbits);
        apply_swap_mode456(aqep, 1, d0, d1, cabits);
    } else {
        uint32_t t0 = c0, t1 = c1;
        c0 = d0;
        c1 = d1;
        d0 = t0;
        d1 = t1;
        apply_swap_mode456(aqep, 1, c0, c1, cbits);
        apply_swap_mode456(qep, 4, d0, d1, cabits);
    }
    BitWriter bw;
    bw.clear();
    bw.put(MODE + 1, 1u << MODE);
    bw.put(2, (uint32_t)(rot + 1) & 3);
    if (MODE == 4) bw.put(1, (uint32_t)swap);
#pragma unroll
    for (int p = 0; p < 3; p++) {
        bw.put(cepbits, (uint32_t)qep[p]);
        bw.put(cepbits, (uint32_t)qep[4 + p]);
    }
    bw.put(caepbits, (uint32_t)aqep[0]);
    bw.put(caepbits, (uint32_t)aqep[1]);
    code_qblock(bw, c0, c1, cbits, 0);
    code_qblock(bw, d0, d1, cabits, 0);
    out = make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
    return err;
}

// ---- mode 6 (bc7.rs:494-515, 762-817) -------------------------------------------

template <int CH>
BCN_DEV float mode6(const Blk& blk, uint32_t refine, uint4& out) {
    float ep[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    block_segment<CH, true>(blk, 0xFFFFu, ep);
    if (CH == 3) {
        ep[3] = 255.0f;
        ep[7] = 255.0f;
    }
    int qep[8];
    quant0367_pair<7, CH, 4, false>(qep, ep);
#pragma unroll
    for (int i = 0; i < 8; i++) ep[i] = (float)qep[i];
    uint32_t q0, q1;
    float err = block_quant<CH, 4, 1>(blk, ep, 0, q0, q1);
    for (uint32_t it = 0; it < refine; it++) {
        opt_endpoints<CH, 4>(ep, blk, q0, q1, 0xFFFFu);
        quant0367_pair<7, CH, 4, false>(qep, ep);
#pragma unroll
        for (int i = 0; i < 8; i++) ep[i] = (float)qep[i];
        err = block_quant<CH, 4, 1>(blk, ep, 0, q0, q1);
    }
    apply_swap_mode456(qep, 4, q0, q1, 4);
    BitWriter bw;
    bw.clear();
    bw.put(7, 64);
#pragma unroll
    for (int p = 0; p < 4; p++) {
        bw.put(7, (uint32_t)qep[p] >> 1);
        bw.put(7, (uint32_t)qep[4 + p] >> 1);
    }
    bw.put(1, (uint32_t)qep[0] & 1);
    bw.put(1, (uint32_t)qep[4] & 1);
    code_qblock(bw, q0, q1, 4, 0);
    out = make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
    return err;
}

// ---- the kernel -----------------------------------------------------------------

// Candidate-mode bookkeeping index: 0 mode0, 1 mode2, 2 mode1, 3 mode3, 4 mode7
// (the reference evaluation order).
struct Plan {
    int count[5];
    int total;
    int k_a, k_b;        // top-k lengths of the bound lists
    bool bounds_a, bounds_b;
    int n45_4, n45_5;    // mode-4 / mode-5 candidate counts
    bool run6;
};

BCN_DEV Plan make_plan(const BC7SettingsDev& s) {
    Plan p;
    bool ms0 = s.mode_selection[0] != 0, ms1 = s.mode_selection[1] != 0;
    bool run13 = ms1 && (s.fast_skip_threshold_mode1 != 0 || s.fast_skip_threshold_mode3 != 0);
    bool run7 = ms1 && s.fast_skip_threshold_mode7 != 0;
    p.count[0] = ms0 ? 16 : 0;
    p.count[1] = (ms0 && s.skip_mode2 == 0) ? 64 : 0;
    p.count[2] = run13 ? (int)s.fast_skip_threshold_mode1 : 0;
    p.count[3] = run13 ? (int)s.fast_skip_threshold_mode3 : 0;
    p.count[4] = run7 ? (int)s.fast_skip_threshold_mode7 : 0;
    p.total = p.count[0] + p.count[1] + p.count[2] + p.count[3] + p.count[4];
    // Mode 7's bounds use the settings' channel count; with 3 channels they
    // equal the mode 1/3 bounds and one sorted list serves both.
    bool sep7 = run7 && s.channels == 4;
    int k13 = run13 ? (int)max(s.fast_skip_threshold_mode1, s.fast_skip_threshold_mode3) : 0;
    p.bounds_a = run13 || (run7 && !sep7);
    p.bounds_b = sep7;
    p.k_a = max(k13, (run7 && !sep7) ? (int)s.fast_skip_threshold_mode7 : 0);
    p.k_b = sep7 ? (int)s.fast_skip_threshold_mode7 : 0;
    int nrot = s.mode_selection[2] != 0 ? (int)s.channels - (int)s.mode45_channel0 : 0;
    if (nrot < 0) nrot = 0;
    p.n45_4 = 2 * nrot;
    p.n45_5 = nrot;
    p.run6 = s.mode_selection[3] != 0;
    return p;
}

template <int NW>
__global__ void __launch_bounds__(NW * 32) bc7_encode_kernel(const uint8_t* __restrict__ src, size_t stride, uint32_t bw,
                                                              uint32_t nblocks, uint8_t* __restrict__ dst,
                                                              BC7SettingsDev S, bool aligned) {
    static_assert(NW <= 8, "per-warp minima are sized for 8 warps");
    __shared__ Smem sm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t tile0 = blockIdx.x * NB;
    const Plan P = make_plan(S);

    // 1. load ---------------------------------------------------------------
    for (int i = threadIdx.x; i < 128; i += blockDim.x) {
        sm.map[i] = kPartitionMap[i];
        sm.anchors[i] = kAnchors[i];
    }
    for (int t = threadIdx.x; t < NB * 4; t += blockDim.x) {
        int b = t & 31, y = t >> 5;
        uint32_t gi = tile0 + b;
        uint32_t w[4] = {0, 0, 0, 0};
        if (gi < nblocks) {
            uint32_t by = gi / bw, bx = gi - by * bw;
            const uint8_t* row = src + (size_t)(by * 4 + y) * stride + (size_t)bx * 16;
            if (aligned) {
                uint4 v = __ldg(reinterpret_cast<const uint4*>(row));
                w[0] = v.x;
                w[1] = v.y;
                w[2] = v.z;
                w[3] = v.w;
            } else {
                for (int j = 0; j < 16; j++) w[j >> 2] |= (uint32_t)row[j] << (8 * (j & 3));
            }
        }
#pragma unroll
        for (int x = 0; x < 4; x++) {
            int k = y * 4 + x;
            sm.px[k][b] = (float)(w[x] & 0xFF);
            sm.px[16 + k][b] = (float)((w[x] >> 8) & 0xFF);
            sm.px[32 + k][b] = (float)((w[x] >> 16) & 0xFF);
            sm.px[48 + k][b] = (float)(w[x] >> 24);
        }
    }
    __syncthreads();
    const float* pxl = &sm.px[0][lane];
    const Blk blk{pxl};
    if (warp == 0) {
        // compute_opaque_err (bc7.rs:869-879)
        float e = 0.0f;
        if (S.channels != 3)
            for (int k = 0; k < 16; k++) e += sqf(blk(3, k) - 255.0f);
        sm.opaque_err[lane] = e;
    }

    // 2. PCA split bounds ----------------------------------------------------
    const int na = P.bounds_a ? 64 : 0, nb = P.bounds_b ? 64 : 0;
    if (na + nb > 0) {
        float full_a[15], full_b[15];
        if (na) stats_masked<3>(blk, 0xFFFFu, full_a);
        if (nb) stats_masked<4>(blk, 0xFFFFu, full_b);
        for (int item = warp; item < na + nb; item += NW) {
            if (item < na) {
                int part = item;
                float b12 = pca_bound_split<3>(blk, subset_mask_from_map(sm.map[part], 0), full_a);
                sm.u.keys[0][part][lane] = part + (int)b12 * 64;
            } else {
                int part = item - na;
                float b12 = pca_bound_split<4>(blk, subset_mask_from_map(sm.map[part], 0), full_b);
                sm.u.keys[1][part][lane] = part + (int)b12 * 64;
            }
        }
    }
    __syncthreads();

    // 3. top-k (partial_sort_list, common.rs:126-140: ascending, keys unique) --
    for (int set = 0; set < 2; set++) {
        int K = set == 0 ? P.k_a : P.k_b;
        if (K == 0 || warp != (set % NW)) continue;
        for (int k = 0; k < K; k++) {
            int best = INT_MAX, bi = 0;
            for (int q = 0; q < 64; q++) {
                int v = sm.u.keys[set][q][lane];
                if (v < best) {
                    best = v;
                    bi = q;
                }
            }
            sm.list[set][k][lane] = (uint8_t)bi;
            sm.u.keys[set][bi][lane] = INT_MAX;
        }
    }
    __syncthreads();

    // 4. partition candidates of modes 0/2/1/3/7 ----------------------------------
    {
        float berr[5];
        int bcand[5];
#pragma unroll
        for (int m = 0; m < 5; m++) {
            berr[m] = __int_as_float(0x7f800000);
            bcand[m] = -1;
        }
        const int list7 = P.bounds_b ? 1 : 0;
        for (int item = warp; item < P.total; item += NW) {
            int mi = 0, ci = item;
            while (ci >= P.count[mi]) {
                ci -= P.count[mi];
                mi++;
            }
            int qep[24];
            uint32_t q0, q1;
            float err;
            switch (mi) {
                case 0: err = eval_part<0>(blk, sm.map, ci + 64, qep, q0, q1); break;
                case 1: err = eval_part<2>(blk, sm.map, ci + 64, qep, q0, q1); break;
                case 2: err = eval_part<1>(blk, sm.map, sm.list[0][ci][lane], qep, q0, q1); break;
                case 3: err = eval_part<3>(blk, sm.map, sm.list[0][ci][lane], qep, q0, q1); break;
                default: err = eval_part<7>(blk, sm.map, sm.list[list7][ci][lane], qep, q0, q1); break;
            }
#pragma unroll
            for (int m = 0; m < 5; m++)
                if (m == mi && err < berr[m]) {
                    berr[m] = err;
                    bcand[m] = ci;
                }
        }
#pragma unroll
        for (int m = 0; m < 5; m++) {
            sm.u.c.err[m][warp][lane] = berr[m];
            sm.u.c.cand[m][warp][lane] = bcand[m];
        }
    }
    __syncthreads();
    if (warp == 0) {
        for (int m = 0; m < 5; m++) {
            float be = __int_as_float(0x7f800000);
            int bc = -1;
            for (int w = 0; w < NW; w++) {
                float e = sm.u.c.err[m][w][lane];
                int c = sm.u.c.cand[m][w][lane];
                if (c >= 0 && (bc < 0 || e < be || (e == be && c < bc))) {
                    be = e;
                    bc = c;
                }
            }
            sm.winner[m][lane] = bc;
            sm.slot_err[m][lane] = be;  // unrefined error of the winner (phase 5 input)
        }
    }
    __syncthreads();

    // 5. chains: refinements, mode 4/5 candidates, mode 6 -------------------------
    {
        const int n_ref = 5, n45 = P.n45_4 + P.n45_5, n_items = n_ref + n45 + 1;
        const int list7 = P.bounds_b ? 1 : 0;
        for (int item = warp; item < n_items; item += NW) {
            float err = __int_as_float(0x7f800000);
            uint4 data = make_uint4(0, 0, 0, 0);
            if (item < n_ref) {
                int mi = item;
                int wc = sm.winner[mi][lane];
                float e0 = sm.slot_err[mi][lane];
                if (P.count[mi] > 0 && wc >= 0) {
                    float oe = sm.opaque_err[lane];
                    switch (mi) {
                        case 0: err = refine_and_code<0>(blk, sm.map, wc + 64, e0, S.refine_iterations[0], oe, data); break;
                        case 1: err = refine_and_code<2>(blk, sm.map, wc + 64, e0, S.refine_iterations[2], oe, data); break;
                        case 2:
                            err = refine_and_code<1>(blk, sm.map, sm.list[0][wc][lane], e0, S.refine_iterations[1], oe, data);
                            break;
                        case 3:
                            err = refine_and_code<3>(blk, sm.map, sm.list[0][wc][lane], e0, S.refine_iterations[3], oe, data);
                            break;
                        default:
                            err = refine_and_code<7>(blk, sm.map, sm.list[list7][wc][lane], e0, S.refine_iterations[7], oe,
                                                     data);
                            break;
                    }
                }
            } else if (item < n_ref + n45) {
                int c = item - n_ref;
                if (c < P.n45_4) {
                    int rot = (int)S.mode45_channel0 + c / 2, swap = c & 1;
                    err = mode45_candidate<4>(pxl, (int)S.channels, S.refine_iterations[4], S.refine_iterations_channel,
                                              rot, swap, data);
                } else {
                    int rot = (int)S.mode45_channel0 + (c - P.n45_4);
                    err = mode45_candidate<5>(pxl, (int)S.channels, S.refine_iterations[5], S.refine_iterations_channel,
                                              rot, 0, data);
                }
            } else if (P.run6) {
                if (S.channels == 3) err = mode6<3>(blk, S.refine_iterations[6], data);
                else err = mode6<4>(blk, S.refine_iterations[6], data);
            }
            // Refinement items overwrite the unrefined error phase 4 left in
            // their own slot; no other warp reads that slot.
            sm.slot_err[item][lane] = err;
            sm.slot_data[item][lane] = data;
        }
    }
    __syncthreads();

    // 6. select (the reference's sequential strict comparisons) --------------------
    if (warp == 0) {
        float best = __int_as_float(0x7f800000);
        uint4 data = make_uint4(0, 0, 0, 0);
        for (int s = 0; s < 5; s++) {
            float e = sm.slot_err[s][lane];
            if (e < best) {
                best = e;
                data = sm.slot_data[s][lane];
            }
        }
        const int b45 = 5;
        float be = best;
        int cand = -1;
        for (int c = 0; c < P.n45_4; c++) {
            float e = sm.slot_err[b45 + c][lane];
            if (e < be) {
                be = e;
                cand = b45 + c;
            }
        }
        if (be < best) {
            best = be;
            data = sm.slot_data[cand][lane];
        }
        for (int c = 0; c < P.n45_5; c++) {
            float e = sm.slot_err[b45 + P.n45_4 + c][lane];
            if (e < be) {
                be = e;
                cand = b45 + P.n45_4 + c;
            }
        }
        if (be < best) {
            best = be;
            data = sm.slot_data[cand][lane];
        }
        int s6 = b45 + P.n45_4 + P.n45_5;
        float e6 = sm.slot_err[s6][lane];
        if (P.run6 && e6 < best) {
            best = e6;
            data = sm.slot_data[s6][lane];
        }
        // 7. store
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

}  // namespace bc7

void launch_bc7_encode(const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst,
                       const BC7SettingsDev& settings, cudaStream_t s) {
    uint32_t n = bw * bh;
    if (n == 0) return;
    constexpr int NW = 4;
    bool aligned = ((uintptr_t)src % 16 == 0) && (stride % 16 == 0);
    uint32_t grid = (n + bc7::NB - 1) / bc7::NB;
    bc7::bc7_encode_kernel<NW><<<grid, NW * 32, 0, s>>>(src, stride, bw, n, dst, settings, aligned);
}

}  // namespace bcn
