// BC7 block-level device code shared by the encoder pipeline
// (bc7_encode.cu) and the endpoint-refinement kernels (bc7_refine.cu):
// endpoint quantisation per mode, partition-candidate evaluation, refinement
// and bit coding of every mode (src/encode/bc7.rs), in the reference's
// operation order.
#pragma once
#include "bc_common.cuh"
#include "bptc_math.cuh"

namespace bcn {
namespace bc7 {

using namespace bptc;

// Mode 4/5 candidate block (bc7.rs:680-696): channel `rot` replaced by alpha
// (4-channel settings) or by 255 (3-channel settings, whose kernel fills the
// staged alpha row with 255 first), so channel c reads row o[c]: its own or
// the alpha row, chosen once per candidate. Volatile reads: every use is a
// shared-memory load, so the compiler keeps no register copy of the block
// across the refinement loops (which cost this long kernel spills).
// The packed pixel words get the same rotation with one byte permute (byte c
// <- byte 3 for c = rot; byte 3 is outside the 3 channels read), and the
// channel square sums are read from the rotated channel's row.
template <bool CH4>
struct BlkRot {
    const float* p;
    int o[3];
    uint32_t sel;
    int rot;
    BCN_DEV BlkRot(const float* pxlane, int rot_) : p(pxlane), rot(rot_) {
        sel = 0x3210u;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            o[c] = (c == rot_ ? 48 : c * 16) * NB;
            if (c == rot_) sel = (sel & ~(0xFu << (4 * c))) | (3u << (4 * c));
        }
    }
    BCN_DEV float operator()(int c, int k) const {
        const volatile float* q = p + o[c];
        return q[k * NB];
    }
    BCN_DEV uint32_t packed(int k) const {
        const volatile float* q = p + PX_PACKED * NB;
        return __byte_perm(__float_as_uint(q[k * NB]), 0u, sel);
    }
    BCN_DEV int sq(int c) const { return __float_as_int(p[PX_SQ * NB + (o[c] >> 4)]); }
    // channels 0-2 of pixels 4g..4g+3 after the rotation, one byte per pixel
    BCN_DEV void group_bytes(int g, uint32_t c[4]) const {
        const volatile float* q = p + PX_PACKED * NB;
        uint32_t o4[4];
        transpose_bytes4(__float_as_uint(q[(4 * g) * NB]), __float_as_uint(q[(4 * g + 1) * NB]),
                         __float_as_uint(q[(4 * g + 2) * NB]), __float_as_uint(q[(4 * g + 3) * NB]), o4);
#pragma unroll
        for (int ch = 0; ch < 3; ch++) c[ch] = ch == rot ? o4[3] : o4[ch];
        c[3] = o4[3];
    }
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
                int v = (int)((div_const<255>(ep[i * 4 + p]) * (float)levels2 - (float)b) / 2.0f + 0.5f) * 2 + b;
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
            int v = (int)((div_const<255>(ep[i]) * 127.0f - (float)b) / 2.0f + 0.5f) * 2 + b;
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
    for (int i = 0; i < N; i++) qep[i] = clampi((int)(div_const<255>(ep[i]) * (float)(levels - 1) + 0.5f), 0, levels - 1);
}

// ep_quant_dequant (bc7.rs:102-237) of one endpoint pair of a partitioned
// mode: q = the quantised endpoints, e = their dequantised values; channel 3
// is handled only for mode 7 (4 channels).
template <int MODE>
BCN_DEV void quant_dequant_pair(int* q, float* e) {
    if (MODE == 0) quant0367_pair<4, 3, 3, true>(q, e);
    else if (MODE == 3) quant0367_pair<7, 3, 3, false>(q, e);
    else if (MODE == 7) quant0367_pair<5, 4, 4, false>(q, e);
    else if (MODE == 1) quant1_pair(q, e);
    else {
#pragma unroll
        for (int i = 0; i < 8; i++)
            if ((i & 3) != 3) q[i] = clampi((int)(div_const<255>(e[i]) * 31.0f + 0.5f), 0, 31);
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

// ep_quant_dequant for the partitioned modes over all their pairs.
template <int MODE>
BCN_DEV void quant_dequant_part(int qep[24], float ep[24]) {
    constexpr int pairs = (MODE == 0 || MODE == 2) ? 3 : 2;
#pragma unroll
    for (int j = 0; j < pairs; j++) quant_dequant_pair<MODE>(qep + 8 * j, ep + 8 * j);
}

// ---- candidate evaluation of modes 0/1/2/3/7 (bc7.rs:517-538) -----------------

template <int MODE>
struct ModeTraits {
    static constexpr int bits = (MODE == 0 || MODE == 1) ? 3 : 2;
    static constexpr int pairs = (MODE == 0 || MODE == 2) ? 3 : 2;
    static constexpr int ch = MODE == 7 ? 4 : 3;
};

// Unquantised endpoints (block_segment of each subset, bc7.rs:517-538) of a
// two-subset partition (modes 1, 3, 7) into ep[0..7] and ep[8..15], given
// the whole block's statistics (full[i * NB], lane-strided like the pixels).
// Every statistic is a sum of 8-bit values or of their products, an integer
// below 2^24 however it is summed, so the larger subset's statistics are the
// whole block's minus the smaller one's, bit for bit. Only the smaller
// subset is summed, which also bounds the warp's divergent loop (each lane
// has its own partition here) by 8 pixels. The result depends on the
// channel count only, not on the mode: modes 1 and 3 share it.
template <int CH, class B>
BCN_DEV void segment_part2(const B& blk, uint32_t pattern, const float* full, float ep[16]) {
#pragma unroll
    for (int i = 0; i < 16; i++) ep[i] = 0.0f;
    const uint32_t m1 = subset_mask_from_map(pattern, 1), m0 = ~m1 & 0xFFFFu;
    const bool small1 = __popc(m1) <= 8;
    float ss[15], st[15];
    stats_masked<CH, true>(blk, small1 ? m1 : m0, ss);
#pragma unroll
    for (int i = 0; i < 15; i++) st[i] = small1 ? full[i * NB] - ss[i] : ss[i];
    block_segment_from_stats<CH, true, true>(blk, m0, st, ep);
#pragma unroll
    for (int i = 0; i < 15; i++) st[i] = small1 ? ss[i] : full[i * NB] - ss[i];
    block_segment_from_stats<CH, true, true>(blk, m1, st, ep + 8);
}

// Quantisation and index fit of a two-subset candidate from its unquantised
// endpoints (ep is overwritten with the dequantised ones): its error.
template <int MODE, class B>
BCN_DEV float quant_fit_part2(const B& blk, uint32_t pattern, float ep[16]) {
    using T = ModeTraits<MODE>;
    static_assert(T::pairs == 2, "two-subset modes");
    int qep[16];
#pragma unroll
    for (int j = 0; j < 2; j++) quant_dequant_pair<MODE>(qep + 8 * j, ep + 8 * j);
    uint32_t q0, q1;
    return block_quant<T::ch, T::bits, 2, true>(blk, ep, pattern, q0, q1);
}

// One subset (pixel mask) of a mode-0 / mode-2 candidate: its endpoint fit
// (block_segment), quantisation and index fit, as the reference does them
// for each subset of a partition. Everything here depends only on the
// subset's pixels, so a subset shared by several partitions gives them the
// same result. Returns the subset's index-fit error minus its pixels' v . v
// (an exact integer; the partition's error is the sum over its subsets plus
// the block's v . v).
template <int MODE, class B>
BCN_DEV int eval_subset(const B& blk, uint32_t mask) {
    static_assert(MODE == 0 || MODE == 2, "three-subset modes");
    using T = ModeTraits<MODE>;
    float ep[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    block_segment<T::ch, true, true>(blk, mask, ep);
    int qep[8];
    quant_dequant_pair<MODE>(qep, ep);
    const FitPair f = fit_pair<T::ch>(ep);
    int total = 0;
    for (uint32_t m = mask; m; m &= m - 1) {
        int be;
        fit_pixel_pk<T::bits>(blk.packed(__ffs(m) - 1), f, be);
        total += be;
    }
    return total;
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

// Quantised endpoints of a mode (all < 256) as 24 bytes in 6 words; slots a
// mode does not code (pairs beyond its count, channel 3 below mode 7) are 0.
template <int MODE>
BCN_DEV void pack_qep(uint32_t pk[6], const int qep[24]) {
    using T = ModeTraits<MODE>;
#pragma unroll
    for (int w = 0; w < 6; w++) {
        uint32_t v = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = 4 * w + b;
            if (i / 8 < T::pairs && (i & 3) < T::ch) v |= (uint32_t)(qep[i] & 0xFF) << (8 * b);
        }
        pk[w] = v;
    }
}

// Refinement of a mode's winning partition (bc7.rs:571-609), then coding.
template <int MODE, class B>
BCN_DEV float refine_and_code(const B& blk, const uint32_t* map, int part_id, float best_err, uint32_t iters,
                              float opaque_err, uint4& out) {
    using T = ModeTraits<MODE>;
    // the best quantised endpoints (all < 256) kept as 24 bytes in 6 words
    uint32_t best_pk[6];
    uint32_t bq0 = 0, bq1 = 0;
    const uint32_t pattern = map[part_id];
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = 0.0f;
#pragma unroll
    for (int j = 0; j < T::pairs; j++)
        block_segment<T::ch, true, true>(blk, subset_mask_from_map(pattern, j), ep + 8 * j);
    // Pass 0 re-creates the winner's state (its error is best_err already);
    // passes 1..iters fit the endpoints to the best indices and keep a
    // strictly better result. One copy of the quantise + index-fit code.
    // A pass after which the best indices are unchanged is repeated exactly
    // by every later pass (same endpoint-fit input, same outcome, and a
    // repeat cannot be strictly better), so the loop stops there.
#pragma unroll 1
    for (uint32_t it = 0;; it++) {
        uint32_t pk[6], q0, q1;
        {
            int qep[24];
            quant_dequant_part<MODE>(qep, ep);
            pack_qep<MODE>(pk, qep);  // 6 words live across the index fit instead of 24
        }
        float err = block_quant<T::ch, T::bits, T::pairs, true>(blk, ep, pattern, q0, q1);
        const uint32_t pb0 = bq0, pb1 = bq1;
        if (it == 0 || err < best_err) {
#pragma unroll
            for (int i = 0; i < 6; i++) best_pk[i] = pk[i];
            bq0 = q0;
            bq1 = q1;
            if (it != 0) best_err = err;
        }
        if (it == iters || (it != 0 && bq0 == pb0 && bq1 == pb1)) break;
#pragma unroll
        for (int i = 0; i < 24; i++) ep[i] = 0.0f;
#pragma unroll
        for (int j = 0; j < T::pairs; j++)
            opt_endpoints<T::ch, T::bits, true>(ep + 8 * j, blk, bq0, bq1, subset_mask_from_map(pattern, j));
    }
    if (MODE != 7) best_err += opaque_err;
    int best_qep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) best_qep[i] = (int)((best_pk[i >> 2] >> (8 * (i & 3))) & 0xFF);
    out = code_mode01237<MODE>(best_qep, bq0, bq1, part_id);
    return best_err;
}

// ---- mode 4/5 (bc7.rs:239-369, 442-492, 657-733) ---------------------------------

// The rotated-out scalar channel of a block, read from shared memory on use
// (no register copy of its 16 values).
struct Chan {
    const float* p;  // channel row of the block's lane in the tile
    BCN_DEV float operator[](int k) const { return ((const volatile float*)p)[k * NB]; }
};

BCN_DEV void channel_quant_dequant(int qep[2], float ep[2], int epbits) {
    int elevels = 1 << epbits;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        qep[i] = clampi((int)(div_const<255>(ep[i]) * (float)(elevels - 1) + 0.5f), 0, elevels - 1);
        ep[i] = (float)unpack_to_byte(qep[i], epbits);
    }
}

template <class C>
BCN_DEV float channel_opt_quant(uint32_t& q0, uint32_t& q1, const C& cb, int bits, const float ep[2]) {
    int levels = 1 << bits;
    q0 = 0;
    q1 = 0;
    int total = 0;  // integer pixel errors (pixel_err2), exact
    // ep are dequantised values in [0, 255]: (64 - w) * ia + w * ib + 32 =
    // (64 * ia + 32) + w * (ib - ia) >= 0, so / 64 is >> 6
    int ia = (int)ep[0], ib = (int)ep[1];
    const int bs = ia * 64 + 32, df = ib - ia;
    // (cb - ep0) / den: an 8-bit difference over an 8-bit difference plus
    // 0.001, done with den's reciprocal and one fused correction step, which
    // gives the IEEE quotient for every such pair (checked exhaustively by
    // the oracle test)
    const float den = ep[1] - ep[0] + 0.001f, rden = __frcp_rn(den);
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const float x = cb[k] - ep[0], qx = x * rden;
        float proj = fmaf(fmaf(-qx, den, x), rden, qx);
        int q1i = clampi((int)(proj * (float)levels + 0.5f), 1, levels - 1);
        int w0 = bits == 2 ? bptc_w<2>(q1i - 1) : (bits == 3 ? bptc_w<3>(q1i - 1) : unquant_w(bits, q1i - 1));
        int w1 = bits == 2 ? bptc_w<2>(q1i) : (bits == 3 ? bptc_w<3>(q1i) : unquant_w(bits, q1i));
        int err0 = 0, err1 = 0;
        pixel_err2(bs, df, cb[k], w0, w1, err0, err1);
        int be = err0 < err1 ? err0 : err1;
        int bq = err0 < err1 ? q1i - 1 : q1i;
        if (k < 8) q0 |= (uint32_t)bq << (4 * k);
        else q1 |= (uint32_t)bq << (4 * (k - 8));
        total += be;
    }
    return (float)total;
}

template <class C>
BCN_DEV void channel_opt_endpoints(float ep[2], const C& cb, int bits, uint32_t q0, uint32_t q1) {
    int levels = 1 << bits;
    float lm1 = (float)(levels - 1);
    float atb1 = 0.0f, sum_q = 0.0f, sum_qq = 0.0f, sum = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float q = (float)(((k < 8 ? q0 : q1) >> (4 * (k & 7))) & 15);
        float x = lm1 - q;
        sum_q += q;
        sum_qq = mac<true>(sum_qq, q, q);
        sum += cb[k];
        atb1 = mac<true>(atb1, x, cb[k]);
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

// bc7_code_mode45 (bc7.rs:442-492): colour endpoints qep (3 channels of two
// RGBA slots), colour indices q0/q1 (2 bits, or 3 when swap = 1), scalar
// endpoints aqep and indices a0/a1 (3/2 bits in mode 4, 2 in mode 5), encoder
// rotation rot (3 = none) and the mode-4 index-selector swap.
template <int MODE>
BCN_DEV uint4 code_mode45(int qep[8], uint32_t q0, uint32_t q1, int aqep[2], uint32_t a0, uint32_t a1, int rot,
                          int swap) {
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
    return make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
}

// bc7_code_mode6 (bc7.rs:494-515): 7-bit endpoints with one p-bit each and
// 4-bit indices.
BCN_DEV uint4 code_mode6(int qep[8], uint32_t q0, uint32_t q1) {
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
    return make_uint4(bw.d[0], bw.d[1], bw.d[2], bw.d[3]);
}

// One mode-4/5 candidate: rotation `rot`, index swap SWAP (mode 4 only),
// CH4 = 4-channel settings. Returns its error and its coded block
// (bc7_code_mode45 for MODE). The index widths are compile-time so that one
// launch runs a single instruction stream.
template <int MODE, int SWAP, bool CH4>
BCN_DEV float mode45_candidate(const float* pxlane, uint32_t refine, uint32_t refine_channel, int rot, uint4& out) {
    constexpr int bits = SWAP ? 3 : 2;
    constexpr int abits = SWAP ? 2 : (MODE == 4 ? 3 : 2);
    constexpr int aepbits = MODE == 4 ? 6 : 8;
    const int swap = SWAP;
    const BlkRot<CH4> cb(pxlane, rot < 3 ? rot : -1);
    float ep[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    block_segment<3, true, true>(cb, 0xFFFFu, ep);
    // quantise + index fit, then `refine` times: endpoint fit, quantise +
    // index fit (one copy of each step in the code: the kernel is
    // instruction-cache bound). The endpoint fit depends only on the indices
    // (and the pixels): once a pass returns the indices it was given, every
    // later pass repeats it exactly, so the loop stops there.
    int qep[8];
    constexpr int EPB = MODE == 4 ? 5 : 7;
    uint32_t q0, q1, p0 = 0, p1 = 0;
    float err;
#pragma unroll 1
    for (uint32_t it = 0;; it++) {
        quant245<EPB, 8>(qep, ep);
#pragma unroll
        for (int i = 0; i < 8; i++) ep[i] = (float)unpack_to_byte(qep[i], EPB);
        err = block_quant<3, bits, 1, true>(cb, ep, 0, q0, q1);
        if (it == refine || (it != 0 && q0 == p0 && q1 == p1)) break;
        p0 = q0;
        p1 = q1;
        opt_endpoints<3, bits, true>(ep, cb, q0, q1, 0xFFFFu);
    }
    // scalar channel (opt_channel, bc7.rs:239-266)
    const Chan chan{pxlane + rot * 16 * NB};
    float aep[2] = {255.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 16; k++) {
        aep[0] = fminf(aep[0], chan[k]);
        aep[1] = fmaxf(aep[1], chan[k]);
    }
    int aqep[2];
    uint32_t a0, a1, pa0 = 0, pa1 = 0;
    float aerr;
#pragma unroll 1
    for (uint32_t it = 0;; it++) {  // stops at a repeat, as above
        channel_quant_dequant(aqep, aep, aepbits);
        aerr = channel_opt_quant(a0, a1, chan, abits, aep);
        if (it == refine_channel || (it != 0 && a0 == pa0 && a1 == pa1)) break;
        pa0 = a0;
        pa1 = a1;
        channel_opt_endpoints(aep, chan, abits, a0, a1);
    }
    err += aerr;

    out = code_mode45<MODE>(qep, q0, q1, aqep, a0, a1, rot, swap);
    return err;
}

// ---- mode 6 (bc7.rs:494-515, 762-817) -------------------------------------------

template <int CH, class B>
BCN_DEV float mode6(const B& blk, uint32_t refine, uint4& out) {
    float ep[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    block_segment<CH, true, true>(blk, 0xFFFFu, ep);
    if (CH == 3) {
        ep[3] = 255.0f;
        ep[7] = 255.0f;
    }
    // quantise + index fit, then `refine` times: endpoint fit, quantise +
    // index fit (one copy of each step in the code). A pass's input is the
    // indices and, with 3 channels, the alpha endpoints it carries over (the
    // endpoint fit writes channels 0-2 only); a pass whose output repeats its
    // input is repeated exactly by every later pass, so the loop stops there.
    int qep[8];
    uint32_t q0, q1, p0 = 0, p1 = 0;
    int pa0 = 0, pa1 = 0;
    float err;
#pragma unroll 1
    for (uint32_t it = 0;; it++) {
        quant0367_pair<7, CH, 4, false>(qep, ep);
#pragma unroll
        for (int i = 0; i < 8; i++) ep[i] = (float)qep[i];
        err = block_quant<CH, 4, 1, true>(blk, ep, 0, q0, q1);
        if (it == refine || (it != 0 && q0 == p0 && q1 == p1 && qep[3] == pa0 && qep[7] == pa1)) break;
        p0 = q0;
        p1 = q1;
        pa0 = qep[3];
        pa1 = qep[7];
        opt_endpoints<CH, 4, true>(ep, blk, q0, q1, 0xFFFFu);
    }
    out = code_mode6(qep, q0, q1);
    return err;
}

}  // namespace bc7
}  // namespace bcn
