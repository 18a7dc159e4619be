// Shared float math of the BC6H and BC7 encoders (the reference's
// src/encode/common.rs), written for the tiled kernels: a block is read
// through a view object (planar, lane-strided shared memory), and every sum
// keeps the reference's operation order so results are bit-identical.
#pragma once
#include "bc_common.cuh"

namespace bcn {
namespace bptc {

constexpr int NB = 32;  // blocks per tile; lane l of each warp owns block l

// Planar view of one block in shared memory: channel c, pixel k. The BC7
// kernels also stage rows PX_PACKED.. (each pixel's four bytes in one word)
// and PX_SQ.. (per channel, the sum of the squares of its 16 values), which
// the integer index fit reads through packed() and sq().
constexpr int PX_PACKED = 64, PX_SQ = 80, PX_ROWS = 84;

// Transposes four pixel words (4 channel bytes each) into four channel words
// (the 4 pixels' bytes of one channel each): c[ch] byte i = w_i byte ch.
BCN_DEV void transpose_bytes4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t c[4]) {
    const uint32_t t0 = __byte_perm(w0, w1, 0x5140), t1 = __byte_perm(w2, w3, 0x5140);
    const uint32_t t2 = __byte_perm(w0, w1, 0x7362), t3 = __byte_perm(w2, w3, 0x7362);
    c[0] = __byte_perm(t0, t1, 0x5410);
    c[1] = __byte_perm(t0, t1, 0x7632);
    c[2] = __byte_perm(t2, t3, 0x5410);
    c[3] = __byte_perm(t2, t3, 0x7632);
}

struct Blk {
    const float* p;
    BCN_DEV float operator()(int c, int k) const { return p[(c * 16 + k) * NB]; }
    BCN_DEV uint32_t packed(int k) const { return __float_as_uint(p[(PX_PACKED + k) * NB]); }
    BCN_DEV int sq(int c) const { return __float_as_int(p[(PX_SQ + c) * NB]); }
    // channels 0-3 of pixels 4g..4g+3, one byte per pixel
    BCN_DEV void group_bytes(int g, uint32_t c[4]) const {
        transpose_bytes4(packed(4 * g), packed(4 * g + 1), packed(4 * g + 2), packed(4 * g + 3), c);
    }
};

// ---- shared math (src/encode/common.rs) -------------------------------------

BCN_DEV int unquant_w(int bits, int i) {
    // (i*64 + (L-1)/2) / (L-1), L = 2^bits: equals the reference table
    // get_unquant_value (common.rs:6-21) for every index.
    int l1 = (1 << bits) - 1;
    return (i * 64 + (l1 >> 1)) / l1;
}

BCN_DEV float sel3(int j, float a, float b, float c) { return j == 0 ? a : (j == 1 ? b : c); }

// Product-accumulate acc + x * y of the statistics. INT: x, y and acc are
// integers whose products and sums stay below 2^24 (8-bit pixels, at most
// 16 of them), so the product and the sum are exact either way and one fused
// multiply-add gives the same number as the reference's multiply then add.
template <bool INT>
BCN_DEV float mac(float acc, float x, float y) {
    return INT ? fmaf(x, y, acc) : acc + x * y;
}

// common.rs:294-332 over the set pixels only (adding the reference's +0.0
// terms of unset pixels changes none of the non-negative sums).
template <int CH, bool INT = false, class B>
BCN_DEV void stats_masked(const B& blk, uint32_t mask, float st[15]) {
#pragma unroll
    for (int i = 0; i < 15; i++) st[i] = 0.0f;
    for (uint32_t m = mask & 0xFFFFu; m; m &= m - 1) {
        int k = __ffs(m) - 1;
        float r = blk(0, k), g = blk(1, k), b = blk(2, k);
        st[14] += 1.0f;
        st[10] += r;
        st[11] += g;
        st[12] += b;
        st[0] = mac<INT>(st[0], r, r);
        st[1] = mac<INT>(st[1], r, g);
        st[2] = mac<INT>(st[2], r, b);
        st[4] = mac<INT>(st[4], g, g);
        st[5] = mac<INT>(st[5], g, b);
        st[7] = mac<INT>(st[7], b, b);
        if (CH == 4) {
            float a = blk(3, k);
            st[13] += a;
            st[3] = mac<INT>(st[3], r, a);
            st[6] = mac<INT>(st[6], g, a);
            st[8] = mac<INT>(st[8], b, a);
            st[9] = mac<INT>(st[9], a, a);
        }
    }
}

// x / n for an integer-valued x in [0, 2^24] and a pixel count n in
// [1, 16], r = RN(1 / n): q = RN(x * r), then one correction step
// q + RN(x - q * n) * r with fused multiply-adds (Markstein's correction,
// IBM J. Res. Develop. 34(1), 1990). Over that whole domain it equals the
// IEEE quotient x / n bit for bit (checked exhaustively on the CPU for every
// integer x in [0, 2^24] and every n), at three multiply-adds instead of a
// division.
BCN_DEV float div_count(float x, float n, float r) {
    float q = x * r;
    return fmaf(fmaf(-q, n, x), r, q);
}

// common.rs:334-350 (entries of a 3-channel call outside its 6 stay 0).
// INT: the statistics are sums of 8-bit pixel values and their products
// (integers below 2^24, BC7), so the divisions by the pixel count use
// div_count; otherwise IEEE division (BC6H's scaled half-float values).
template <int CH, bool INT = false>
BCN_DEV void covar_from_stats(float cv[10], const float st[15]) {
    const float n = st[14], r = __frcp_rn(n);  // RN(1 / n), the IEEE reciprocal
    auto dv = [&](float x) { return INT ? div_count(x, n, r) : x / n; };
    cv[0] = st[0] - dv(st[10] * st[10]);
    cv[1] = st[1] - dv(st[10] * st[11]);
    cv[2] = st[2] - dv(st[10] * st[12]);
    cv[4] = st[4] - dv(st[11] * st[11]);
    cv[5] = st[5] - dv(st[11] * st[12]);
    cv[7] = st[7] - dv(st[12] * st[12]);
    if (CH == 4) {
        cv[3] = st[3] - dv(st[10] * st[13]);
        cv[6] = st[6] - dv(st[11] * st[13]);
        cv[8] = st[8] - dv(st[12] * st[13]);
        cv[9] = st[9] - dv(st[13] * st[13]);
    } else {
        cv[3] = cv[6] = cv[8] = cv[9] = 0.0f;
    }
}

template <int CH>
BCN_DEV void ssymv(float a[4], const float c[10], const float b[4]) {
    if (CH == 3) {
        a[0] = c[0] * b[0] + c[1] * b[1] + c[2] * b[2];
        a[1] = c[1] * b[0] + c[4] * b[1] + c[5] * b[2];
        a[2] = c[2] * b[0] + c[5] * b[1] + c[7] * b[2];
    } else {
        a[0] = c[0] * b[0] + c[1] * b[1] + c[2] * b[2] + c[3] * b[3];
        a[1] = c[1] * b[0] + c[4] * b[1] + c[5] * b[2] + c[6] * b[3];
        a[2] = c[2] * b[0] + c[5] * b[1] + c[7] * b[2] + c[8] * b[3];
        a[3] = c[3] * b[0] + c[6] * b[1] + c[8] * b[2] + c[9] * b[3];
    }
}

// common.rs:260-292
template <int CH, int ITERS>
BCN_DEV void compute_axis(float axis[4], const float cv[10]) {
    float a[4] = {1.0f, 1.0f, 1.0f, 1.0f};
#pragma unroll
    for (int i = 0; i < ITERS; i++) {
        ssymv<CH>(axis, cv, a);
#pragma unroll
        for (int p = 0; p < CH; p++) a[p] = axis[p];
        if (i % 2 == 1) {
            float n = 0.0f;
#pragma unroll
            for (int p = 0; p < CH; p++) n += sqf(axis[p]);
            float rn = __frcp_rn(sqrtf(n));  // the IEEE 1 / x
#pragma unroll
            for (int p = 0; p < CH; p++) a[p] *= rn;
        }
    }
#pragma unroll
    for (int p = 0; p < CH; p++) axis[p] = a[p];
}

// common.rs:208-245
template <int CH>
BCN_DEV float pca_bound(const float cv[10]) {
    float cs[10];
    const float inv_var = 1.0f / 65536.0f;
#pragma unroll
    for (int i = 0; i < 10; i++) cs[i] = cv[i] * inv_var;
    const float eps = 0.001f * 0.001f;
    cs[0] += eps;
    cs[4] += eps;
    cs[7] += eps;
    float axis[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    compute_axis<CH, 4>(axis, cs);
    float av[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    ssymv<CH>(av, cs, axis);
    float s = 0.0f;
#pragma unroll
    for (int p = 0; p < CH; p++) s += sqf(av[p]);
    float lambda = sqrtf(s);
    float bound = cs[0] + cs[4] + cs[7];
    if (CH == 4) bound += cs[9];
    bound -= lambda;
    return fmaxf(bound, 0.0f);
}

// common.rs:396-420
template <int CH, bool INT = false>
BCN_DEV float pca_bound_split(const Blk& blk, uint32_t mask, const float full[15]) {
    float st[15], cv[10];
    stats_masked<CH, INT>(blk, mask, st);
    covar_from_stats<CH, INT>(cv, st);
    float b = 0.0f;
    b += pca_bound<CH>(cv);
#pragma unroll
    for (int i = 0; i < 15; i++) st[i] = full[i] - st[i];
    covar_from_stats<CH, INT>(cv, st);
    b += pca_bound<CH>(cv);
    return sqrtf(b) * 256.0f;
}

// Entry e of stats_masked<CH>(blk, 0xFFFF, st) alone: 0-9 the channel
// products (r*r, r*g, r*b, r*a, g*g, g*b, g*a, b*b, b*a, a*a), 10-13 the
// channel sums, 14 the pixel count; entries of alpha stay 0 when CH = 3.
// Summed over all 16 pixels in order, the same as stats_masked (8-bit
// pixels: exact integer sums).
template <int CH, class B>
BCN_DEV float stat_entry(const B& blk, int e) {
    if (e == 14) return 16.0f;
    const int ca = e < 4 ? 0 : (e < 7 ? 1 : (e < 9 ? 2 : (e == 9 ? 3 : e - 10)));
    const int cb = e < 4 ? e : (e < 7 ? e - 3 : (e < 9 ? e - 5 : 3));
    if (CH == 3 && (ca == 3 || (e < 10 && cb == 3))) return 0.0f;
    float acc = 0.0f;
    if (e >= 10) {
#pragma unroll
        for (int k = 0; k < 16; k++) acc += blk(ca, k);
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) acc = mac<true>(acc, blk(ca, k), blk(cb, k));
    }
    return acc;
}

// common.rs:483-518 (+ bc7.rs:371-379 clamp when CLAMP), from the subset's
// statistics st as stats_masked<CH> gives them (st is consumed).
template <int CH, bool CLAMP, bool INT = false, class B>
BCN_DEV void block_segment_from_stats(const B& blk, uint32_t mask, float st[15], float ep[8]) {
    float cv[10], dc[4] = {0.0f, 0.0f, 0.0f, 0.0f}, axis[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int p = 0; p < CH; p++) dc[p] = INT ? div_count(st[10 + p], st[14], __frcp_rn(st[14])) : st[10 + p] / st[14];
    covar_from_stats<CH, INT>(cv, st);
    const float inv_var = 1.0f / 65536.0f;
#pragma unroll
    for (int i = 0; i < 10; i++) cv[i] *= inv_var;
    const float eps = 0.001f * 0.001f;
    cv[0] += eps;
    cv[4] += eps;
    cv[7] += eps;
    cv[9] += eps;
    compute_axis<CH, 8>(axis, cv);
    float e0 = __int_as_float(0x7f800000), e1 = __int_as_float(0xff800000);
    for (uint32_t m = mask & 0xFFFFu; m; m &= m - 1) {
        int k = __ffs(m) - 1;
        float dot = 0.0f;
#pragma unroll
        for (int p = 0; p < CH; p++) dot += axis[p] * (blk(p, k) - dc[p]);
        e0 = fminf(e0, dot);
        e1 = fmaxf(e1, dot);
    }
    if (e1 - e0 < 1.0f) {
        e0 -= 0.5f;
        e1 += 0.5f;
    }
#pragma unroll
    for (int p = 0; p < CH; p++) {
        float a = e0 * axis[p] + dc[p];
        float b = e1 * axis[p] + dc[p];
        if (CLAMP) {
            a = clampf_r(a, 0.0f, 255.0f);
            b = clampf_r(b, 0.0f, 255.0f);
        }
        ep[p] = a;
        ep[4 + p] = b;
    }
}

// common.rs:483-518 with the statistics of the subset's pixels.
template <int CH, bool CLAMP, bool INT = false, class B>
BCN_DEV void block_segment(const B& blk, uint32_t mask, float ep[8]) {
    float st[15];
    stats_masked<CH, INT>(blk, mask, st);
    block_segment_from_stats<CH, CLAMP, INT>(blk, mask, st, ep);
}

// BPTC index weight (common.rs:6-21) of a BITS-bit index as a byte-table
// lookup: the 4/8/16 weights packed in registers and selected with a byte
// permute.
template <int BITS>
BCN_DEV int bptc_w(int i) {
    if (BITS == 2) return (int)__byte_perm(0x402B1500u, 0u, (uint32_t)i | 0x4440u);
    if (BITS == 3) return (int)(__byte_perm(0x1B120900u, 0x40372E25u, (uint32_t)i) & 0xFFu);
    uint32_t lo = __byte_perm(0x0D090400u, 0x1E1A1511u, (uint32_t)i & 7u);
    uint32_t hi = __byte_perm(0x2F2B2622u, 0x403C3733u, (uint32_t)i & 7u);
    return (int)(((i & 8) ? hi : lo) & 0xFFu);
}

template <int PAIRS, class T>
BCN_DEV T sel_pair(int j, T a, T b, T c) {
    return PAIRS == 1 ? a : (PAIRS == 2 ? (j == 0 ? a : b) : (j == 0 ? a : (j == 1 ? b : c)));
}

// Squared errors of one channel of a pixel against two index weights, in
// integers: the decoded value is d = (bs + w * df) >> 6 (bs = 64 * e0 + 32,
// df = e1 - e0, both endpoints bytes) and v is the pixel's byte (an exact
// integer in a float). Since 64 * v is a multiple of 64,
// d - v = ((bs - 64 * v) + w * df) >> 6 with an arithmetic shift. Every
// value involved is an integer well inside 2^24, so the float computation
// (d - v)^2 summed over the channels -- all exact -- gives the same numbers;
// the comparisons and totals built from them are unchanged.
BCN_DEV void pixel_err2(int bs, int df, float v, int w0, int w1, int& err0, int& err1) {
    const int bsv = bs - ((int)v << 6);
    const int a0 = (bsv + w0 * df) >> 6, a1 = (bsv + w1 * df) >> 6;
    err0 += a0 * a0;
    err1 += a1 * a1;
}

// Index-fit constants of one endpoint pair for 8-bit pixels and endpoints
// (ia / ib the pair's two endpoints per channel, df = ib - ia; channels at
// and above CH are 0 throughout):
//   pos, neg    max(df, 0) and max(-df, 0) per channel, one byte each;
//   nbase       -sum ia * df;
//   dv, rdv     sum df^2 in the reference's operation order, RN(1 / dv);
//   bs01, bs23  4 * (64 * ia + 32) of channels 0/1 (2/3) in the low / high
//               16-bit half;
//   df01, df23  the integer 4 * df_0 + 2^16 * 4 * df_1 (2/3) mod 2^32.
struct FitPair {
    uint32_t pos, neg, bs01, bs23, df01, df23;
    int nbase;
    float dv, rdv;
};

template <int CH>
BCN_DEV FitPair fit_pair(const float* ep) {
    FitPair f;
    int ia[4] = {0, 0, 0, 0}, df[4] = {0, 0, 0, 0};
    float div = 0.0f;
#pragma unroll
    for (int p = 0; p < CH; p++) {
        const float d = ep[4 + p] - ep[p];
        div += sqf(d);
        ia[p] = (int)ep[p];
        df[p] = (int)ep[4 + p] - ia[p];
    }
    f.dv = div;
    f.rdv = __frcp_rn(div);
    f.pos = 0;
    f.neg = 0;
    f.nbase = 0;
#pragma unroll
    for (int p = 0; p < CH; p++) {
        f.pos |= (uint32_t)max(df[p], 0) << (8 * p);
        f.neg |= (uint32_t)max(-df[p], 0) << (8 * p);
        f.nbase -= ia[p] * df[p];
    }
    uint32_t bs[4];
#pragma unroll
    for (int p = 0; p < 4; p++) bs[p] = p < CH ? (uint32_t)(256 * ia[p] + 128) : 0u;
    f.bs01 = bs[0] + (bs[1] << 16);
    f.bs23 = bs[2] + (bs[3] << 16);
    f.df01 = (uint32_t)(4 * df[0]) + ((uint32_t)(4 * df[1]) << 16);
    f.df23 = (uint32_t)(4 * df[2]) + ((uint32_t)(4 * df[3]) << 16);
    return f;
}

template <int PAIRS>
BCN_DEV FitPair sel_fit(int j, const FitPair* f) {
    const FitPair& a = f[0];
    const FitPair& b = f[PAIRS > 1 ? 1 : 0];
    const FitPair& c = f[PAIRS > 2 ? 2 : 0];
    FitPair r;
    r.pos = sel_pair<PAIRS>(j, a.pos, b.pos, c.pos);
    r.neg = sel_pair<PAIRS>(j, a.neg, b.neg, c.neg);
    r.bs01 = sel_pair<PAIRS>(j, a.bs01, b.bs01, c.bs01);
    r.bs23 = sel_pair<PAIRS>(j, a.bs23, b.bs23, c.bs23);
    r.df01 = sel_pair<PAIRS>(j, a.df01, b.df01, c.df01);
    r.df23 = sel_pair<PAIRS>(j, a.df23, b.df23, c.df23);
    r.nbase = sel_pair<PAIRS>(j, a.nbase, b.nbase, c.nbase);
    r.dv = sel_pair<PAIRS>(j, a.dv, b.dv, c.dv);
    r.rdv = sel_pair<PAIRS>(j, a.rdv, b.rdv, c.rdv);
    return r;
}

// One pixel of block_quant's integer path: v = the pixel's bytes packed in a
// word (channels at and above the pair's CH are ignored: their pos, neg, bs
// and df bytes are 0). Every quantity is an exact integer:
//   * the projection sum (v - ia) . df is sum v * df - sum ia * df, with
//     sum v * df = v . pos - v . neg (byte dot products); the reference's
//     float sum of exact integer terms is that integer. The quotient by dv is
//     the reciprocal and one fused correction step (exact for all such
//     integer pairs);
//   * the decoded value of index weight w is d = (64 * ia + 32 + w * df) >> 6,
//     and 4 * (64 * ia + 32 + w * df) lies in [128, 65408], so
//     bs01 + w * df01 holds it for channels 0 and 1 in its two 16-bit halves
//     (no borrow between them) and byte 1 of each half is d: one byte permute
//     gathers the four decoded channels d (0 above CH);
//   * the squared error sum (d - v)^2 over the channels is
//     d . d - 2 d . v + v . v; the last term is the same for both candidate
//     indices and is added once per block by the caller.
// So the index chosen and its error are the reference's (errors compared
// with the same strict "<"). Returns the index; be = its error minus v . v.
template <int BITS>
BCN_DEV uint32_t fit_pixel_pk(uint32_t v, const FitPair& f, int& be) {
    constexpr int levels = 1 << BITS;
    float proj = (float)(int)(__dp4a(v, f.pos, (uint32_t)f.nbase) - __dp4a(v, f.neg, 0u));
    const float q = proj * f.rdv;
    proj = fmaf(fmaf(-q, f.dv, proj), f.rdv, q);
    const int q1i = clampi((int)(proj * (float)levels + 0.5f), 1, levels - 1);
    const uint32_t w0 = (uint32_t)bptc_w<BITS>(q1i - 1), w1 = (uint32_t)bptc_w<BITS>(q1i);
    const uint32_t d0 = __byte_perm(f.bs01 + w0 * f.df01, f.bs23 + w0 * f.df23, 0x7531);
    const uint32_t d1 = __byte_perm(f.bs01 + w1 * f.df01, f.bs23 + w1 * f.df23, 0x7531);
    const int e0 = (int)__dp4a(d0, d0, 0u) - 2 * (int)__dp4a(d0, v, 0u);
    const int e1 = (int)__dp4a(d1, d1, 0u) - 2 * (int)__dp4a(d1, v, 0u);
    be = e1;
    uint32_t bq = (uint32_t)q1i;
    if (e0 < e1) {
        be = e0;
        bq = (uint32_t)q1i - 1u;
    }
    return bq;
}

// sum over the block's pixels of v . v over the first CH channels
template <int CH, class B>
BCN_DEV int block_sq(const B& blk) {
    int s = blk.sq(0) + blk.sq(1) + blk.sq(2);
    if (CH == 4) s += blk.sq(3);
    return s;
}

// common.rs:422-481. ep holds PAIRS endpoint pairs at stride 8, dequantised
// values in [0, 255]. Everything that depends only on the pair is computed
// once per pair with the reference's own operations (so the per-pixel values
// are the same numbers): eb - ea, the sum of its squares, and the decoder's
// interpolation (64 - w) * ia + w * ib + 32 written as
// (64 * ia + 32) + w * (ib - ia), which is non-negative, so / 64 is >> 6.
// INT: pixels and endpoints are 8-bit integers (BC7), so each pixel is
// fitted in integer arithmetic by fit_pixel_pk from the block's packed
// pixel words (the projection is an integer divided by an integer, both at
// most 4 * 255^2 in magnitude, taken with the divisor's reciprocal and one
// fused correction step, which equals the IEEE quotient over that whole
// domain -- checked exhaustively by the oracle test -- and the pixel errors
// and their total are exact integers, below 2^24). Otherwise the float path
// with IEEE division (BC6H).
template <int CH, int BITS, int PAIRS, bool INT = false, class B>
BCN_DEV float block_quant(const B& blk, const float* ep, uint32_t pattern, uint32_t& q0, uint32_t& q1) {
    if constexpr (INT) {
        FitPair fp[PAIRS];
#pragma unroll
        for (int j = 0; j < PAIRS; j++) fp[j] = fit_pair<CH>(ep + 8 * j);
        int total = 0;
        q0 = 0;
        q1 = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int j = PAIRS == 1 ? 0 : (int)((pattern >> (2 * k)) & 3);
            int be;
            const uint32_t bq = fit_pixel_pk<BITS>(blk.packed(k), sel_fit<PAIRS>(j, fp), be);
            if (k < 8) q0 |= bq << (4 * k);
            else q1 |= bq << (4 * (k - 8));
            total += be;
        }
        return (float)(total + block_sq<CH>(blk));
    }
    // float path (BC6H): IEEE division
    constexpr int levels = 1 << BITS;
    float dd[PAIRS][CH], dv[PAIRS];
    int base[PAIRS][CH], dif[PAIRS][CH];
#pragma unroll
    for (int j = 0; j < PAIRS; j++) {
        float div = 0.0f;
#pragma unroll
        for (int p = 0; p < CH; p++) {
            dd[j][p] = ep[8 * j + 4 + p] - ep[8 * j + p];
            div += sqf(dd[j][p]);
            int ia = (int)ep[8 * j + p], ib = (int)ep[8 * j + 4 + p];
            base[j][p] = ia * 64 + 32;
            dif[j][p] = ib - ia;
        }
        dv[j] = div;
    }
    float total = 0.0f;
    q0 = 0;
    q1 = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        int j = PAIRS == 1 ? 0 : (int)((pattern >> (2 * k)) & 3);
        float proj = 0.0f;
#pragma unroll
        for (int p = 0; p < CH; p++) {
            // indices stay inside the caller's PAIRS * 8 endpoint array
            float ea = sel_pair<PAIRS>(j, ep[p], ep[PAIRS > 1 ? 8 + p : p], ep[PAIRS > 2 ? 16 + p : p]);
            float d = sel_pair<PAIRS>(j, dd[0][p], dd[PAIRS > 1 ? 1 : 0][p], dd[PAIRS > 2 ? 2 : 0][p]);
            proj += (blk(p, k) - ea) * d;
        }
        proj /= sel_pair<PAIRS>(j, dv[0], dv[PAIRS > 1 ? 1 : 0], dv[PAIRS > 2 ? 2 : 0]);
        int q1i = clampi((int)(proj * (float)levels + 0.5f), 1, levels - 1);
        int w0 = bptc_w<BITS>(q1i - 1), w1 = bptc_w<BITS>(q1i);
        float err0 = 0.0f, err1 = 0.0f;
#pragma unroll
        for (int p = 0; p < CH; p++) {
            int bs = sel_pair<PAIRS>(j, base[0][p], base[PAIRS > 1 ? 1 : 0][p], base[PAIRS > 2 ? 2 : 0][p]);
            int df = sel_pair<PAIRS>(j, dif[0][p], dif[PAIRS > 1 ? 1 : 0][p], dif[PAIRS > 2 ? 2 : 0][p]);
            float v = blk(p, k);
            float d0 = (float)((uint32_t)(bs + w0 * df) >> 6);
            float d1 = (float)((uint32_t)(bs + w1 * df) >> 6);
            err0 += sqf(d0 - v);
            err1 += sqf(d1 - v);
        }
        float be = err1;
        int bq = q1i;
        if (err0 < err1) {
            be = err0;
            bq = q1i - 1;
        }
        if (k < 8) q0 |= (uint32_t)bq << (4 * k);
        else q1 |= (uint32_t)bq << (4 * (k - 8));
        total += be;
    }
    return total;
}

// common.rs:142-205. Writes ep[0..CH) and ep[4..4+CH). INT: 8-bit pixels
// (the sums of index and pixel products are exact integers, see mac).
// INT: 8-bit pixels, so every sum is an exact integer below 2^24, in any
// order: they are taken four pixels at a time as byte dot products of the
// channel bytes (group_bytes), the index bytes and the subset's pixel mask
// bytes, and converted to float once (the same values as the reference's
// float sums).
template <int CH, int BITS, bool INT = false, class B>
BCN_DEV void opt_endpoints(float* ep, const B& blk, uint32_t q0, uint32_t q1, uint32_t mask) {
    constexpr int levels = 1 << BITS;
    const float lm1 = (float)(levels - 1);
    float atb1[4] = {0.0f, 0.0f, 0.0f, 0.0f}, sum[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float sum_q = 0.0f, sum_qq = 0.0f;
    if constexpr (INT) {
        uint32_t sq = 0, sqq = 0, sc[4] = {0, 0, 0, 0}, at[4] = {0, 0, 0, 0};
        const uint32_t lmb = (uint32_t)(levels - 1) * 0x01010101u;
#pragma unroll
        for (int g = 0; g < 4; g++) {
            uint32_t c[4];
            blk.group_bytes(g, c);
            // index bytes of pixels 4g..4g+3 (nibbles of q0 / q1)
            const uint32_t h = (g < 2 ? q0 : q1) >> (16 * (g & 1));
            const uint32_t qb = __byte_perm(h & 0x0F0Fu, (h >> 4) & 0x0F0Fu, 0x5140);
            // mask bit of pixel 4g+i -> byte i (0 or 1), and 0 / 0xFF
            const uint32_t mb = (((mask >> (4 * g)) & 0xFu) * 0x00204081u) & 0x01010101u, mf = mb * 0xFFu;
            const uint32_t xb = (lmb - qb) & mf;  // bytes lm1 - q of the subset's pixels
            sq = __dp4a(qb, mb, sq);
            sqq = __dp4a(qb & mf, qb, sqq);
#pragma unroll
            for (int p = 0; p < CH; p++) {
                sc[p] = __dp4a(c[p], mb, sc[p]);
                at[p] = __dp4a(c[p], xb, at[p]);
            }
        }
        sum_q = (float)sq;
        sum_qq = (float)sqq;
        sum[4] = (float)__popc(mask & 0xFFFFu);
#pragma unroll
        for (int p = 0; p < CH; p++) {
            sum[p] = (float)sc[p];
            atb1[p] = (float)at[p];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            float q = (float)(((k < 8 ? q0 : q1) >> (4 * (k & 7))) & 15);
            if (((mask >> k) & 1) == 0) continue;
            float x = lm1 - q;
            sum_q += q;
            sum_qq += q * q;
            sum[4] += 1.0f;
#pragma unroll
            for (int p = 0; p < CH; p++) {
                float v = blk(p, k);
                sum[p] += v;
                atb1[p] += x * v;
            }
        }
    }
    float atb2[4];
#pragma unroll
    for (int p = 0; p < CH; p++) atb2[p] = lm1 * sum[p] - atb1[p];
    float cxx = sum[4] * sqf(lm1) - 2.0f * lm1 * sum_q + sum_qq;
    float cyy = sum_qq;
    float cxy = lm1 * sum_q - sum_qq;
    float det = cxx * cyy - cxy * cxy;
    float scale = lm1 / det;
#pragma unroll
    for (int p = 0; p < CH; p++) {
        ep[p] = (atb1[p] * cyy - atb2[p] * cxy) * scale;
        ep[4 + p] = (atb2[p] * cxx - atb1[p] * cxy) * scale;
    }
    if (fabsf(det) < 0.001f) {
#pragma unroll
        for (int p = 0; p < CH; p++) {
            ep[p] = sum[p] / sum[4];
            ep[4 + p] = ep[p];
        }
    }
}

BCN_DEV int unpack_to_byte(int v, int bits) {
    int vv = v << (8 - bits);
    return vv + (vv >> bits);
}

}  // namespace bptc
}  // namespace bcn
