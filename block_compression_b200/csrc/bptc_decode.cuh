// Bit-exact BC7 block decoding (the reference's src/decode/block.rs:801-1403)
// as a device function, shared by the decode kernel (bc_decode.cu) and the
// endpoint-refinement kernels (bc7_refine.cu).
#pragma once
#include "bc_common.cuh"

namespace bcn {


// 128-bit little-endian bit reader (block.rs:1341-1403).
struct Bits128 {
    uint64_t lo, hi;
    BCN_DEV uint32_t read(uint32_t n) {
        uint64_t mask = (1ull << n) - 1;
        uint32_t b = (uint32_t)(lo & mask);
        lo = (lo >> n) | ((hi & mask) << (64 - n));
        hi >>= n;
        return b;
    }
    BCN_DEV int ri(uint32_t n) { return (int)read(n); }
    BCN_DEV int rev(uint32_t n) {
        int b = ri(n), r = 0;
        for (uint32_t i = 0; i < n; i++) {
            r = (r << 1) | (b & 1);
            b >>= 1;
        }
        return r;
    }
};

// Partition-set entry (subset, 0x80 on anchors) derived from the encoder
// tables; equal to the decoder tables of block.rs:279-312 and :810-947.
BCN_DEV uint32_t partition_set(uint32_t table_index, uint32_t k) {
    uint32_t subset = (kPartitionMap[table_index] >> (2 * k)) & 3;
    uint32_t a = kAnchors[table_index];
    uint32_t anchor = subset == 0 ? 0 : (subset == 1 ? (a >> 4) : (a & 15));
    return subset | (k == anchor ? 0x80u : 0u);
}

BCN_DEV int interp(int a, int b, int w) { return (a * (64 - w) + b * w + 32) >> 6; }
BCN_DEV int w_of(int bits, int i) {
    int l1 = (1 << bits) - 1;
    return (i * 64 + (l1 >> 1)) / l1;
}

// ---- BC7 (block.rs:801-1252) --------------------------------------------------
//
// One decoder per mode: every field of a mode sits at a fixed bit position,
// so a mode compiles to straight-line funnel shifts. The index bits are read
// as one bit string in which a zero is re-inserted above each anchor index
// (anchors are stored one bit short); pixel k's index is then at bits
// [k*IB, k*IB + IB). Interpolation runs on two channels at once in 16-bit
// lanes: (e0 * (64 - w) + e1 * w + 32) >> 6 stays below 2^16 per lane.

// Partition tables in global memory: the lanes of a warp read different
// partitions, which the constant cache would serialise.
__device__ const uint32_t kDecPartitionMap[128] = {BCN_PARTITION_MAP_VALUES};
__device__ const uint8_t kDecAnchors[128] = {BCN_ANCHOR_VALUES};

// n <= 32 bits at bit `pos` of the block (d[4] = 0 pads the end).
BCN_DEV uint32_t bits_at(const uint32_t d[5], int pos, int n) {
    uint32_t v = __funnelshift_r(d[pos >> 5], d[(pos >> 5) + 1], pos & 31);
    return n == 32 ? v : (v & ((1u << n) - 1u));
}

// Up to 64 bits from bit `pos`, zero past bit 127.
BCN_DEV uint64_t bits64_at(const uint32_t d[5], int pos) {
    int w = pos >> 5, s = pos & 31;
    uint32_t x2 = w + 2 < 5 ? d[w + 2] : 0u;
    uint32_t lo = __funnelshift_r(d[w], d[w + 1], s), hi = __funnelshift_r(d[w + 1], x2, s);
    return (uint64_t)lo | ((uint64_t)hi << 32);
}

BCN_DEV uint64_t insert_zero(uint64_t x, uint32_t p) {
    uint64_t m = (1ull << p) - 1ull;
    return (x & m) | ((x & ~m) << 1);
}

// Bit replication of a P-bit value to 8 bits.
template <int P>
BCN_DEV uint32_t expand8(uint32_t v) {
    if constexpr (P >= 8) return v;
    else if constexpr (P >= 4) return (v << (8 - P)) | (v >> (2 * P - 8));
    else return v;  // never instantiated for a decoded field (P >= 4 in every mode)
}

// BPTC index weights (0..64) of 2-, 3- and 4-bit indices, as byte tables.
template <int IB>
BCN_DEV uint32_t bptc_weight(uint32_t i) {
    if (IB == 2) return __byte_perm(0x402B1500u, 0u, i | 0x4440u);  // bytes 1-3 from the zero word
    if (IB == 3) return __byte_perm(0x1B120900u, 0x40372E25u, i) & 0xFFu;
    uint32_t lo = __byte_perm(0x0D090400u, 0x1E1A1511u, i & 7u), hi = __byte_perm(0x2F2B2622u, 0x403C3733u, i & 7u);
    return ((i & 8u) ? hi : lo) & 0xFFu;
}

// Two 8-bit channels in 16-bit lanes, interpolated with one weight.
BCN_DEV uint32_t lerp2(uint32_t e0, uint32_t e1, uint32_t w) { return (e0 * (64u - w) + e1 * w + 0x00200020u) >> 6; }

// emit(k, texel) receives pixel k's RGBA8 texel (R in the low byte).
// PSTRIDE > 0: the caller gives each thread a palette of 8 words at
// pal[0], pal[PSTRIDE], ..., pal[7 * PSTRIDE] (shared memory, one column per
// thread). The two-subset modes with 2-bit indices (3 and 7) then form their
// 4 texels per subset once, with the same arithmetic as the per-pixel path
// below, and look each pixel's texel up by (subset, index) -- fewer integer
// instructions per pixel than selecting the subset's endpoints and
// interpolating 16 times. (Mode 2 would need 12 words; that much shared
// memory cost the sorted decoder a CTA per SM and measured slower.)
template <int MODE, int PSTRIDE = 0, class Emit>
BCN_DEV void decode_bc7_mode(const uint32_t d[5], Emit&& emit, uint32_t* pal = nullptr) {
    constexpr int NS = (MODE == 0 || MODE == 2) ? 3 : ((MODE == 1 || MODE == 3 || MODE == 7) ? 2 : 1);
    constexpr int NEP = 2 * NS;
    constexpr int PB = MODE == 0 ? 4 : (NS > 1 ? 6 : 0);
    constexpr int CB = MODE == 0 ? 4 : (MODE == 1 ? 6 : (MODE == 2 || MODE == 4 || MODE == 7) ? 5 : 7);
    constexpr int AB = MODE == 4 ? 6 : (MODE == 5 ? 8 : (MODE == 6 ? 7 : (MODE == 7 ? 5 : 0)));
    constexpr int PBT = (MODE == 0 || MODE == 3 || MODE == 6 || MODE == 7) ? 1 : (MODE == 1 ? 2 : 0);
    constexpr int IB = (MODE == 0 || MODE == 1) ? 3 : (MODE == 6 ? 4 : 2);
    constexpr int IB2 = MODE == 4 ? 3 : (MODE == 5 ? 2 : 0);
    constexpr int HDR = MODE + 1 + PB + ((MODE == 4 || MODE == 5) ? 2 : 0) + (MODE == 4 ? 1 : 0);
    constexpr int PP = HDR + 3 * NEP * CB + NEP * AB;
    constexpr int IS = PP + (PBT == 1 ? NEP : (PBT == 2 ? 2 : 0));
    constexpr int T1 = 16 * IB - NS;
    constexpr int PC = CB + (PBT ? 1 : 0), PA = AB + (PBT ? 1 : 0);

    uint32_t part = PB ? bits_at(d, MODE + 1, PB) : 0u;
    uint32_t rot = 0, isb = 0;
    if (MODE == 4 || MODE == 5) rot = bits_at(d, MODE + 1, 2);
    if (MODE == 4) isb = bits_at(d, MODE + 3, 1);
    uint32_t erg[NEP], eba[NEP];
#pragma unroll
    for (int j = 0; j < NEP; j++) {
        uint32_t pb = PBT == 1 ? bits_at(d, PP + j, 1) : (PBT == 2 ? bits_at(d, PP + (j >> 1), 1) : 0u);
        uint32_t c[3];
#pragma unroll
        for (int ch = 0; ch < 3; ch++) {
            uint32_t v = bits_at(d, HDR + (ch * NEP + j) * CB, CB);
            c[ch] = expand8<PC>(PBT ? ((v << 1) | pb) : v);
        }
        uint32_t a = 255u;
        if constexpr (AB > 0) {
            uint32_t v = bits_at(d, HDR + 3 * NEP * CB + j * AB, AB);
            a = expand8<PA>(PBT ? ((v << 1) | pb) : v);
        }
        erg[j] = c[0] | (c[1] << 16);
        eba[j] = c[2] | (a << 16);
    }
    uint32_t table = NS == 3 ? 64u + part : part;
    uint32_t map = NS > 1 ? __ldg(&kDecPartitionMap[table]) : 0u;
    uint64_t x = bits64_at(d, IS);
    if constexpr (T1 < 64) x &= (1ull << T1) - 1ull;
    x = insert_zero(x, IB - 1);
    if (NS == 2) {
        uint32_t a1 = __ldg(&kDecAnchors[table]) >> 4;
        x = insert_zero(x, a1 * IB + IB - 1);
    } else if (NS == 3) {
        uint32_t an = __ldg(&kDecAnchors[table]);
        uint32_t a1 = an >> 4, a2 = an & 15u;
        uint32_t lo = a1 < a2 ? a1 : a2, hi = a1 < a2 ? a2 : a1;
        x = insert_zero(x, lo * IB + IB - 1);
        x = insert_zero(x, hi * IB + IB - 1);
    }
    uint64_t y = 0;
    if constexpr (IB2 > 0) {
        y = bits64_at(d, IS + T1) & ((1ull << (16 * IB2 - 1)) - 1ull);
        y = insert_zero(y, IB2 - 1);
    }
    // Per subset: base = e0 * 64 + 32 and delta = e1 - e0 in two 16-bit lanes,
    // so a texel pair is base + delta * w. Lanes may borrow from each other in
    // the delta, but the sum is e0 * (64 - w) + e1 * w + 32 exactly (modulo
    // 2^32), whose lanes never exceed 16 bits.
    uint32_t brg[NS], drg[NS], bba[NS], dba[NS], da[NS];
#pragma unroll
    for (int j = 0; j < NS; j++) {
        brg[j] = erg[2 * j] * 64u + 0x00200020u;
        drg[j] = erg[2 * j + 1] - erg[2 * j];
        bba[j] = eba[2 * j] * 64u + 0x00200020u;
        if constexpr (IB2 > 0) {  // B and A interpolate with different weights
            dba[j] = (eba[2 * j + 1] & 0xFFFFu) - (eba[2 * j] & 0xFFFFu);
            da[j] = ((eba[2 * j + 1] >> 16) - (eba[2 * j] >> 16)) << 16;
        } else {
            dba[j] = eba[2 * j + 1] - eba[2 * j];
            da[j] = 0;
        }
    }
    if constexpr (PSTRIDE > 0 && IB == 2 && IB2 == 0 && NS == 2) {
#pragma unroll
        for (int j = 0; j < NS; j++)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t w = bptc_weight<2>((uint32_t)i);
                pal[(4 * j + i) * PSTRIDE] = __byte_perm((brg[j] + drg[j] * w) >> 6, (bba[j] + dba[j] * w) >> 6, 0x6420u);
            }
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint32_t e = ((map >> (2 * k)) & 3u) * 4u + ((uint32_t)(x >> (2 * k)) & 3u);
            emit(k, pal[e * PSTRIDE]);
        }
        return;
    }
    // rotation: swap alpha with R (1), G (2) or B (3)
    const uint32_t rot_sel = rot == 1 ? 0x0213u : (rot == 2 ? 0x1230u : (rot == 3 ? 0x2310u : 0x3210u));
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t s = NS > 1 ? ((map >> (2 * k)) & 3u) : 0u;
        uint32_t b_rg = brg[0], d_rg = drg[0], b_ba = bba[0], d_ba = dba[0], d_a = da[0];
        if constexpr (NS > 1) {
            if (s == 1) {
                b_rg = brg[1];
                d_rg = drg[1];
                b_ba = bba[1];
                d_ba = dba[1];
            }
        }
        if constexpr (NS > 2) {
            if (s == 2) {
                b_rg = brg[2];
                d_rg = drg[2];
                b_ba = bba[2];
                d_ba = dba[2];
            }
        }
        uint32_t w1 = bptc_weight<IB>((uint32_t)(x >> (k * IB)) & ((1u << IB) - 1u));
        uint32_t px;
        if constexpr (IB2 > 0) {
            uint32_t w2 = bptc_weight<IB2>((uint32_t)(y >> (k * IB2)) & ((1u << IB2) - 1u));
            uint32_t wc = isb ? w2 : w1, wa = isb ? w1 : w2;
            uint32_t rg = (b_rg + d_rg * wc) >> 6;
            uint32_t ba = (b_ba + d_ba * wc + d_a * wa) >> 6;
            px = __byte_perm(__byte_perm(rg, ba, 0x6420u), 0u, rot_sel);
        } else {
            (void)d_a;
            px = __byte_perm((b_rg + d_rg * w1) >> 6, (b_ba + d_ba * w1) >> 6, 0x6420u);
        }
        emit(k, px);
    }
}

// Decodes one BC7 block, handing each texel to emit(k, texel); a reserved
// mode encoding gives 16 zero texels.
template <int PSTRIDE = 0, class Emit>
BCN_DEV void decode_bc7_each(uint64_t lo, uint64_t hi, Emit&& emit, uint32_t* pal = nullptr) {
    const uint32_t d[5] = {(uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32), 0u};
    uint32_t low = d[0] & 0xFFu;
    int mode = low ? __ffs((int)low) - 1 : 8;
    switch (mode) {
        case 0: decode_bc7_mode<0, PSTRIDE>(d, emit, pal); break;
        case 1: decode_bc7_mode<1, PSTRIDE>(d, emit, pal); break;
        case 2: decode_bc7_mode<2, PSTRIDE>(d, emit, pal); break;
        case 3: decode_bc7_mode<3, PSTRIDE>(d, emit, pal); break;
        case 4: decode_bc7_mode<4, PSTRIDE>(d, emit, pal); break;
        case 5: decode_bc7_mode<5, PSTRIDE>(d, emit, pal); break;
        case 6: decode_bc7_mode<6, PSTRIDE>(d, emit, pal); break;
        case 7: decode_bc7_mode<7, PSTRIDE>(d, emit, pal); break;
        default:
#pragma unroll
            for (int k = 0; k < 16; k++) emit(k, 0u);
    }
}

BCN_DEV void decode_bc7_block(uint64_t lo, uint64_t hi, uint32_t out[16]) {
    decode_bc7_each(lo, hi, [&](int k, uint32_t px) { out[k] = px; });
}

}  // namespace bcn
