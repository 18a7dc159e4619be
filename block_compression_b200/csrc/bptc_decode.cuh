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

BCN_DEV void decode_bc7_block(uint64_t lo, uint64_t hi, uint32_t out[16]) {
    const uint32_t abits0 = 0x57757564u;  // RGB bits per mode, 4 bits each: 4,6,5,7,5,7,7,5
    const uint32_t abits1 = 0x57860000u;  // alpha bits per mode: 0,0,0,0,6,8,7,5
    const uint32_t has_pbits = 0xCB;
    Bits128 bs{lo, hi};
    uint32_t mode = 0;
    while (mode < 8 && bs.read(1) == 0) mode++;
    if (mode >= 8) {
        for (int k = 0; k < 16; k++) out[k] = 0;
        return;
    }
    uint32_t cbits = (abits0 >> (4 * mode)) & 15, abits = (abits1 >> (4 * mode)) & 15;
    uint32_t partition = 0, nparts = 1, rotation = 0, isb = 0;
    if (mode == 0 || mode == 1 || mode == 2 || mode == 3 || mode == 7) {
        nparts = (mode == 0 || mode == 2) ? 3 : 2;
        partition = bs.read(mode == 0 ? 4 : 6);
    }
    uint32_t nep = nparts * 2;
    if (mode == 4 || mode == 5) {
        rotation = bs.read(2);
        if (mode == 4) isb = bs.read(1);
    }
    int ep[6][4];
#pragma unroll
    for (int j = 0; j < 6; j++)
#pragma unroll
        for (int c = 0; c < 4; c++) ep[j][c] = 0;
    for (int c = 0; c < 3; c++)
        for (uint32_t j = 0; j < nep; j++) {
            int v = (int)bs.read(cbits);
#pragma unroll
            for (int jj = 0; jj < 6; jj++)
                if (jj == (int)j) ep[jj][c] = v;
        }
    if (abits > 0)
        for (uint32_t j = 0; j < nep; j++) {
            int v = (int)bs.read(abits);
#pragma unroll
            for (int jj = 0; jj < 6; jj++)
                if (jj == (int)j) ep[jj][3] = v;
        }
    uint32_t pb = (has_pbits >> mode) & 1;
    if (mode == 0 || mode == 1 || mode == 3 || mode == 6 || mode == 7) {
#pragma unroll
        for (int j = 0; j < 6; j++)
#pragma unroll
            for (int c = 0; c < 4; c++) ep[j][c] <<= 1;
        if (mode == 1) {
            int i0 = (int)bs.read(1), j0 = (int)bs.read(1);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                ep[0][c] |= i0;
                ep[1][c] |= i0;
                ep[2][c] |= j0;
                ep[3][c] |= j0;
            }
        } else if (pb) {
            for (uint32_t j = 0; j < nep; j++) {
                int b = (int)bs.read(1);
#pragma unroll
                for (int jj = 0; jj < 6; jj++)
                    if (jj == (int)j)
#pragma unroll
                        for (int c = 0; c < 4; c++) ep[jj][c] |= b;
            }
        }
    }
    {
        uint32_t jc = cbits + pb, ja = abits + pb;
#pragma unroll
        for (int j = 0; j < 6; j++) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                ep[j][c] <<= 8 - jc;
                ep[j][c] |= ep[j][c] >> jc;
            }
            ep[j][3] <<= 8 - ja;
            ep[j][3] |= ep[j][3] >> ja;
            if (abits == 0) ep[j][3] = 0xFF;
        }
    }
    uint32_t ib = (mode == 0 || mode == 1) ? 3 : (mode == 6 ? 4 : 2);
    uint32_t ib2 = mode == 4 ? 3 : (mode == 5 ? 2 : 0);
    uint32_t table = nparts == 3 ? 64 + partition : partition;
    uint32_t idx[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t ps = nparts == 1 ? (k == 0 ? 0x80u : 0u) : partition_set(table, k);
        idx[k] = bs.read((ps & 0x80) ? ib - 1 : ib);
    }
#pragma unroll
    for (int k = 0; k < 16; k++) {
        uint32_t s = nparts == 1 ? 0u : (partition_set(table, k) & 3);
        const int* e0 = s == 0 ? ep[0] : (s == 1 ? ep[2] : ep[4]);
        const int* e1 = s == 0 ? ep[1] : (s == 1 ? ep[3] : ep[5]);
        int r, g, b, a;
        int w = w_of((int)ib, (int)idx[k]);
        if (ib2 == 0) {
            r = interp(e0[0], e1[0], w);
            g = interp(e0[1], e1[1], w);
            b = interp(e0[2], e1[2], w);
            a = interp(e0[3], e1[3], w);
        } else {
            int i2 = (int)bs.read(k == 0 ? ib2 - 1 : ib2);
            int w2 = w_of((int)ib2, i2);
            if (isb == 0) {
                r = interp(e0[0], e1[0], w);
                g = interp(e0[1], e1[1], w);
                b = interp(e0[2], e1[2], w);
                a = interp(e0[3], e1[3], w2);
            } else {
                r = interp(e0[0], e1[0], w2);
                g = interp(e0[1], e1[1], w2);
                b = interp(e0[2], e1[2], w2);
                a = interp(e0[3], e1[3], w);
            }
        }
        int t;
        if (rotation == 1) {
            t = a;
            a = r;
            r = t;
        } else if (rotation == 2) {
            t = a;
            a = g;
            g = t;
        } else if (rotation == 3) {
            t = a;
            a = b;
            b = t;
        }
        out[k] = (uint32_t)(r & 0xFF) | ((uint32_t)(g & 0xFF) << 8) | ((uint32_t)(b & 0xFF) << 16) |
                 ((uint32_t)(a & 0xFF) << 24);
    }
}
}  // namespace bcn
