// BC6H and BC7 decode kernels for sm_100a (bit-exact restatement of the
// reference decoders, src/decode/block.rs:262-1403, and of the image drivers'
// output layouts, src/decode.rs:151-324).
//
// One thread decodes one block; a warp covers 32 neighbouring blocks, so the
// 16-byte block reads are one contiguous 512-byte span and each output row
// of the warp is a contiguous span.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bptc_decode.cuh"

namespace bcn {


__global__ void __launch_bounds__(128) bc7_decode_kernel(const uint8_t* __restrict__ blocks, uint32_t bw, uint32_t bh,
                                                         uint8_t* __restrict__ out, size_t pitch, bool aligned) {
    uint32_t n = bw * bh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t by = i / bw, bx = i - by * bw;
        uint64_t lo = 0, hi = 0;
        const uint8_t* b = blocks + (size_t)i * 16;
        if (aligned) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(b));
            lo = (uint64_t)v.x | ((uint64_t)v.y << 32);
            hi = (uint64_t)v.z | ((uint64_t)v.w << 32);
        } else {
            for (int j = 0; j < 8; j++) lo |= (uint64_t)b[j] << (8 * j);
            for (int j = 0; j < 8; j++) hi |= (uint64_t)b[8 + j] << (8 * j);
        }
        uint32_t px[16];
        decode_bc7_block(lo, hi, px);
#pragma unroll
        for (int y = 0; y < 4; y++) {
            uint8_t* row = out + (size_t)(by * 4 + y) * pitch + (size_t)bx * 16;
            if (aligned) {
                *reinterpret_cast<uint4*>(row) = make_uint4(px[y * 4], px[y * 4 + 1], px[y * 4 + 2], px[y * 4 + 3]);
            } else {
                for (int x = 0; x < 4; x++)
                    for (int c = 0; c < 4; c++) row[4 * x + c] = (uint8_t)(px[y * 4 + x] >> (8 * c));
            }
        }
    }
}

// ---- BC6H (block.rs:262-796) -----------------------------------------------------

BCN_DEV int extend_sign(int v, int bits) { return (int)((uint32_t)v << (32 - bits)) >> (32 - bits); }

BCN_DEV int unquantize_u(int v, int bits) {
    if (bits >= 15) return v;
    if (v == 0) return 0;
    if (v == (1 << bits) - 1) return 0xFFFF;
    return ((v << 16) + 0x8000) >> bits;
}

// Unsigned BC6H (the only form the image drivers use): 16 pixels of RGB
// f16 bit patterns.
BCN_DEV void decode_bc6h_block_u(uint64_t lo, uint64_t hi, uint16_t out[48]) {
    Bits128 bs{lo, hi};
    int r[4] = {0, 0, 0, 0}, g[4] = {0, 0, 0, 0}, b[4] = {0, 0, 0, 0};
    uint32_t mode = bs.read(2);
    if (mode > 1) mode |= bs.read(3) << 2;
    int part = 0;
    switch (mode) {
        case 0x00:
            g[2] |= bs.ri(1) << 4; b[2] |= bs.ri(1) << 4; b[3] |= bs.ri(1) << 4;
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(5); g[3] |= bs.ri(1) << 4; g[2] |= bs.ri(4);
            g[1] |= bs.ri(5); b[3] |= bs.ri(1); g[3] |= bs.ri(4);
            b[1] |= bs.ri(5); b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4);
            r[2] |= bs.ri(5); b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(5);
            b[3] |= bs.ri(1) << 3; part = bs.ri(5); mode = 0;
            break;
        case 0x01:
            g[2] |= bs.ri(1) << 5; g[3] |= bs.ri(1) << 4; g[3] |= bs.ri(1) << 5;
            r[0] |= bs.ri(7); b[3] |= bs.ri(1); b[3] |= bs.ri(1) << 1;
            b[2] |= bs.ri(1) << 4; g[0] |= bs.ri(7); b[2] |= bs.ri(1) << 5;
            b[3] |= bs.ri(1) << 2; g[2] |= bs.ri(1) << 4; b[0] |= bs.ri(7);
            b[3] |= bs.ri(1) << 3; b[3] |= bs.ri(1) << 5; b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(6); g[2] |= bs.ri(4); g[1] |= bs.ri(6);
            g[3] |= bs.ri(4); b[1] |= bs.ri(6); b[2] |= bs.ri(4);
            r[2] |= bs.ri(6); r[3] |= bs.ri(6); part = bs.ri(5); mode = 1;
            break;
        case 0x02:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(5); r[0] |= bs.ri(1) << 10; g[2] |= bs.ri(4);
            g[1] |= bs.ri(4); g[0] |= bs.ri(1) << 10; b[3] |= bs.ri(1);
            g[3] |= bs.ri(4); b[1] |= bs.ri(4); b[0] |= bs.ri(1) << 10;
            b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4); r[2] |= bs.ri(5);
            b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(5); b[3] |= bs.ri(1) << 3;
            part = bs.ri(5); mode = 2;
            break;
        case 0x06:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(4); r[0] |= bs.ri(1) << 10; g[3] |= bs.ri(1) << 4;
            g[2] |= bs.ri(4); g[1] |= bs.ri(5); g[0] |= bs.ri(1) << 10;
            g[3] |= bs.ri(4); b[1] |= bs.ri(4); b[0] |= bs.ri(1) << 10;
            b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4); r[2] |= bs.ri(4);
            b[3] |= bs.ri(1); b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(4);
            g[2] |= bs.ri(1) << 4; b[3] |= bs.ri(1) << 3; part = bs.ri(5); mode = 3;
            break;
        case 0x0A:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(4); r[0] |= bs.ri(1) << 10; b[2] |= bs.ri(1) << 4;
            g[2] |= bs.ri(4); g[1] |= bs.ri(4); g[0] |= bs.ri(1) << 10;
            b[3] |= bs.ri(1); g[3] |= bs.ri(4); b[1] |= bs.ri(5);
            b[0] |= bs.ri(1) << 10; b[2] |= bs.ri(4); r[2] |= bs.ri(4);
            b[3] |= bs.ri(1) << 1; b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(4);
            b[3] |= bs.ri(1) << 4; b[3] |= bs.ri(1) << 3; part = bs.ri(5); mode = 4;
            break;
        case 0x0E:
            r[0] |= bs.ri(9); b[2] |= bs.ri(1) << 4; g[0] |= bs.ri(9);
            g[2] |= bs.ri(1) << 4; b[0] |= bs.ri(9); b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(5); g[3] |= bs.ri(1) << 4; g[2] |= bs.ri(4);
            g[1] |= bs.ri(5); b[3] |= bs.ri(1); g[3] |= bs.ri(4);
            b[1] |= bs.ri(5); b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4);
            r[2] |= bs.ri(5); b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(5);
            b[3] |= bs.ri(1) << 3; part = bs.ri(5); mode = 5;
            break;
        case 0x12:
            r[0] |= bs.ri(8); g[3] |= bs.ri(1) << 4; b[2] |= bs.ri(1) << 4;
            g[0] |= bs.ri(8); b[3] |= bs.ri(1) << 2; g[2] |= bs.ri(1) << 4;
            b[0] |= bs.ri(8); b[3] |= bs.ri(1) << 3; b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(6); g[2] |= bs.ri(4); g[1] |= bs.ri(5);
            b[3] |= bs.ri(1); g[3] |= bs.ri(4); b[1] |= bs.ri(5);
            b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4); r[2] |= bs.ri(6);
            r[3] |= bs.ri(6); part = bs.ri(5); mode = 6;
            break;
        case 0x16:
            r[0] |= bs.ri(8); b[3] |= bs.ri(1); b[2] |= bs.ri(1) << 4;
            g[0] |= bs.ri(8); g[2] |= bs.ri(1) << 5; g[2] |= bs.ri(1) << 4;
            b[0] |= bs.ri(8); g[3] |= bs.ri(1) << 5; b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(5); g[3] |= bs.ri(1) << 4; g[2] |= bs.ri(4);
            g[1] |= bs.ri(6); g[3] |= bs.ri(4); b[1] |= bs.ri(5);
            b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(4); r[2] |= bs.ri(5);
            b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(5); b[3] |= bs.ri(1) << 3;
            part = bs.ri(5); mode = 7;
            break;
        case 0x1A:
            r[0] |= bs.ri(8); b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(1) << 4;
            g[0] |= bs.ri(8); b[2] |= bs.ri(1) << 5; g[2] |= bs.ri(1) << 4;
            b[0] |= bs.ri(8); b[3] |= bs.ri(1) << 5; b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(5); g[3] |= bs.ri(1) << 4; g[2] |= bs.ri(4);
            g[1] |= bs.ri(5); b[3] |= bs.ri(1); g[3] |= bs.ri(4);
            b[1] |= bs.ri(6); b[2] |= bs.ri(4); r[2] |= bs.ri(5);
            b[3] |= bs.ri(1) << 2; r[3] |= bs.ri(5); b[3] |= bs.ri(1) << 3;
            part = bs.ri(5); mode = 8;
            break;
        case 0x1E:
            r[0] |= bs.ri(6); g[3] |= bs.ri(1) << 4; b[3] |= bs.ri(1);
            b[3] |= bs.ri(1) << 1; b[2] |= bs.ri(1) << 4; g[0] |= bs.ri(6);
            g[2] |= bs.ri(1) << 5; b[2] |= bs.ri(1) << 5; b[3] |= bs.ri(1) << 2;
            g[2] |= bs.ri(1) << 4; b[0] |= bs.ri(6); g[3] |= bs.ri(1) << 5;
            b[3] |= bs.ri(1) << 3; b[3] |= bs.ri(1) << 5; b[3] |= bs.ri(1) << 4;
            r[1] |= bs.ri(6); g[2] |= bs.ri(4); g[1] |= bs.ri(6);
            g[3] |= bs.ri(4); b[1] |= bs.ri(6); b[2] |= bs.ri(4);
            r[2] |= bs.ri(6); r[3] |= bs.ri(6); part = bs.ri(5); mode = 9;
            break;
        case 0x03:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(10); g[1] |= bs.ri(10); b[1] |= bs.ri(10);
            mode = 10;
            break;
        case 0x07:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(9); r[0] |= bs.ri(1) << 10; g[1] |= bs.ri(9);
            g[0] |= bs.ri(1) << 10; b[1] |= bs.ri(9); b[0] |= bs.ri(1) << 10;
            mode = 11;
            break;
        case 0x0B:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(8); r[0] |= bs.rev(2) << 10; g[1] |= bs.ri(8);
            g[0] |= bs.rev(2) << 10; b[1] |= bs.ri(8); b[0] |= bs.rev(2) << 10;
            mode = 12;
            break;
        case 0x0F:
            r[0] |= bs.ri(10); g[0] |= bs.ri(10); b[0] |= bs.ri(10);
            r[1] |= bs.ri(4); r[0] |= bs.rev(6) << 10; g[1] |= bs.ri(4);
            g[0] |= bs.rev(6) << 10; b[1] |= bs.ri(4); b[0] |= bs.rev(6) << 10;
            mode = 13;
            break;
        default:
            for (int i = 0; i < 48; i++) out[i] = 0;
            return;
    }
    // ACTUAL_BITS_COUNT (block.rs:269-274)
    const uint8_t kB0[14] = {10, 7, 11, 11, 11, 9, 8, 8, 8, 6, 10, 11, 12, 16};
    const uint8_t kBR[14] = {5, 6, 5, 4, 4, 5, 6, 5, 5, 6, 10, 9, 8, 4};
    const uint8_t kBG[14] = {5, 6, 4, 5, 4, 5, 5, 6, 5, 6, 10, 9, 8, 4};
    const uint8_t kBB[14] = {5, 6, 4, 4, 5, 5, 5, 5, 6, 6, 10, 9, 8, 4};
    int np = mode >= 10 ? 0 : 1;
    int bits0 = kB0[mode];
    if (mode != 9 && mode != 10) {
        for (int i = 1; i < (np + 1) * 2; i++) {
            int rr = extend_sign(i == 1 ? r[1] : (i == 2 ? r[2] : r[3]), kBR[mode]);
            int gg = extend_sign(i == 1 ? g[1] : (i == 2 ? g[2] : g[3]), kBG[mode]);
            int bb = extend_sign(i == 1 ? b[1] : (i == 2 ? b[2] : b[3]), kBB[mode]);
            int m = (1 << bits0) - 1;
            rr = (rr + r[0]) & m;
            gg = (gg + g[0]) & m;
            bb = (bb + b[0]) & m;
            if (i == 1) { r[1] = rr; g[1] = gg; b[1] = bb; }
            else if (i == 2) { r[2] = rr; g[2] = gg; b[2] = bb; }
            else { r[3] = rr; g[3] = gg; b[3] = bb; }
        }
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (i >= (np + 1) * 2) break;
        r[i] = unquantize_u(r[i], bits0);
        g[i] = unquantize_u(g[i], bits0);
        b[i] = unquantize_u(b[i], bits0);
    }
    // Index bits: 46 bits from bit 82 (two subsets, 3-bit indices) or 63 bits
    // from bit 65 (one subset, 4-bit); a zero is re-inserted above each anchor
    // index so that pixel k's index sits at bits [k*ib, k*ib + ib).
    const uint32_t d[5] = {(uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32), 0u};
    uint32_t map = 0;
    uint64_t x;
    if (mode >= 10) {
        x = insert_zero(bits64_at(d, 65), 3);
    } else {
        x = insert_zero(bits64_at(d, 82) & ((1ull << 46) - 1ull), 2);
        uint32_t a1 = __ldg(&kDecAnchors[part]) >> 4;
        x = insert_zero(x, a1 * 3 + 2);
        map = __ldg(&kDecPartitionMap[part]);
    }
#pragma unroll
    for (int k = 0; k < 16; k++) {
        int w;
        if (mode >= 10) w = (int)bptc_weight<4>((uint32_t)(x >> (4 * k)) & 15u);
        else w = (int)bptc_weight<3>((uint32_t)(x >> (3 * k)) & 7u);
        bool e = ((map >> (2 * k)) & 1u) != 0;
        int r0 = e ? r[2] : r[0], r1 = e ? r[3] : r[1];
        int g0 = e ? g[2] : g[0], g1 = e ? g[3] : g[1];
        int b0 = e ? b[2] : b[0], b1 = e ? b[3] : b[1];
        out[k * 3 + 0] = (uint16_t)((interp(r0, r1, w) * 31) >> 6);
        out[k * 3 + 1] = (uint16_t)((interp(g0, g1, w) * 31) >> 6);
        out[k * 3 + 2] = (uint16_t)((interp(b0, b1, w) * 31) >> 6);
    }
}

// f16 (non-negative, finite: the unsigned decoder never produces more than
// 0x7BFF) -> sRGB u8, the reference's linear_to_srgb (decode.rs:151-159)
// evaluated on the host for every such bit pattern.
__device__ uint8_t g_half_to_srgb[0x7C00];

__global__ void __launch_bounds__(128) bc6h_decode_kernel(const uint8_t* __restrict__ blocks, uint32_t bw, uint32_t bh,
                                                          void* __restrict__ out, size_t pitch, int fmt, bool aligned) {
    uint32_t n = bw * bh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t by = i / bw, bx = i - by * bw;
        const uint8_t* b = blocks + (size_t)i * 16;
        uint64_t lo = 0, hi = 0;
        if (aligned) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(b));
            lo = (uint64_t)v.x | ((uint64_t)v.y << 32);
            hi = (uint64_t)v.z | ((uint64_t)v.w << 32);
        } else {
            for (int j = 0; j < 8; j++) lo |= (uint64_t)b[j] << (8 * j);
            for (int j = 0; j < 8; j++) hi |= (uint64_t)b[8 + j] << (8 * j);
        }
        uint16_t h[48];
        decode_bc6h_block_u(lo, hi, h);
#pragma unroll
        for (int y = 0; y < 4; y++) {
            size_t row = (size_t)(by * 4 + y) * pitch + (size_t)bx * 16;
            if (fmt == 0) {
                uint8_t* o = reinterpret_cast<uint8_t*>(out) + row;
                uint32_t px[4];
#pragma unroll
                for (int x = 0; x < 4; x++) {
                    px[x] = 0;
#pragma unroll
                    for (int c = 0; c < 3; c++)
                        px[x] |= (uint32_t)__ldg(&g_half_to_srgb[min((int)h[(y * 4 + x) * 3 + c], 0x7BFF)]) << (8 * c);
                }
                if (aligned) {
                    *reinterpret_cast<uint4*>(o) = make_uint4(px[0], px[1], px[2], px[3]);
                } else {
                    for (int j = 0; j < 16; j++) o[j] = (uint8_t)(px[j >> 2] >> (8 * (j & 3)));
                }
            } else if (fmt == 1) {
                uint16_t* o = reinterpret_cast<uint16_t*>(out) + row;
                if (aligned) {
                    uint32_t w[6];
#pragma unroll
                    for (int j = 0; j < 6; j++) w[j] = (uint32_t)h[y * 12 + 2 * j] | ((uint32_t)h[y * 12 + 2 * j + 1] << 16);
                    uint2* o2 = reinterpret_cast<uint2*>(o);
                    o2[0] = make_uint2(w[0], w[1]);
                    o2[1] = make_uint2(w[2], w[3]);
                    o2[2] = make_uint2(w[4], w[5]);
                } else {
                    for (int j = 0; j < 12; j++) o[j] = h[y * 12 + j];
                }
            } else {
                float* o = reinterpret_cast<float*>(out) + row;
                float f[12];
#pragma unroll
                for (int j = 0; j < 12; j++) f[j] = __half2float(__ushort_as_half(h[y * 12 + j]));
                if (aligned) {
                    float4* o4 = reinterpret_cast<float4*>(o);
                    o4[0] = make_float4(f[0], f[1], f[2], f[3]);
                    o4[1] = make_float4(f[4], f[5], f[6], f[7]);
                    o4[2] = make_float4(f[8], f[9], f[10], f[11]);
                } else {
                    for (int j = 0; j < 12; j++) o[j] = f[j];
                }
            }
        }
    }
}

static int grid_for(uint32_t n) {
    uint32_t g = (n + 127) / 128;
    return (int)(g > 148u * 64u ? 148u * 64u : (g == 0 ? 1 : g));
}

void launch_bc7_decode(const uint8_t* blocks, uint32_t bw, uint32_t bh, uint8_t* out, size_t pitch, cudaStream_t s) {
    if (bw == 0 || bh == 0) return;
    bool aligned = ((uintptr_t)blocks % 16 == 0) && ((uintptr_t)out % 16 == 0) && (pitch % 16 == 0);
    bc7_decode_kernel<<<grid_for(bw * bh), 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned);
}

void launch_bc6h_decode(const uint8_t* blocks, uint32_t bw, uint32_t bh, void* out, size_t pitch, int out_format,
                        cudaStream_t s) {
    if (bw == 0 || bh == 0) return;
    // aligned: 16-byte block loads, and row stores of 16 B (RGBA8), 8 B
    // (RGBA16F, rows start at 32-byte multiples) or 16 B (RGBA32F)
    size_t esize = out_format == 0 ? 1 : (out_format == 1 ? 2 : 4);
    bool aligned = ((uintptr_t)blocks % 16 == 0) && ((uintptr_t)out % 16 == 0) && ((pitch * esize) % 16 == 0);
    bc6h_decode_kernel<<<grid_for(bw * bh), 128, 0, s>>>(blocks, bw, bh, out, pitch, out_format, aligned);
}

}  // namespace bcn

namespace bcn {
cudaError_t set_half_to_srgb_table(const uint8_t* host) {
    return cudaMemcpyToSymbol(g_half_to_srgb, host, sizeof(g_half_to_srgb));
}
}  // namespace bcn
