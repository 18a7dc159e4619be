// BC1-BC5 encode and decode kernels for sm_100a.
//
// Bandwidth-bound paths: one thread owns one 4x4 block. A warp covers 32
// neighbouring blocks of a block row, so each of the 4 source rows is read as
// one contiguous 512-byte span of 128-bit loads, and the 8/16-byte outputs of
// the warp land in one contiguous span as 64/128-bit stores. The per-block
// arithmetic follows the reference encoder (src/encode/bc1_to_5.rs) operation
// for operation so the output is bit-identical; see bc_common.cuh for the
// float rules.
#include <cuda_runtime.h>

#include "bc_common.cuh"
#include "bc_kernels.h"
#include "bc1_block.cuh"
#include "bc_check.cuh"

namespace bcn {

// ---- BC1 colour (bc1_to_5.rs:157-429) ---------------------------------------

struct Px16 {
    float r[16], g[16], b[16], a[16];
};

// bc1_to_5.rs:280-321: 2-bit index per pixel by projection onto the
// quantised endpoint direction.
BCN_DEV uint32_t fast_quant(const Px16& px, int p0, int p1) {
    float c0[3], c1[3], dir[3];
    dec_rgb565(c0, p0);
    dec_rgb565(c1, p1);
    for (int p = 0; p < 3; p++) dir[p] = c1[p] - c0[p];
    float sq_norm = 0.0f;
    for (int p = 0; p < 3; p++) sq_norm += dir[p] * dir[p];
    float rsq_norm = __frcp_rn(sq_norm);  // the IEEE 1 / x
    for (int p = 0; p < 3; p++) dir[p] *= rsq_norm * 3.0f;
    float bias = 0.5f;
    for (int p = 0; p < 3; p++) bias -= c0[p] * dir[p];
    uint32_t bits = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        // The reference starts the sum at 0.0; starting at the first term
        // differs only in the sign of a zero sum, which neither the
        // following additions of non-zero terms nor the truncation below
        // can see.
        float dot = px.r[k] * dir[0];
        dot += px.g[k] * dir[1];
        dot += px.b[k] * dir[2];
        int q = clampi((int)(dot + bias), 0, 3);
        bits += (uint32_t)q << (2 * k);
    }
    return bits;
}

// bc1_to_5.rs:323-374: least-squares endpoints for fixed indices.
BCN_DEV void bc1_refine(const Px16& px, int pe[2], uint32_t bits, const float dc[3]) {
    float c0[3], c1[3];
    if ((bits ^ (bits * 4u)) < 4) {
        for (int p = 0; p < 3; p++) c0[p] = c1[p] = dc[p];
    } else {
        // integer products and sums below 2^24: the fused multiply-adds give
        // the reference's multiply-then-add results exactly
        float atb1[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int k = 0; k < 16; k++) {
            float x = (float)(3u - ((bits >> (2 * k)) & 3u));
            atb1[0] = fmaf(x, px.r[k], atb1[0]);
            atb1[1] = fmaf(x, px.g[k], atb1[1]);
            atb1[2] = fmaf(x, px.b[k], atb1[2]);
        }
        // sum q and sum q^2 over the 16 two-bit indices from the counts of
        // each index value (exact integers, the reference's float sums)
        const uint32_t lo = bits & 0x55555555u, hi = (bits >> 1) & 0x55555555u;
        const int n3 = __popc(lo & hi), n1 = __popc(lo) - n3, n2 = __popc(hi) - n3;
        const float sum_q = (float)(n1 + 2 * n2 + 3 * n3), sum_qq = (float)(n1 + 4 * n2 + 9 * n3);
        float sum[3], atb2[3];
        for (int p = 0; p < 3; p++) {
            sum[p] = dc[p] * 16.0f;
            atb2[p] = 3.0f * sum[p] - atb1[p];
        }
        float cxx = 144.0f - 6.0f * sum_q + sum_qq;  // 16*9 - (2*3)*sum_q + sum_qq
        float cyy = sum_qq;
        float cxy = 3.0f * sum_q - sum_qq;
        float scale = 3.0f * __frcp_rn(cxx * cyy - cxy * cxy);
        for (int p = 0; p < 3; p++) {
            c0[p] = clampf_r((atb1[p] * cyy - atb2[p] * cxy) * scale, 0.0f, 255.0f);
            c1[p] = clampf_r((atb2[p] * cxx - atb1[p] * cxy) * scale, 0.0f, 255.0f);
        }
    }
    pe[0] = enc_rgb565(c0[0], c0[1], c0[2]);
    pe[1] = enc_rgb565(c1[0], c1[1], c1[2]);
}

BCN_DEV uint32_t fix_qbits(uint32_t q) {
    uint32_t q0 = q & 0x55555555u, q1 = q & 0xAAAAAAAAu;
    return (q1 >> 1) + (q1 ^ (q0 << 1));
}

// bc1_to_5.rs:386-429
BCN_DEV void bc1_core(const Px16& px, uint32_t& w0, uint32_t& w1) {
    float dc[3];
    {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; k++) acc += px.r[k];
        dc[0] = acc / 16.0f;
        acc = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; k++) acc += px.g[k];
        dc[1] = acc / 16.0f;
        acc = 0.0f;
#pragma unroll
        for (int k = 0; k < 16; k++) acc += px.b[k];
        dc[2] = acc / 16.0f;
    }
    // x = pixel - mean is n / 16 with |n| < 2^12 (the mean is a sum of 16
    // bytes over 16), so every product x * y is n * m / 256 with
    // |n * m| < 2^24: exact in f32. A fused multiply-add of an exact product
    // rounds the sum once, exactly as the reference's multiply then add.
    float cv[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float x0 = px.r[k] - dc[0], x1 = px.g[k] - dc[1], x2 = px.b[k] - dc[2];
        cv[0] = fmaf(x0, x0, cv[0]);
        cv[1] = fmaf(x0, x1, cv[1]);
        cv[2] = fmaf(x0, x2, cv[2]);
        cv[3] = fmaf(x1, x1, cv[3]);
        cv[4] = fmaf(x1, x2, cv[4]);
        cv[5] = fmaf(x2, x2, cv[5]);
    }
    const float eps = 1.1920929e-7f;  // f32::EPSILON
    cv[0] += eps;
    cv[3] += eps;
    cv[5] += eps;
    // compute_axis3, 4 power iterations, renormalised after the odd ones.
    float a[3] = {1.0f, 1.0f, 1.0f}, ax[3];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        ax[0] = cv[0] * a[0] + cv[1] * a[1] + cv[2] * a[2];
        ax[1] = cv[1] * a[0] + cv[3] * a[1] + cv[4] * a[2];
        ax[2] = cv[2] * a[0] + cv[4] * a[1] + cv[5] * a[2];
        a[0] = ax[0];
        a[1] = ax[1];
        a[2] = ax[2];
        if (i % 2 == 1) {
            float n = 0.0f;
            n += ax[0] * ax[0];
            n += ax[1] * ax[1];
            n += ax[2] * ax[2];
            float rn = __frcp_rn(sqrtf(n));
            a[0] *= rn;
            a[1] *= rn;
            a[2] *= rn;
        }
    }
    // pick_endpoints
    float min_dot = 65536.0f, max_dot = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        // Without the reference's leading 0.0 the sum can differ only in
        // the sign of a zero; a -0 extreme gives the same endpoint as +0
        // (the range test and dc + 0 * axis cannot tell them apart).
        float dot = (px.r[k] - dc[0]) * a[0];
        dot += (px.g[k] - dc[1]) * a[1];
        dot += (px.b[k] - dc[2]) * a[2];
        min_dot = fminf(min_dot, dot);
        max_dot = fmaxf(max_dot, dot);
    }
    if (max_dot - min_dot < 1.0f) {
        min_dot -= 0.5f;
        max_dot += 0.5f;
    }
    float norm_sq = 0.0f;
    norm_sq += a[0] * a[0];
    norm_sq += a[1] * a[1];
    norm_sq += a[2] * a[2];
    float rnorm_sq = __frcp_rn(norm_sq);
    float c0[3], c1[3];
    for (int p = 0; p < 3; p++) {
        c0[p] = clampf_r(dc[p] + min_dot * rnorm_sq * a[p], 0.0f, 255.0f);
        c1[p] = clampf_r(dc[p] + max_dot * rnorm_sq * a[p], 0.0f, 255.0f);
    }
    int p[2];
    p[0] = enc_rgb565(c0[0], c0[1], c0[2]);
    p[1] = enc_rgb565(c1[0], c1[1], c1[2]);
    if (p[0] < p[1]) {
        int t = p[0];
        p[0] = p[1];
        p[1] = t;
    }
    uint32_t q = fast_quant(px, p[0], p[1]);
    // one refinement round (refine_iterations = 1)
    bc1_refine(px, p, q, dc);
    if (p[0] < p[1]) {
        int t = p[0];
        p[0] = p[1];
        p[1] = t;
    }
    w0 = ((uint32_t)p[1] << 16) | (uint32_t)p[0];
    w1 = fix_qbits(fast_quant(px, p[0], p[1]));
}

// bc1_to_5.rs:431-472: 8-level alpha / single channel block.
BCN_DEV void bc3_alpha(const float* v, uint32_t& w0, uint32_t& w1) {
    float e0 = 255.0f, e1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        e0 = fminf(e0, v[k]);
        e1 = fmaxf(e1, v[k]);
    }
    if (e0 == e1) e1 = e0 + 0.1f;
    float scale = 7.0f / (e1 - e0);
    uint32_t qb0 = 0, qb1 = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float proj = (v[k] - e0) * scale + 0.5f;
        int q = clampi((int)proj, 0, 7);
        q = 7 - q;
        if (q > 0) q += 1;
        if (q == 8) q = 1;
        if (k < 8) qb0 |= (uint32_t)q << (k * 3);
        else qb1 |= (uint32_t)q << ((k - 8) * 3);
    }
    uint32_t a0 = min((uint32_t)e0, 255u), a1 = min((uint32_t)e1, 255u);
    w0 = (a0 << 8) | a1 | (qb0 << 16);
    w1 = (qb0 >> 16) | (qb1 << 8);
}

// ---- loads / stores -------------------------------------------------------

// Loads the 4x4 RGBA8 block at (bx, by). ALIGNED: row base + 16*bx is
// 16-byte aligned, so each row is one 128-bit load.
template <bool ALIGNED>
BCN_DEV void load_rgba8(const uint8_t* __restrict__ src, size_t stride, uint32_t bx, uint32_t by, Px16& px) {
#pragma unroll
    for (int y = 0; y < 4; y++) {
        const uint8_t* row = src + (size_t)(by * 4 + y) * stride + (size_t)bx * 16;
        uint32_t w[4];
        if (ALIGNED) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(row));
            w[0] = v.x;
            w[1] = v.y;
            w[2] = v.z;
            w[3] = v.w;
        } else {
            for (int x = 0; x < 4; x++)
                w[x] = (uint32_t)row[4 * x] | ((uint32_t)row[4 * x + 1] << 8) | ((uint32_t)row[4 * x + 2] << 16) |
                       ((uint32_t)row[4 * x + 3] << 24);
        }
#pragma unroll
        for (int x = 0; x < 4; x++) {
            px.r[y * 4 + x] = byte_to_float(w[x], 0);
            px.g[y * 4 + x] = byte_to_float(w[x], 1);
            px.b[y * 4 + x] = byte_to_float(w[x], 2);
            px.a[y * 4 + x] = byte_to_float(w[x], 3);
        }
    }
}

template <bool ALIGNED>
BCN_DEV void store_block(uint8_t* dst, const uint32_t* w, int words) {
    if (ALIGNED) {
        if (words == 2) *reinterpret_cast<uint2*>(dst) = make_uint2(w[0], w[1]);
        else *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
    } else {
        for (int i = 0; i < words; i++) reinterpret_cast<uint32_t*>(dst)[i] = w[i];
    }
}

// ---- encode kernel -----------------------------------------------------------

BCN_DEV void encode_bc15_block(int variant, const Px16& px, uint32_t w[4]) {
    switch (variant) {
        case BC_BC1:
            bc1_core(px, w[0], w[1]);
            break;
        case BC_BC2: {
            // bc1_to_5.rs:84-115
            uint32_t a0 = 0, a1 = 0;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                float alpha = px.a[k] / 255.0f;
                uint32_t a4 = (uint32_t)(alpha * 15.0f);
                if (k < 8) a0 |= a4 << (4 * k);
                else a1 |= a4 << (4 * (k - 8));
            }
            w[0] = a0;
            w[1] = a1;
            bc1_core(px, w[2], w[3]);
            break;
        }
        case BC_BC3:
            bc3_alpha(px.a, w[0], w[1]);
            bc1_core(px, w[2], w[3]);
            break;
        case BC_BC4:
            bc3_alpha(px.r, w[0], w[1]);
            break;
        default:  // BC5
            bc3_alpha(px.r, w[0], w[1]);
            bc3_alpha(px.g, w[2], w[3]);
            break;
    }
}

// Minimum resident CTAs of 128 threads per SM asked of the register
// allocator for the encode kernel: 5 caps BC1 at 96 registers (a 144-byte
// spill), 1% faster at 8192x8192 than 4 CTAs at 127 registers; 6 (80
// registers) is 11% slower.
#ifndef BCN_BC15_MINB
#define BCN_BC15_MINB 5
#endif
template <int VARIANT, bool ALIGNED_SRC, bool ALIGNED_DST>
__global__ void __launch_bounds__(128, BCN_BC15_MINB) bc15_encode_kernel(const uint8_t* __restrict__ src, size_t stride,
                                                           uint32_t bw, uint32_t bh, uint8_t* __restrict__ dst) {
    uint32_t n = bw * bh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t by = i / bw, bx = i - by * bw;
        if (!BCN_GUARD(by, bh, CHECK_BC15_LOAD) || !BCN_GUARD(bx, bw, CHECK_BC15_LOAD)) continue;
        Px16 px;
        load_rgba8<ALIGNED_SRC>(src, stride, bx, by, px);
        uint32_t w[4];
        encode_bc15_block(VARIANT, px, w);
        constexpr int words = (VARIANT == BC_BC1 || VARIANT == BC_BC4) ? 2 : 4;
        if (BCN_GUARD(i, n, CHECK_BC15_STORE)) store_block<ALIGNED_DST>(dst + (size_t)i * (words * 4), w, words);
    }
}

// ---- BC1-BC5 decode (src/decode/block.rs:124-258, src/decode.rs:60-148) ------

// Decodes one BC1-BC5 block to 16 RGBA8 pixels, with the reference's RGBA8
// conventions (BC4 -> (R,0,0,0), BC5 -> (R,G,0,0)).
BCN_DEV void decode_bc15_rgba8(int variant, const uint32_t* w, uint32_t out[16]) {
    if (variant == BC_BC1) {
        decode_color(w[0], w[1], false, out);
    } else if (variant == BC_BC2) {
        decode_color(w[2], w[3], true, out);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            uint32_t a = ((k < 8 ? w[0] : w[1]) >> (4 * (k & 7))) & 15;
            out[k] = (out[k] & 0x00FFFFFFu) | ((a * 17) << 24);
        }
    } else if (variant == BC_BC3) {
        decode_color(w[2], w[3], true, out);
        uint32_t a[16];
        decode_smooth(w[0], w[1], a);
#pragma unroll
        for (int k = 0; k < 16; k++) out[k] = (out[k] & 0x00FFFFFFu) | (a[k] << 24);
    } else if (variant == BC_BC4) {
        decode_smooth(w[0], w[1], out);
    } else {
        uint32_t r[16], g[16];
        decode_smooth(w[0], w[1], r);
        decode_smooth(w[2], w[3], g);
#pragma unroll
        for (int k = 0; k < 16; k++) out[k] = r[k] | (g[k] << 8);
    }
}

// 12 resident CTAs per SM (40 registers, no spill) keep more block reads in
// flight than the compiler's 48 registers: BC1 85% instead of 82% of HBM at
// 8192x8192, BC3 76% instead of 74%, BC5 81% instead of 79%.
template <int VARIANT>
__global__ void __launch_bounds__(128, 12) bc15_decode_kernel(const uint8_t* __restrict__ blocks, uint32_t bw, uint32_t bh,
                                                           uint8_t* __restrict__ out, size_t pitch, bool aligned) {
    constexpr int words = (VARIANT == BC_BC1 || VARIANT == BC_BC4) ? 2 : 4;
    uint32_t n = bw * bh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t by = i / bw, bx = i - by * bw;
        uint32_t w[4] = {0, 0, 0, 0};
        const uint8_t* b = blocks + (size_t)i * words * 4;
        if (aligned) {
            if (words == 2) {
                uint2 v = __ldg(reinterpret_cast<const uint2*>(b));
                w[0] = v.x;
                w[1] = v.y;
            } else {
                uint4 v = __ldg(reinterpret_cast<const uint4*>(b));
                w[0] = v.x;
                w[1] = v.y;
                w[2] = v.z;
                w[3] = v.w;
            }
        } else {
            for (int j = 0; j < words * 4; j++) w[j >> 2] |= (uint32_t)b[j] << (8 * (j & 3));
        }
        uint32_t px[16];
        decode_bc15_rgba8(VARIANT, w, px);
        if (!BCN_GUARD(by, bh, CHECK_DECODE_STORE) || !BCN_GUARD(bx, bw, CHECK_DECODE_STORE)) continue;
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

// ---- batched: persistent work-queue kernel ---------------------------------------
//
// One launch encodes the tiles (32 blocks) of many BC1-BC5 regions of mixed
// variants. CTAs stay resident and claim work from a global counter: each
// claim hands NWARP*tiles_per_claim consecutive tiles to the CTA, warp w
// takes tiles base + i*NWARP + w. The loop ends when a claim starts past the
// last tile, so it runs at most ntiles / (NWARP*tiles_per_claim) + 1 times
// per CTA (no waiting on other CTAs).
template <int THREADS>
__global__ void __launch_bounds__(THREADS) bc15_batch_kernel(const TaskDesc* __restrict__ tasks,
                                                              const uint32_t* __restrict__ tile_task, uint32_t ntiles,
                                                              uint32_t* counter, int tiles_per_claim) {
    constexpr int NWARP = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t base_s;
    for (;;) {
        if (threadIdx.x == 0) base_s = atomicAdd(counter, (uint32_t)(NWARP * tiles_per_claim));
        __syncthreads();
        const uint32_t base = base_s;
        __syncthreads();
        if (base >= ntiles) break;
        for (int i = 0; i < tiles_per_claim; i++) {
            const uint32_t tile = base + (uint32_t)(i * NWARP + warp);
            if (tile >= ntiles) break;
            const TaskDesc d = tasks[tile_task[tile]];
            const uint32_t lb = (tile - d.tile_base) * 32 + lane;
            if (lb >= d.bw * d.bh) continue;
            const uint32_t by = lb / d.bw, bx = lb - by * d.bw;
            Px16 px;
            if (d.aligned) load_rgba8<true>(d.src, d.stride, bx, by, px);
            else load_rgba8<false>(d.src, d.stride, bx, by, px);
            uint32_t w[4];
            encode_bc15_block((int)d.variant, px, w);
            const int words = (d.variant == BC_BC1 || d.variant == BC_BC4) ? 2 : 4;
            uint8_t* o = d.dst + (size_t)lb * (words * 4);
            if (((uintptr_t)o & (words * 4 - 1)) == 0) {
                if (words == 2) *reinterpret_cast<uint2*>(o) = make_uint2(w[0], w[1]);
                else *reinterpret_cast<uint4*>(o) = make_uint4(w[0], w[1], w[2], w[3]);
            } else {
                for (int j = 0; j < words; j++) reinterpret_cast<uint32_t*>(o)[j] = w[j];
            }
        }
    }
}

cudaError_t launch_bc15_batch(const TaskDesc* tasks_dev, const uint32_t* tile_task_dev, uint32_t ntiles,
                              uint32_t* counter_dev, int threads, int ctas, int tiles_per_claim, cudaStream_t s) {
    if (ntiles == 0) return cudaSuccess;
    if (tiles_per_claim < 1) tiles_per_claim = 1;
    if (threads == 256) bc15_batch_kernel<256><<<ctas, 256, 0, s>>>(tasks_dev, tile_task_dev, ntiles, counter_dev,
                                                                   tiles_per_claim);
    else bc15_batch_kernel<128><<<ctas, 128, 0, s>>>(tasks_dev, tile_task_dev, ntiles, counter_dev, tiles_per_claim);
    return cudaGetLastError();
}

// ---- launchers ------------------------------------------------------------------

static int grid_for(uint32_t n, int threads) {
    // Enough CTAs to fill the machine several times over; the kernels loop
    // grid-stride over any remainder.
    uint32_t g = (n + threads - 1) / threads;
    return (int)(g > 148u * 64u ? 148u * 64u : (g == 0 ? 1 : g));
}

template <int V>
static void launch_encode(const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst, bool asrc,
                          bool adst, cudaStream_t s) {
    int g = grid_for(bw * bh, 128);
    if (asrc && adst) bc15_encode_kernel<V, true, true><<<g, 128, 0, s>>>(src, stride, bw, bh, dst);
    else if (asrc) bc15_encode_kernel<V, true, false><<<g, 128, 0, s>>>(src, stride, bw, bh, dst);
    else if (adst) bc15_encode_kernel<V, false, true><<<g, 128, 0, s>>>(src, stride, bw, bh, dst);
    else bc15_encode_kernel<V, false, false><<<g, 128, 0, s>>>(src, stride, bw, bh, dst);
}

void launch_bc15_encode(int variant, const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst,
                        cudaStream_t s) {
    if (bw == 0 || bh == 0) return;
    bool asrc = ((uintptr_t)src % 16 == 0) && (stride % 16 == 0);
    size_t bb = (variant == BC_BC1 || variant == BC_BC4) ? 8 : 16;
    bool adst = ((uintptr_t)dst % bb) == 0;
    switch (variant) {
        case BC_BC1: launch_encode<BC_BC1>(src, stride, bw, bh, dst, asrc, adst, s); break;
        case BC_BC2: launch_encode<BC_BC2>(src, stride, bw, bh, dst, asrc, adst, s); break;
        case BC_BC3: launch_encode<BC_BC3>(src, stride, bw, bh, dst, asrc, adst, s); break;
        case BC_BC4: launch_encode<BC_BC4>(src, stride, bw, bh, dst, asrc, adst, s); break;
        default: launch_encode<BC_BC5>(src, stride, bw, bh, dst, asrc, adst, s); break;
    }
}

void launch_bc15_decode(int variant, const uint8_t* blocks, uint32_t bw, uint32_t bh, uint8_t* out, size_t pitch,
                        cudaStream_t s) {
    if (bw == 0 || bh == 0) return;
    size_t bb = (variant == BC_BC1 || variant == BC_BC4) ? 8 : 16;
    bool aligned = ((uintptr_t)blocks % bb == 0) && ((uintptr_t)out % 16 == 0) && (pitch % 16 == 0);
    int g = grid_for(bw * bh, 128);
    switch (variant) {
        case BC_BC1: bc15_decode_kernel<BC_BC1><<<g, 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned); break;
        case BC_BC2: bc15_decode_kernel<BC_BC2><<<g, 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned); break;
        case BC_BC3: bc15_decode_kernel<BC_BC3><<<g, 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned); break;
        case BC_BC4: bc15_decode_kernel<BC_BC4><<<g, 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned); break;
        default: bc15_decode_kernel<BC_BC5><<<g, 128, 0, s>>>(blocks, bw, bh, out, pitch, aligned); break;
    }
}

}  // namespace bcn

namespace bcn {
cudaError_t check_take_bc15(unsigned long long out[3]) { return check_record_take(out); }
}  // namespace bcn
