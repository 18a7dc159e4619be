// Differentiable BC1 / BC7 decode and gradient endpoint refinement (no
// reference counterpart).
//
// Standalone kernels (one thread per block) expose the pieces a training
// loop needs: block parsing into fixed metadata + continuous endpoints, the
// relaxed decode, and its adjoint. The refinement kernel fuses the whole
// loop for one block per thread: relaxed decode -> MSE gradient -> adjoint ->
// Adam step, then re-quantisation of the endpoints with the encoder's own
// quantisers (src/encode/bc7.rs:97-276, src/encode/bc1_to_5.rs:268-278),
// coding with the block's fixed mode, partition, rotation, index selector and
// indices (bc7_code_*, bc7.rs:381-515), a bit-exact decode of the coded
// block and its exact squared error against the source. The best coded block
// replaces the input only if that error is strictly lower, so no block gets
// worse.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>

#include "../../include/bc_capi.h"
#include "bc1_block.cuh"
#include "bc7_device.cuh"
#include "bc_kernels.h"
#include "bc_relaxed.cuh"
#include "bptc_decode.cuh"

namespace bcn {
namespace {

constexpr int kThreads = 128;

BCN_DEV uint4 load_block16(const uint8_t* p, bool aligned) {
    if (aligned) return __ldg(reinterpret_cast<const uint4*>(p));
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; i++)
        w[i] = (uint32_t)p[4 * i] | (uint32_t)p[4 * i + 1] << 8 | (uint32_t)p[4 * i + 2] << 16 |
               (uint32_t)p[4 * i + 3] << 24;
    return make_uint4(w[0], w[1], w[2], w[3]);
}

BCN_DEV void store_words(uint8_t* p, const uint32_t* w, int words, bool aligned) {
    if (aligned) {
        if (words == 4) *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
        else *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
        return;
    }
    for (int i = 0; i < 4 * words; i++) p[i] = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
}

// The 16 source pixels of block (bx, by), RGBA8 packed, row-major.
BCN_DEV void load_src(const uint8_t* src, size_t stride, uint32_t bx, uint32_t by, bool aligned, uint32_t px[16]) {
#pragma unroll
    for (int y = 0; y < 4; y++) {
        const uint8_t* row = src + (size_t)(by * 4 + y) * stride + (size_t)bx * 16;
        if (aligned) {
            uint4 v = __ldg(reinterpret_cast<const uint4*>(row));
            px[4 * y] = v.x;
            px[4 * y + 1] = v.y;
            px[4 * y + 2] = v.z;
            px[4 * y + 3] = v.w;
        } else {
#pragma unroll
            for (int x = 0; x < 4; x++)
                px[4 * y + x] = (uint32_t)row[4 * x] | (uint32_t)row[4 * x + 1] << 8 |
                                (uint32_t)row[4 * x + 2] << 16 | (uint32_t)row[4 * x + 3] << 24;
        }
    }
}

BCN_DEV float chan(uint32_t px, int c) { return (float)((px >> (8 * c)) & 0xFF); }

// Exact squared error of decoded texels against the source over the first
// `channels` channels.
BCN_DEV uint32_t exact_err(const uint32_t dec[16], const uint32_t src[16], uint32_t channels) {
    uint32_t err = 0;
#pragma unroll
    for (int k = 0; k < 16; k++)
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (c >= (int)channels) continue;
            int d = (int)((dec[k] >> (8 * c)) & 0xFF) - (int)((src[k] >> (8 * c)) & 0xFF);
            err += (uint32_t)(d * d);
        }
    return err;
}

// Squared error of one texel over the first `channels` channels: per-byte
// absolute differences, then the dot product of those bytes with themselves.
BCN_DEV uint32_t texel_err(uint32_t a, uint32_t b, uint32_t channels) {
    uint32_t d = __vabsdiffu4(a, b);
    if (channels == 3) d &= 0x00FFFFFFu;
    return (uint32_t)__dp4a(d, d, 0u);
}

// Exact error of a coded block, decoded texel by texel (no texel array).
BCN_DEV uint32_t bc7_exact_err(uint4 blk, const uint32_t src[16], uint32_t channels) {
    uint32_t err = 0;
    decode_bc7_each((uint64_t)blk.x | ((uint64_t)blk.y << 32), (uint64_t)blk.z | ((uint64_t)blk.w << 32),
                    [&](int k, uint32_t px) { err += texel_err(px, src[k], channels); });
    return err;
}

BCN_DEV uint32_t bc1_exact_err(uint32_t w0, uint32_t w1, const uint32_t src[16]) {
    uint32_t dec[16];
    decode_color(w0, w1, false, dec);
    return exact_err(dec, src, 3);
}

// Re-quantises continuous endpoints with the mode's quantiser and codes them
// with the block's fixed indices (bc7.rs:97-276 and 381-515).
BCN_DEV uint4 bc7_requant_code(const uint32_t meta[6], const float theta[24], uint32_t channels) {
    using namespace bc7;
    uint32_t mode = meta[0] & 15, partition = (meta[0] >> 4) & 63, rotation = (meta[0] >> 10) & 3;
    int isb = (int)((meta[0] >> 12) & 1);
    float ep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) ep[i] = clampf_r(theta[i], 0.0f, 255.0f);
    int qep[24];
#pragma unroll
    for (int i = 0; i < 24; i++) qep[i] = 0;
    switch (mode) {
        case 0:
            quant_dequant_part<0>(qep, ep);
            return code_mode01237<0>(qep, meta[1], meta[2], 64 + (int)partition);
        case 1:
            quant_dequant_part<1>(qep, ep);
            return code_mode01237<1>(qep, meta[1], meta[2], (int)partition);
        case 2:
            quant_dequant_part<2>(qep, ep);
            return code_mode01237<2>(qep, meta[1], meta[2], 64 + (int)partition);
        case 3:
            quant_dequant_part<3>(qep, ep);
            return code_mode01237<3>(qep, meta[1], meta[2], (int)partition);
        case 7:
            quant_dequant_part<7>(qep, ep);
            return code_mode01237<7>(qep, meta[1], meta[2], (int)partition);
        case 6:
            if (channels == 4) quant0367_pair<7, 4, 4, false>(qep, ep);
            else quant0367_pair<7, 3, 4, false>(qep, ep);
            return code_mode6(qep, meta[1], meta[2]);
        default: {  // 4, 5
            int aqep[2];
            float aep[2] = {ep[3], ep[7]};
            int rot = (int)((rotation + 3) & 3);  // the stored field is the encoder's rotation + 1
            if (mode == 4) {
                quant245<5, 8>(qep, ep);
                channel_quant_dequant(aqep, aep, 6);
                return code_mode45<4>(qep, meta[1], meta[2], aqep, meta[3], meta[4], rot, isb);
            }
            quant245<7, 8>(qep, ep);
            channel_quant_dequant(aqep, aep, 8);
            return code_mode45<5>(qep, meta[1], meta[2], aqep, meta[3], meta[4], rot, 0);
        }
    }
}

// BC1 re-quantisation with enc_rgb565 and the fixed indices. A four-colour
// block whose endpoints come out in the wrong order is swapped with indices
// 0<->1, 2<->3 (the encoder's ordering, bc1_to_5.rs:406-409); equal endpoints
// would decode in the three-colour mode, so every index then points at
// endpoint 0. A three-colour block keeps colour0 <= colour1.
BCN_DEV void bc1_requant_code(const uint32_t meta[2], const float theta[6], uint32_t& w0, uint32_t& w1) {
    int p0 = enc_rgb565(clampf_r(theta[0], 0.0f, 255.0f), clampf_r(theta[1], 0.0f, 255.0f),
                        clampf_r(theta[2], 0.0f, 255.0f));
    int p1 = enc_rgb565(clampf_r(theta[3], 0.0f, 255.0f), clampf_r(theta[4], 0.0f, 255.0f),
                        clampf_r(theta[5], 0.0f, 255.0f));
    uint32_t idx = meta[1];
    bool four = (meta[0] & 0xFFFF) > (meta[0] >> 16);
    if (four) {
        if (p0 < p1) {
            int t = p0;
            p0 = p1;
            p1 = t;
            idx ^= 0x55555555u;
        } else if (p0 == p1) {
            idx = 0;
        }
    } else if (p0 > p1) {
        int t = p0;
        p0 = p1;
        p1 = t;
        idx ^= ~(idx >> 1) & 0x55555555u;
    }
    w0 = (uint32_t)p0 | (uint32_t)p1 << 16;
    w1 = idx;
}

BCN_DEV void add_stats(unsigned long long* stats, uint32_t active, uint32_t improved, uint32_t before,
                       uint32_t after) {
    if (!stats) return;
    // Per-block errors are below 2^22, so a warp's sums fit in 32 bits.
    uint32_t a = __reduce_add_sync(0xFFFFFFFFu, active);
    uint32_t i = __reduce_add_sync(0xFFFFFFFFu, improved);
    uint32_t b = __reduce_add_sync(0xFFFFFFFFu, before);
    uint32_t f = __reduce_add_sync(0xFFFFFFFFu, after);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(stats + 0, (unsigned long long)a);
        atomicAdd(stats + 1, (unsigned long long)i);
        atomicAdd(stats + 2, (unsigned long long)b);
        atomicAdd(stats + 3, (unsigned long long)f);
    }
}

// ---- standalone kernels -------------------------------------------------------

__global__ void __launch_bounds__(kThreads) bc7_parse_kernel(const uint8_t* __restrict__ blocks, uint32_t n,
                                                             bool aligned, uint32_t* __restrict__ meta,
                                                             float* __restrict__ ep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 b = load_block16(blocks + (size_t)i * 16, aligned);
    uint32_t m[6];
    float e[24];
    relax::bc7_parse((uint64_t)b.x | ((uint64_t)b.y << 32), (uint64_t)b.z | ((uint64_t)b.w << 32), m, e);
    uint4* mo = reinterpret_cast<uint4*>(meta + (size_t)i * 8);
    mo[0] = make_uint4(m[0], m[1], m[2], m[3]);
    mo[1] = make_uint4(m[4], m[5], 0, 0);
    float4* eo = reinterpret_cast<float4*>(ep + (size_t)i * 24);
#pragma unroll
    for (int j = 0; j < 6; j++) eo[j] = make_float4(e[4 * j], e[4 * j + 1], e[4 * j + 2], e[4 * j + 3]);
}

BCN_DEV void load_bc7_state(const uint32_t* meta, const float* ep, uint32_t i, uint32_t m[6], float e[24]) {
    uint4 a = reinterpret_cast<const uint4*>(meta + (size_t)i * 8)[0];
    uint4 b = reinterpret_cast<const uint4*>(meta + (size_t)i * 8)[1];
    m[0] = a.x;
    m[1] = a.y;
    m[2] = a.z;
    m[3] = a.w;
    m[4] = b.x;
    m[5] = b.y;
    if (!ep) return;
    const float4* ei = reinterpret_cast<const float4*>(ep + (size_t)i * 24);
#pragma unroll
    for (int j = 0; j < 6; j++) {
        float4 v = ei[j];
        e[4 * j] = v.x;
        e[4 * j + 1] = v.y;
        e[4 * j + 2] = v.z;
        e[4 * j + 3] = v.w;
    }
}

// One thread per pixel: out[(i * 16 + k) * 4 + c].
__global__ void __launch_bounds__(kThreads) bc7_relaxed_kernel(const uint32_t* __restrict__ meta,
                                                               const float* __restrict__ ep, uint32_t n,
                                                               float* __restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n * 16) return;
    uint32_t i = (uint32_t)(t >> 4);
    int k = (int)(t & 15);
    uint32_t m[6];
    float e[24];
    load_bc7_state(meta, ep, i, m, e);
    float px[4];
    relax::bc7_relaxed_px(m, e, k, px);
    reinterpret_cast<float4*>(out)[t] = make_float4(px[0], px[1], px[2], px[3]);
}

__global__ void __launch_bounds__(kThreads) bc7_adjoint_kernel(const uint32_t* __restrict__ meta,
                                                               const float* __restrict__ g, uint32_t n,
                                                               float* __restrict__ gep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t m[6];
    load_bc7_state(meta, nullptr, i, m, nullptr);
    float ge[24];
#pragma unroll
    for (int j = 0; j < 24; j++) ge[j] = 0.0f;
    const float4* gi = reinterpret_cast<const float4*>(g) + (size_t)i * 16;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float4 v = gi[k];
        float gk[4] = {v.x, v.y, v.z, v.w};
        relax::bc7_adjoint_px(m, k, gk, ge);
    }
    float4* go = reinterpret_cast<float4*>(gep + (size_t)i * 24);
#pragma unroll
    for (int j = 0; j < 6; j++) go[j] = make_float4(ge[4 * j], ge[4 * j + 1], ge[4 * j + 2], ge[4 * j + 3]);
}

__global__ void __launch_bounds__(kThreads) bc1_parse_kernel(const uint8_t* __restrict__ blocks, uint32_t n,
                                                             bool aligned, uint32_t* __restrict__ meta,
                                                             float* __restrict__ ep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* p = blocks + (size_t)i * 8;
    uint32_t w0, w1;
    if (aligned) {
        uint2 v = __ldg(reinterpret_cast<const uint2*>(p));
        w0 = v.x;
        w1 = v.y;
    } else {
        w0 = (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
        w1 = (uint32_t)p[4] | (uint32_t)p[5] << 8 | (uint32_t)p[6] << 16 | (uint32_t)p[7] << 24;
    }
    uint32_t m[2];
    float e[6];
    relax::bc1_parse(w0, w1, m, e);
    meta[2 * (size_t)i] = m[0];
    meta[2 * (size_t)i + 1] = m[1];
#pragma unroll
    for (int j = 0; j < 6; j++) ep[(size_t)i * 6 + j] = e[j];
}

__global__ void __launch_bounds__(kThreads) bc1_relaxed_kernel(const uint32_t* __restrict__ meta,
                                                               const float* __restrict__ ep, uint32_t n,
                                                               float* __restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n * 16) return;
    uint32_t i = (uint32_t)(t >> 4);
    int k = (int)(t & 15);
    uint32_t m[2] = {meta[2 * (size_t)i], meta[2 * (size_t)i + 1]};
    float e[6];
#pragma unroll
    for (int j = 0; j < 6; j++) e[j] = ep[(size_t)i * 6 + j];
    float px[4];
    relax::bc1_relaxed_px(m, e, k, px);
    reinterpret_cast<float4*>(out)[t] = make_float4(px[0], px[1], px[2], px[3]);
}

__global__ void __launch_bounds__(kThreads) bc1_adjoint_kernel(const uint32_t* __restrict__ meta,
                                                               const float* __restrict__ g, uint32_t n,
                                                               float* __restrict__ gep) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t m[2] = {meta[2 * (size_t)i], meta[2 * (size_t)i + 1]};
    float ge[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const float4* gi = reinterpret_cast<const float4*>(g) + (size_t)i * 16;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        float4 v = gi[k];
        float gk[4] = {v.x, v.y, v.z, v.w};
        relax::bc1_adjoint_px(m, k, gk, ge);
    }
#pragma unroll
    for (int j = 0; j < 6; j++) gep[(size_t)i * 6 + j] = ge[j];
}

// ---- fused refinement -----------------------------------------------------------

// One launch refines up to kMaxImages images; grid.y selects the image.
constexpr int kMaxImages = 16;
struct RefineImage {
    const uint8_t* src;
    size_t stride;
    uint8_t* blocks;
    float* theta_out;
    uint32_t bw, bh;
    bool src_aligned, blk_aligned;
};
struct RefineBatch {
    RefineImage img[kMaxImages];
};

__global__ void __launch_bounds__(kThreads) bc7_endpoint_refine_kernel(const __grid_constant__ RefineBatch batch,
                                                                       uint32_t channels, uint32_t steps, float lr,
                                                                       unsigned long long* __restrict__ stats) {
    const RefineImage& im = batch.img[blockIdx.y];
    const uint8_t* __restrict__ src = im.src;
    const size_t stride = im.stride;
    const bool src_aligned = im.src_aligned, blk_aligned = im.blk_aligned;
    const uint32_t bw = im.bw, bh = im.bh;
    uint8_t* __restrict__ blocks = im.blocks;
    float* __restrict__ theta_out = im.theta_out;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < bw * bh;
    uint32_t active = 0, improved = 0, before = 0, after = 0;
    if (live) {
        uint32_t by = i / bw, bx = i - by * bw;
        uint32_t s[16];
        load_src(src, stride, bx, by, src_aligned, s);
        uint8_t* bp = blocks + (size_t)i * 16;
        uint4 best = load_block16(bp, blk_aligned);
        uint32_t m[6];
        float th[24];
        relax::bc7_parse((uint64_t)best.x | ((uint64_t)best.y << 32), (uint64_t)best.z | ((uint64_t)best.w << 32), m,
                         th);
        uint32_t best_err = bc7_exact_err(best, s, channels);
        before = best_err;
        if ((m[0] & 15) < 8) {
            active = 1;
            float mo[24], vo[24];
#pragma unroll
            for (int j = 0; j < 24; j++) mo[j] = vo[j] = 0.0f;
            float b1t = 1.0f, b2t = 1.0f;
            bool changed = false;
            for (uint32_t it = 0; it < steps; it++) {
                float ge[24];
#pragma unroll
                for (int j = 0; j < 24; j++) ge[j] = 0.0f;
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    float px[4], g[4];
                    relax::bc7_relaxed_px(m, th, k, px);
#pragma unroll
                    for (int c = 0; c < 4; c++) g[c] = c < (int)channels ? 2.0f * (px[c] - chan(s[k], c)) : 0.0f;
                    relax::bc7_adjoint_px(m, k, g, ge);
                }
                b1t *= 0.9f;
                b2t *= 0.999f;
                relax::adam_step<24>(th, mo, vo, ge, lr, b1t, b2t);
                uint4 cand = bc7_requant_code(m, th, channels);
                uint32_t err = bc7_exact_err(cand, s, channels);
                if (err < best_err) {
                    best_err = err;
                    best = cand;
                    changed = true;
                }
            }
            if (changed) {
                const uint32_t w[4] = {best.x, best.y, best.z, best.w};
                store_words(bp, w, 4, blk_aligned);
                improved = 1;
            }
        }
        after = best_err;
        if (theta_out) {
#pragma unroll
            for (int j = 0; j < 24; j++) theta_out[(size_t)i * 24 + j] = th[j];
        }
    }
    add_stats(stats, active, improved, before, after);
}

__global__ void __launch_bounds__(kThreads) bc1_endpoint_refine_kernel(const __grid_constant__ RefineBatch batch,
                                                                       uint32_t steps, float lr,
                                                                       unsigned long long* __restrict__ stats) {
    const RefineImage& im = batch.img[blockIdx.y];
    const uint8_t* __restrict__ src = im.src;
    const size_t stride = im.stride;
    const bool src_aligned = im.src_aligned, blk_aligned = im.blk_aligned;
    const uint32_t bw = im.bw, bh = im.bh;
    uint8_t* __restrict__ blocks = im.blocks;
    float* __restrict__ theta_out = im.theta_out;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < bw * bh;
    uint32_t active = 0, improved = 0, before = 0, after = 0;
    if (live) {
        uint32_t by = i / bw, bx = i - by * bw;
        uint32_t s[16];
        load_src(src, stride, bx, by, src_aligned, s);
        uint8_t* bp = blocks + (size_t)i * 8;
        uint32_t b0, b1;
        if (blk_aligned) {
            uint2 v = *reinterpret_cast<const uint2*>(bp);
            b0 = v.x;
            b1 = v.y;
        } else {
            b0 = (uint32_t)bp[0] | (uint32_t)bp[1] << 8 | (uint32_t)bp[2] << 16 | (uint32_t)bp[3] << 24;
            b1 = (uint32_t)bp[4] | (uint32_t)bp[5] << 8 | (uint32_t)bp[6] << 16 | (uint32_t)bp[7] << 24;
        }
        uint32_t m[2];
        float th[6];
        relax::bc1_parse(b0, b1, m, th);
        uint32_t best_err = bc1_exact_err(b0, b1, s);
        before = best_err;
        active = 1;
        float mo[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, vo[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        float b1t = 1.0f, b2t = 1.0f;
        bool changed = false;
        for (uint32_t it = 0; it < steps; it++) {
            float ge[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int k = 0; k < 16; k++) {
                float px[4], g[4];
                relax::bc1_relaxed_px(m, th, k, px);
#pragma unroll
                for (int c = 0; c < 4; c++) g[c] = c < 3 ? 2.0f * (px[c] - chan(s[k], c)) : 0.0f;
                relax::bc1_adjoint_px(m, k, g, ge);
            }
            b1t *= 0.9f;
            b2t *= 0.999f;
            relax::adam_step<6>(th, mo, vo, ge, lr, b1t, b2t);
            uint32_t c0, c1;
            bc1_requant_code(m, th, c0, c1);
            uint32_t err = bc1_exact_err(c0, c1, s);
            if (err < best_err) {
                best_err = err;
                b0 = c0;
                b1 = c1;
                changed = true;
            }
        }
        if (changed) {
            const uint32_t w[2] = {b0, b1};
            store_words(bp, w, 2, blk_aligned);
            improved = 1;
        }
        after = best_err;
        if (theta_out) {
#pragma unroll
            for (int j = 0; j < 6; j++) theta_out[(size_t)i * 6 + j] = th[j];
        }
    }
    add_stats(stats, active, improved, before, after);
}

int finish_launch() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    return BC_OK;
}

unsigned grid_for(uint64_t threads) { return (unsigned)((threads + kThreads - 1) / kThreads); }

bool aligned_to(const void* p, size_t a) { return ((uintptr_t)p % a) == 0; }

int check_refine_args(const uint8_t* src, size_t stride, uint32_t width, uint32_t height, const uint8_t* blocks,
                      size_t blocks_len, size_t block_bytes, uint32_t steps, float lr) {
    if (!src || !blocks) return BC_ERR_NULL;
    if (width % 4 != 0 || height % 4 != 0) return BC_ERR_DIMS;
    if (!std::isfinite(lr) || lr < 0.0f || steps > 100000) return BC_ERR_SETTINGS;
    if (stride < (size_t)width * 4) return BC_ERR_SRC_SIZE;
    if (blocks_len != (size_t)(width / 4) * (height / 4) * block_bytes) return BC_ERR_DST_SIZE;
    if ((uint64_t)(width / 4) * (height / 4) >= (1ull << 31)) return BC_ERR_DIMS;
    return BC_OK;
}

}  // namespace
}  // namespace bcn

using namespace bcn;

extern "C" int bc_bc7_parse_device(const uint8_t* blocks, size_t nblocks, uint32_t* meta, float* endpoints,
                                   void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!blocks || !meta || !endpoints) return BC_ERR_NULL;
    if (nblocks >= (1ull << 31)) return BC_ERR_DIMS;
    if (!aligned_to(meta, 16) || !aligned_to(endpoints, 16)) return BC_ERR_DST_SIZE;
    bc7_parse_kernel<<<grid_for(nblocks), kThreads, 0, (cudaStream_t)stream>>>(blocks, (uint32_t)nblocks,
                                                                              aligned_to(blocks, 16), meta,
                                                                              endpoints);
    return finish_launch();
}

extern "C" int bc_bc7_decode_relaxed_device(const uint32_t* meta, const float* endpoints, size_t nblocks,
                                            float* out, void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!meta || !endpoints || !out) return BC_ERR_NULL;
    if (nblocks >= (1ull << 27)) return BC_ERR_DIMS;
    if (!aligned_to(meta, 16) || !aligned_to(endpoints, 16) || !aligned_to(out, 16)) return BC_ERR_SRC_SIZE;
    bc7_relaxed_kernel<<<grid_for((uint64_t)nblocks * 16), kThreads, 0, (cudaStream_t)stream>>>(
        meta, endpoints, (uint32_t)nblocks, out);
    return finish_launch();
}

extern "C" int bc_bc7_decode_adjoint_device(const uint32_t* meta, const float* grad_out, size_t nblocks,
                                            float* grad_endpoints, void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!meta || !grad_out || !grad_endpoints) return BC_ERR_NULL;
    if (nblocks >= (1ull << 31)) return BC_ERR_DIMS;
    if (!aligned_to(meta, 16) || !aligned_to(grad_out, 16) || !aligned_to(grad_endpoints, 16))
        return BC_ERR_SRC_SIZE;
    bc7_adjoint_kernel<<<grid_for(nblocks), kThreads, 0, (cudaStream_t)stream>>>(meta, grad_out, (uint32_t)nblocks,
                                                                                grad_endpoints);
    return finish_launch();
}

extern "C" int bc_bc1_parse_device(const uint8_t* blocks, size_t nblocks, uint32_t* meta, float* endpoints,
                                   void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!blocks || !meta || !endpoints) return BC_ERR_NULL;
    if (nblocks >= (1ull << 31)) return BC_ERR_DIMS;
    bc1_parse_kernel<<<grid_for(nblocks), kThreads, 0, (cudaStream_t)stream>>>(blocks, (uint32_t)nblocks,
                                                                              aligned_to(blocks, 8), meta,
                                                                              endpoints);
    return finish_launch();
}

extern "C" int bc_bc1_decode_relaxed_device(const uint32_t* meta, const float* endpoints, size_t nblocks,
                                            float* out, void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!meta || !endpoints || !out) return BC_ERR_NULL;
    if (nblocks >= (1ull << 27)) return BC_ERR_DIMS;
    if (!aligned_to(out, 16)) return BC_ERR_SRC_SIZE;
    bc1_relaxed_kernel<<<grid_for((uint64_t)nblocks * 16), kThreads, 0, (cudaStream_t)stream>>>(
        meta, endpoints, (uint32_t)nblocks, out);
    return finish_launch();
}

extern "C" int bc_bc1_decode_adjoint_device(const uint32_t* meta, const float* grad_out, size_t nblocks,
                                            float* grad_endpoints, void* stream) {
    if (nblocks == 0) return BC_OK;
    if (!meta || !grad_out || !grad_endpoints) return BC_ERR_NULL;
    if (nblocks >= (1ull << 31)) return BC_ERR_DIMS;
    if (!aligned_to(grad_out, 16)) return BC_ERR_SRC_SIZE;
    bc1_adjoint_kernel<<<grid_for(nblocks), kThreads, 0, (cudaStream_t)stream>>>(meta, grad_out, (uint32_t)nblocks,
                                                                                grad_endpoints);
    return finish_launch();
}

// Validates and launches the images of one refinement call, kMaxImages per
// launch. bytes_per_block: 16 (BC7) or 8 (BC1).
template <class Launch>
int refine_images(const bc_refine_image* images, uint32_t count, uint32_t bytes_per_block, Launch&& launch) {
    if (count == 0) return BC_OK;
    if (!images) return BC_ERR_NULL;
    for (uint32_t i = 0; i < count; i++) {
        const bc_refine_image& im = images[i];
        int st = check_refine_args(im.src, im.src_stride, im.width, im.height, im.blocks, im.blocks_len,
                                   bytes_per_block, 0, 0.0f);
        if (st != BC_OK) return st;
    }
    for (uint32_t first = 0; first < count; first += kMaxImages) {
        uint32_t n = count - first < (uint32_t)kMaxImages ? count - first : (uint32_t)kMaxImages;
        RefineBatch b;
        uint64_t most = 0;
        for (uint32_t j = 0; j < n; j++) {
            const bc_refine_image& im = images[first + j];
            RefineImage& r = b.img[j];
            r.src = im.src;
            r.stride = im.src_stride;
            r.blocks = im.blocks;
            r.theta_out = im.endpoints_out;
            r.bw = im.width / 4;
            r.bh = im.height / 4;
            r.src_aligned = aligned_to(im.src, 16) && im.src_stride % 16 == 0;
            r.blk_aligned = aligned_to(im.blocks, bytes_per_block);
            uint64_t nb = (uint64_t)r.bw * r.bh;
            most = nb > most ? nb : most;
        }
        if (most == 0) continue;
        launch(b, dim3(grid_for(most), n));
        int st = finish_launch();
        if (st != BC_OK) return st;
    }
    return BC_OK;
}

extern "C" int bc_bc7_refine_images_device(const bc_refine_image* images, uint32_t count, uint32_t channels,
                                           uint32_t steps, float lr, uint64_t* stats, void* stream) {
    if (channels != 3 && channels != 4) return BC_ERR_SETTINGS;
    if (!std::isfinite(lr) || lr < 0.0f || steps > 100000) return BC_ERR_SETTINGS;
    return refine_images(images, count, 16, [&](const RefineBatch& b, dim3 grid) {
        bc7_endpoint_refine_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(
            b, channels, steps, lr, reinterpret_cast<unsigned long long*>(stats));
    });
}

extern "C" int bc_bc1_refine_images_device(const bc_refine_image* images, uint32_t count, uint32_t steps, float lr,
                                           uint64_t* stats, void* stream) {
    if (!std::isfinite(lr) || lr < 0.0f || steps > 100000) return BC_ERR_SETTINGS;
    return refine_images(images, count, 8, [&](const RefineBatch& b, dim3 grid) {
        bc1_endpoint_refine_kernel<<<grid, kThreads, 0, (cudaStream_t)stream>>>(
            b, steps, lr, reinterpret_cast<unsigned long long*>(stats));
    });
}

extern "C" int bc_bc7_refine_device(const uint8_t* src, size_t src_stride, uint32_t width, uint32_t height,
                                    uint8_t* blocks, size_t blocks_len, uint32_t channels, uint32_t steps,
                                    float lr, uint64_t* stats, float* endpoints_out, void* stream) {
    int st = check_refine_args(src, src_stride, width, height, blocks, blocks_len, 16, steps, lr);
    if (st != BC_OK) return st;
    const bc_refine_image im = {src, src_stride, width, height, blocks, blocks_len, endpoints_out};
    return bc_bc7_refine_images_device(&im, 1, channels, steps, lr, stats, stream);
}

extern "C" int bc_bc1_refine_device(const uint8_t* src, size_t src_stride, uint32_t width, uint32_t height,
                                    uint8_t* blocks, size_t blocks_len, uint32_t steps, float lr, uint64_t* stats,
                                    float* endpoints_out, void* stream) {
    int st = check_refine_args(src, src_stride, width, height, blocks, blocks_len, 8, steps, lr);
    if (st != BC_OK) return st;
    const bc_refine_image im = {src, src_stride, width, height, blocks, blocks_len, endpoints_out};
    return bc_bc1_refine_images_device(&im, 1, steps, lr, stats, stream);
}
