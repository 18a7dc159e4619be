// Mip-chain generation for the batched encode path: one 2x2 box-filter
// reduction per level, fused with the edge replication that pads a level to
// whole 4x4 blocks.
//
// Level i+1 of a w x h level has size max(1, w/2) x max(1, h/2); pixel (x, y)
// averages source pixels (2x, 2y), (2x+1, 2y), (2x, 2y+1), (2x+1, 2y+1) with
// coordinates clamped to the source, rounded as (sum + 2) / 4 per channel.
// The output buffer holds the level padded up to multiples of 4: padding
// pixels repeat the last valid column / row, so the encoder sees whole
// blocks (the reference API only accepts multiples of 4, src/encode.rs:91-92).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/bc_capi.h"
#include "bc_kernels.h"

namespace bcn {

__global__ void __launch_bounds__(256) box_down_pad_kernel(const uint8_t* __restrict__ src, size_t src_pitch,
                                                           uint32_t sw, uint32_t sh, uint8_t* __restrict__ dst,
                                                           size_t dst_pitch, uint32_t dw, uint32_t dh, uint32_t pw,
                                                           uint32_t ph) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= pw) return;
    for (uint32_t y = blockIdx.y; y < ph; y += gridDim.y) {
    uint32_t vx = min(x, dw - 1), vy = min(y, dh - 1);  // edge replication into the padding
    uint32_t x0 = min(2 * vx, sw - 1), x1 = min(2 * vx + 1, sw - 1);
    uint32_t y0 = min(2 * vy, sh - 1), y1 = min(2 * vy + 1, sh - 1);
    const uint32_t* r0 = reinterpret_cast<const uint32_t*>(src + (size_t)y0 * src_pitch);
    const uint32_t* r1 = reinterpret_cast<const uint32_t*>(src + (size_t)y1 * src_pitch);
    uint32_t a = r0[x0], b = r0[x1], c = r1[x0], d = r1[x1];
    uint32_t out = 0;
#pragma unroll
    for (int ch = 0; ch < 4; ch++) {
        uint32_t s = ((a >> (8 * ch)) & 0xFF) + ((b >> (8 * ch)) & 0xFF) + ((c >> (8 * ch)) & 0xFF) +
                     ((d >> (8 * ch)) & 0xFF);
        out |= ((s + 2) >> 2) << (8 * ch);
    }
    reinterpret_cast<uint32_t*>(dst + (size_t)y * dst_pitch)[x] = out;
    }
}

}  // namespace bcn

using namespace bcn;

extern "C" int bc_mip_level_rgba8_device(const uint8_t* src, size_t src_pitch, uint32_t sw, uint32_t sh,
                                         uint8_t* dst, size_t dst_pitch, size_t dst_len, void* stream) {
    if (!src || !dst) return BC_ERR_NULL;
    if (sw == 0 || sh == 0) return BC_ERR_DIMS;
    if (src_pitch % 4 != 0 || dst_pitch % 4 != 0 || (uintptr_t)src % 4 != 0 || (uintptr_t)dst % 4 != 0)
        return BC_ERR_SRC_SIZE;
    uint32_t dw = sw > 1 ? sw / 2 : 1, dh = sh > 1 ? sh / 2 : 1;
    uint32_t pw = (dw + 3) & ~3u, ph = (dh + 3) & ~3u;
    if (dst_pitch < (size_t)pw * 4) return BC_ERR_DST_SIZE;
    if (dst_len < (size_t)(ph - 1) * dst_pitch + (size_t)pw * 4) return BC_ERR_DST_SIZE;
    dim3 grid((pw + 255) / 256, ph < 65535 ? ph : 65535);
    box_down_pad_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(src, src_pitch, sw, sh, dst, dst_pitch, dw, dh, pw, ph);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    return BC_OK;
}
