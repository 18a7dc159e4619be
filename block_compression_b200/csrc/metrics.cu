// Image-quality metric on the GPU: per-channel sums of squared differences
// between two RGBA8 images in the space the reference's quality tests use
// (tests/metrics.rs:40-114): RGB converted from sRGB to linear
// (tests/common/mod.rs:17-24), alpha as a / 255, all in f64.
//
// Two stream-ordered launches: a fixed grid of CTAs each reduces its share of
// the rows to 4 partial sums, then one CTA adds the partials in CTA order, so
// the result does not depend on scheduling.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/bc_capi.h"
#include "bc_kernels.h"

namespace bcn {
namespace {

constexpr int kThreads = 256;
constexpr int kCtas = 148 * 4;

__device__ double g_srgb_linear[256];

__global__ void __launch_bounds__(kThreads) sse_partial_kernel(const uint8_t* __restrict__ a, size_t pitch_a,
                                                               const uint8_t* __restrict__ b, size_t pitch_b,
                                                               uint32_t width, uint32_t height, uint32_t channels,
                                                               double* __restrict__ partial) {
    __shared__ double lut[256];
    __shared__ double red[kThreads / 32][4];
    for (int i = threadIdx.x; i < 256; i += kThreads) lut[i] = g_srgb_linear[i];
    __syncthreads();
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    const uint64_t total = (uint64_t)width * height;
    for (uint64_t p = (uint64_t)blockIdx.x * kThreads + threadIdx.x; p < total; p += (uint64_t)gridDim.x * kThreads) {
        uint32_t y = (uint32_t)(p / width), x = (uint32_t)(p - (uint64_t)y * width);
        uint32_t va = __ldg(reinterpret_cast<const uint32_t*>(a + (size_t)y * pitch_a) + x);
        uint32_t vb = __ldg(reinterpret_cast<const uint32_t*>(b + (size_t)y * pitch_b) + x);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (c >= (int)channels) continue;
            uint32_t ca = (va >> (8 * c)) & 0xFFu, cb = (vb >> (8 * c)) & 0xFFu;
            double d = c < 3 ? lut[ca] - lut[cb] : (double)ca / 255.0 - (double)cb / 255.0;
            acc[c] += d * d;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; w++) v += red[w][threadIdx.x];
        partial[(size_t)blockIdx.x * 4 + threadIdx.x] = v;
    }
}

__global__ void sse_final_kernel(const double* __restrict__ partial, int n, double* __restrict__ out) {
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int i = 0; i < n; i++) v += partial[(size_t)i * 4 + threadIdx.x];
        out[threadIdx.x] = v;
    }
}

std::mutex g_lut_mu;
bool g_lut_done[64];

// srgb_to_linear (tests/common/mod.rs:17-24) in f64, uploaded once per device.
int ensure_lut() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BC_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_lut_mu);
    if (g_lut_done[dev]) return BC_OK;
    double t[256];
    for (int i = 0; i < 256; i++) {
        double v = (double)i / 255.0;
        t[i] = v <= 0.04045 ? v / 12.92 : std::pow((v + 0.055) / 1.055, 2.4);
    }
    cudaError_t e = cudaMemcpyToSymbol(g_srgb_linear, t, sizeof(t));
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    g_lut_done[dev] = true;
    return BC_OK;
}

}  // namespace
}  // namespace bcn

using namespace bcn;

extern "C" int bc_image_sse_rgba8_device(const uint8_t* a, size_t pitch_a, const uint8_t* b, size_t pitch_b,
                                         uint32_t width, uint32_t height, uint32_t channels, double* sse_out,
                                         void* stream) {
    if (!a || !b || !sse_out) return BC_ERR_NULL;
    if (channels < 1 || channels > 4) return BC_ERR_SETTINGS;
    if (pitch_a < (size_t)width * 4 || pitch_b < (size_t)width * 4) return BC_ERR_SRC_SIZE;
    if (pitch_a % 4 || pitch_b % 4 || (uintptr_t)a % 4 || (uintptr_t)b % 4 || (uintptr_t)sse_out % 8)
        return BC_ERR_SRC_SIZE;
    int st = ensure_lut();
    if (st != BC_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    double* partial = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&partial, sizeof(double) * 4 * kCtas, s);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    sse_partial_kernel<<<kCtas, kThreads, 0, s>>>(a, pitch_a, b, pitch_b, width, height, channels, partial);
    sse_final_kernel<<<1, 32, 0, s>>>(partial, kCtas, sse_out);
    e = cudaGetLastError();
    cudaError_t f = cudaFreeAsync(partial, s);
    if (e == cudaSuccess) e = f;
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    return BC_OK;
}

extern "C" int bc_bc6h_error_device(const uint16_t* src_dev, size_t src_len_elems, size_t src_stride_elems,
                                    const uint8_t* blocks_dev, size_t blocks_len, uint32_t width, uint32_t height,
                                    double* sums_out, double* block_sse_out, void* stream) {
    if (!src_dev || !blocks_dev || !sums_out) return BC_ERR_NULL;
    if (width % 4 || height % 4) return BC_ERR_DIMS;
    const uint32_t bw = width / 4, bh = height / 4;
    if (blocks_len < (size_t)bw * bh * 16) return BC_ERR_SRC_SIZE;
    if (src_stride_elems < (size_t)width * 4) return BC_ERR_SRC_SIZE;
    if (height > 0 && src_len_elems < (size_t)(height - 1) * src_stride_elems + (size_t)width * 4)
        return BC_ERR_SRC_SIZE;
    if ((uintptr_t)sums_out % 8 || (uintptr_t)block_sse_out % 8 || (uintptr_t)src_dev % 2) return BC_ERR_SRC_SIZE;
    if (bw == 0 || bh == 0) return BC_OK;
    cudaStream_t s = (cudaStream_t)stream;
    double* partial = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&partial, bc6h_error_partial_bytes(), s);
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    e = launch_bc6h_error(blocks_dev, bw, bh, src_dev, src_stride_elems, sums_out, block_sse_out, partial, s);
    cudaError_t f = cudaFreeAsync(partial, s);
    if (e == cudaSuccess) e = f;
    if (e != cudaSuccess) {
        record_cuda_error(e);
        return BC_ERR_CUDA;
    }
    return BC_OK;
}
