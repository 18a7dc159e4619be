// Internal launcher declarations shared by the kernel translation units and
// the C-ABI layer (capi.cu). Not part of the public interface.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace bcn {

// Variant ids: order of the reference enum CompressionVariant (src/lib.rs:74-103).
enum Variant { BC_BC1 = 0, BC_BC2 = 1, BC_BC3 = 2, BC_BC4 = 3, BC_BC5 = 4, BC_BC6H = 5, BC_BC7 = 6 };

// Settings with the byte layout of the reference's #[repr(C)] structs
// (src/settings.rs:207-213, :278-288).
struct BC6HSettingsDev {
    uint32_t slow_mode, fast_mode, refine_iterations_1p, refine_iterations_2p, fast_skip_threshold;
};
struct BC7SettingsDev {
    uint32_t refine_iterations[8];
    uint32_t mode_selection[4];
    uint32_t skip_mode2, fast_skip_threshold_mode1, fast_skip_threshold_mode3, fast_skip_threshold_mode7;
    uint32_t mode45_channel0, refine_iterations_channel, channels;
};

// One texture region of a batched launch: blocks of the region are numbered
// row-major from 0; its tiles of 32 blocks occupy the batch's global tile
// range [tile_base, tile_base + ceil(bw*bh/32)).
struct TaskDesc {
    const uint8_t* src;  // row 0 of the region
    uint8_t* dst;        // first block of the region
    uint64_t stride;     // bytes per source row
    uint32_t bw, bh;     // size in blocks
    uint32_t tile_base;
    uint32_t variant;
    uint32_t aligned;    // src and stride 16-byte aligned
    uint32_t pad;
};

// Source pixel formats a BC6H launch can read.
enum Bc6hSource { BC6H_SRC_RGBA16F = 0, BC6H_SRC_RGBA8_SRGB = 1 };

void launch_bc15_encode(int variant, const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst,
                        cudaStream_t s);
void launch_bc15_decode(int variant, const uint8_t* blocks, uint32_t bw, uint32_t bh, uint8_t* out, size_t pitch,
                        cudaStream_t s);
// BC7 runs as a short pipeline of kernels that exchange per-block state
// through `scratch` (device memory of at least bc7_scratch_bytes()).
size_t bc7_scratch_bytes(uint32_t nblocks, const BC7SettingsDev& settings);
// side_stream: run the independent stage chains on library-owned streams
// forked from `s` and joined before the final selection. While `s` captures
// a graph this needs bc7_side_streams_init() on the capturing thread first;
// without it the pipeline stays on `s`.
cudaError_t launch_bc7_encode(const uint8_t* src, size_t stride, uint32_t bw, uint32_t bh, uint8_t* dst,
                              const BC7SettingsDev& settings, void* scratch, cudaStream_t s,
                              bool side_stream = true);
// Batched form: the pipeline over `ntiles` tiles of several regions
// (tasks_dev / tile_task_dev in device memory). search_warps: 4 or 8
// candidates per CTA in the search launches.
size_t bc7_scratch_bytes_tiles(uint32_t ntiles, const BC7SettingsDev& settings);
// Creates the calling thread's BC7 side streams for the current device.
cudaError_t bc7_side_streams_init();
cudaError_t launch_bc7_batch(const TaskDesc* tasks_dev, const uint32_t* tile_task_dev, uint32_t ntiles,
                             const BC7SettingsDev& settings, void* scratch, int search_warps, cudaStream_t s);
// Persistent work-queue kernel over the tiles of BC1-BC5 regions: CTAs claim
// `tiles_per_claim` tiles per warp from *counter (zeroed by the caller) until
// the list is exhausted.
cudaError_t launch_bc15_batch(const TaskDesc* tasks_dev, const uint32_t* tile_task_dev, uint32_t ntiles,
                              uint32_t* counter_dev, int threads, int ctas, int tiles_per_claim, cudaStream_t s);
void launch_bc7_decode(const uint8_t* blocks, uint32_t bw, uint32_t bh, uint8_t* out, size_t pitch, cudaStream_t s);
// BC6H runs as a pipeline of kernels exchanging per-block state through
// `scratch` (device memory of at least bc6h_scratch_bytes()). stride in bytes
// of the source rows (RGBA16F: 8 bytes per pixel; RGBA8: 4).
size_t bc6h_scratch_bytes(uint32_t nblocks, const BC6HSettingsDev& settings);
cudaError_t launch_bc6h_encode(const void* src, size_t stride_bytes, int source_format, uint32_t bw, uint32_t bh,
                               uint8_t* dst, const BC6HSettingsDev& settings, void* scratch, cudaStream_t s);
// out_format: 0 RGBA8 (sRGB-encoded), 1 RGBA16F (RGB triplets in RGBA rows),
// 2 RGBA32F (same layout); pitch in output elements.
void launch_bc6h_decode(const uint8_t* blocks, uint32_t bw, uint32_t bh, void* out, size_t pitch, int out_format,
                        cudaStream_t s);

// Per-block decoders (the reference's decode_block_* functions): kinds in
// the order of the public BC_BLOCK_* values, plus the signed BC6H forms.
enum BlockKind {
    BLOCK_BC1 = 0, BLOCK_BC2 = 1, BLOCK_BC3 = 2, BLOCK_BC4 = 3, BLOCK_BC5 = 4,
    BLOCK_BC6H_HALF = 5, BLOCK_BC6H_FLOAT = 6, BLOCK_BC7 = 7,
    BLOCK_BC6H_HALF_SIGNED = 8, BLOCK_BC6H_FLOAT_SIGNED = 9
};
// Block i (8 or 16 bytes at blocks + i * size) decoded to `out` starting at
// element i * out_block_stride, rows `pitch` elements apart, written in the
// reference's element order.
void launch_decode_blocks(int kind, const uint8_t* blocks, size_t nblocks, void* out, size_t pitch,
                          size_t out_block_stride, cudaStream_t s);

// BC6H quality of `blocks` against the RGBA16F source (pitch in f16
// elements): sums[0] = squared RGB error, sums[1] = squared log2-luminance
// error, both in f64 over the image; block_sse (optional) the squared RGB
// error per block. partial: device scratch of bc6h_error_partial_bytes().
cudaError_t launch_bc6h_error(const uint8_t* blocks, uint32_t bw, uint32_t bh, const uint16_t* src, size_t src_pitch,
                              double* sums, double* block_sse, double* partial, cudaStream_t s);
size_t bc6h_error_partial_bytes();

// Check build (-DBCN_CHECK): each kernel translation unit's record of its
// first failed bounds guard (site, index, extent), read and cleared; release
// builds report none. launch_check_selftest evaluates one guard on the given
// index and extent without accessing memory.
cudaError_t check_take_bc7(unsigned long long out[3]);
cudaError_t check_take_bc6h(unsigned long long out[3]);
cudaError_t check_take_bc15(unsigned long long out[3]);
cudaError_t check_take_decode(unsigned long long out[3]);
cudaError_t launch_check_selftest(unsigned long long index, unsigned long long extent, cudaStream_t s);

// Settings check shared by every BC7 entry point (BC_OK or a BC_ERR_* code),
// and the per-thread record behind bc_last_cuda_error().
int validate_bc7_settings(const void* settings);
void record_cuda_error(cudaError_t e);

// One-time per-device table upload (sRGB conversion LUTs computed on the host).
int upload_bc6h_tables();
// Copies a host table into the device symbol of the translation unit that
// owns it (0x7C00 entries: f16 bits -> sRGB u8; 256 entries: u8 -> f16 bits).
cudaError_t set_half_to_srgb_table(const uint8_t* host);
cudaError_t set_srgb_to_half_table(const uint16_t* host);

}  // namespace bcn
