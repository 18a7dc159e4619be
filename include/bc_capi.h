/* bc_capi.h — C ABI of the B200 (sm_100a) BCn block-compression library.
 *
 * Drop-in boundary for the per-4x4-block BCn codec of the Rust crate
 * block_compression v0.3.0 (novacrazy/block_compression). Every entry point
 * below names the reference interface it replaces. A Rust shim binds these
 * symbols with `extern "C"` and turns a negative status into the same panic
 * the reference raises.
 *
 * Conventions
 *   - Every function returns an int status: BC_OK (0) or a negative BC_ERR_*.
 *     Nothing aborts the process.
 *   - `stream` arguments are cudaStream_t values passed as void* (NULL = the
 *     legacy default stream). *_device entry points are stream-ordered and
 *     asynchronous: they validate arguments, enqueue kernels and return.
 *   - Host-pointer entry points (bc_compress_rgba8, ...) are synchronous and
 *     mirror the reference's CPU functions byte for byte. The encoders cut
 *     the image into bands of block rows (about 4 MiB of source each) and
 *     overlap each band's upload and download with its neighbours' kernels
 *     on library-owned streams; pinned (page-locked) host buffers let the
 *     copies run asynchronously.
 *   - Output blocks are little-endian, in row-major block order, exactly as
 *     the reference writes them (src/encode.rs store_data).
 *   - All work runs on the CUDA device current on the calling thread.
 */
#ifndef BC_CAPI_H
#define BC_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define BC_OK 0
#define BC_ERR_DIMS -1          /* width/height/y-offset not a multiple of 4 (src/encode.rs:91-92) */
#define BC_ERR_DST_SIZE -2      /* destination too small / not the expected size (src/encode.rs:96-101) */
#define BC_ERR_SRC_SIZE -3      /* source buffer shorter than the rows it must cover */
#define BC_ERR_VARIANT -4       /* variant not valid for this entry point (src/encode.rs:247-249) */
#define BC_ERR_SETTINGS -5      /* settings outside the range the reference can run */
#define BC_ERR_NULL -6          /* required pointer is NULL */
#define BC_ERR_CUDA -7          /* a CUDA runtime call failed (bc_last_cuda_error() has the code) */
#define BC_ERR_TASKS -8         /* task queue full / empty handle */
#define BC_ERR_NO_DEVICE -9     /* no usable sm_100 device */

/* ---- variants: order of CompressionVariant (src/lib.rs:74-103) ------------ */
typedef enum bc_variant {
    BC_VARIANT_BC1 = 0,
    BC_VARIANT_BC2 = 1,
    BC_VARIANT_BC3 = 2,
    BC_VARIANT_BC4 = 3,
    BC_VARIANT_BC5 = 4,
    BC_VARIANT_BC6H = 5,
    BC_VARIANT_BC7 = 6
} bc_variant;

/* BC6HSettings, byte layout of the #[repr(C)] struct (src/settings.rs:207-213). */
typedef struct bc_bc6h_settings {
    uint32_t slow_mode;
    uint32_t fast_mode;
    uint32_t refine_iterations_1p;
    uint32_t refine_iterations_2p;
    uint32_t fast_skip_threshold;
} bc_bc6h_settings;

/* BC7Settings, byte layout of the #[repr(C)] struct (src/settings.rs:278-288). */
typedef struct bc_bc7_settings {
    uint32_t refine_iterations[8];
    uint32_t mode_selection[4];
    uint32_t skip_mode2;
    uint32_t fast_skip_threshold_mode1;
    uint32_t fast_skip_threshold_mode3;
    uint32_t fast_skip_threshold_mode7;
    uint32_t mode45_channel0;
    uint32_t refine_iterations_channel;
    uint32_t channels;
} bc_bc7_settings;

/* Quality presets (src/settings.rs:217-441). `name` is the reference
 * constructor name, e.g. "basic", "alpha_basic", "opaque_ultra_fast".
 * Returns BC_ERR_SETTINGS for an unknown name. */
int bc_bc6h_settings_preset(const char* name, bc_bc6h_settings* out);
int bc_bc7_settings_preset(const char* name, bc_bc7_settings* out);

/* ---- sizes (CompressionVariant::bytes_per_row / blocks_byte_size, src/lib.rs:129-157) */
uint32_t bc_bytes_per_row(int variant, uint32_t width);
size_t bc_blocks_byte_size(int variant, uint32_t width, uint32_t height);

/* ---- encode, host buffers (synchronous) ---------------------------------
 * encode::compress_rgba8 (src/encode.rs:83-151). `settings` points to a
 * bc_bc6h_settings for BC6H, a bc_bc7_settings for BC7, and is ignored (may be
 * NULL) for BC1-BC5. stride is in bytes. rgba_len is the length of the
 * source slice, blocks_len of the destination slice. */
int bc_compress_rgba8(int variant, const void* settings, const uint8_t* rgba, size_t rgba_len,
                      uint8_t* blocks, size_t blocks_len, uint32_t width, uint32_t height,
                      uint32_t stride);

/* encode::compress_rgba16 (src/encode.rs:211-251). `rgba` holds IEEE binary16
 * values; stride and rgba_len are in f16 elements. variant must be BC6H. */
int bc_compress_rgba16(int variant, const bc_bc6h_settings* settings, const uint16_t* rgba,
                       size_t rgba_len, uint8_t* blocks, size_t blocks_len, uint32_t width,
                       uint32_t height, uint32_t stride);

/* ---- encode, device buffers (stream-ordered) -------------------------------
 * Same computation on device-resident buffers. Byte strides. */
int bc_compress_rgba8_device(int variant, const void* settings, const uint8_t* rgba_dev,
                             size_t rgba_len, uint8_t* blocks_dev, size_t blocks_len,
                             uint32_t width, uint32_t height, size_t stride_bytes, void* stream);
int bc_compress_rgba16_device(const bc_bc6h_settings* settings, const uint16_t* rgba_dev,
                              size_t rgba_len, uint8_t* blocks_dev, size_t blocks_len,
                              uint32_t width, uint32_t height, size_t stride_elems, void* stream);

/* ---- encode without allocating ---------------------------------------------
 * No counterpart in the reference. BC7 encode of device buffers exactly like
 * bc_compress_rgba8_device (same bytes), except that it allocates nothing:
 * the per-block scratch the BC7 kernels exchange lives in a fixed device
 * array compiled into the library (BC_NOALLOC_SCRATCH_BYTES, held on every
 * GPU that loads the library until the process exits).
 *
 * For callers that must not allocate device memory inside the call: engines
 * and plugins that own every byte of GPU memory through their own budgeted
 * allocator, code on a frame-critical thread that cannot risk an allocator
 * lock or an out-of-memory failure mid-frame, and processes running with the
 * device nearly full.
 *
 * Limits and rules:
 *  - images whose scratch need exceeds BC_NOALLOC_SCRATCH_BYTES are rejected
 *    with BC_ERR_TOO_LARGE; every preset fits images up to 1024x1024 pixels;
 *  - the first call on a device looks up the array's device address (a
 *    one-time set-up per device, repeated only when the device's context was
 *    replaced, as after cudaDeviceReset); make that first call before any
 *    stream capture;
 *  - all calls share the one array and it keeps the last call's contents:
 *    calls that overlap on the GPU (other streams, other host threads) race
 *    and corrupt each other's results; serialise them.
 */
#define BC_NOALLOC_SCRATCH_BYTES (40u * 1024u * 1024u)
#define BC_ERR_TOO_LARGE -10    /* image needs more scratch than BC_NOALLOC_SCRATCH_BYTES */
int bc_compress_bc7_device_noalloc(const bc_bc7_settings* settings, const uint8_t* rgba_dev,
                                   size_t rgba_len, uint8_t* blocks_dev, size_t blocks_len,
                                   uint32_t width, uint32_t height, size_t stride_bytes,
                                   void* stream);

/* ---- decode --------------------------------------------------------------
 * decode::decompress_blocks_as_rgba8 (src/decode.rs:336-387): blocks_len must
 * equal bc_blocks_byte_size(variant, w, h) and rgba_len must equal w*h*4.
 * BC4 decodes to (R,0,0,0), BC5 to (R,G,0,0), BC6H to sRGB-encoded RGB with
 * A=0, as the reference does (src/decode.rs:97-181). */
int bc_decompress_blocks_as_rgba8(int variant, uint32_t width, uint32_t height,
                                  const uint8_t* blocks, size_t blocks_len, uint8_t* rgba,
                                  size_t rgba_len);
/* decode::decompress_blocks_as_rgba16f / rgba32f (src/decode.rs:397-468), BC6H
 * only. Like the reference, each pixel's RGB triplet is written at element
 * (y*width*4 + bx*16 + x*3) of its row, leaving the last 4 elements of every
 * 16-element block row untouched. out_len is in elements (w*h*4). */
int bc_decompress_blocks_as_rgba16f(int variant, uint32_t width, uint32_t height,
                                    const uint8_t* blocks, size_t blocks_len, uint16_t* rgba,
                                    size_t rgba_len);
int bc_decompress_blocks_as_rgba32f(int variant, uint32_t width, uint32_t height,
                                    const uint8_t* blocks, size_t blocks_len, float* rgba,
                                    size_t rgba_len);
/* Device-buffer decode, stream-ordered. out_format: 0 RGBA8, 1 RGBA16F, 2 RGBA32F. */
int bc_decompress_device(int variant, uint32_t width, uint32_t height, const uint8_t* blocks_dev,
                         size_t blocks_len, void* out_dev, size_t out_len, int out_format,
                         void* stream);

/* ---- per-block decoders ----------------------------------------------------
 * decode::decode_block_bc1 .. decode_block_bc5 (src/decode/block.rs:50-119),
 * decode_block_bc6h (:262), decode_block_bc6h_float (:774) and
 * decode_block_bc7 (:801), re-exported by src/decode.rs:7-16. One block of
 * 8 (BC1, BC4) or 16 bytes is decoded into `decompressed_block` with
 * `destination_pitch` output elements between rows (bytes for BC1-BC5 and
 * BC7: RGBA8, R8 for BC4, RG8 for BC5; binary16 values for bc6h; floats for
 * bc6h_float), exactly as the reference writes it:
 *  - only the elements the reference writes are written (e.g. every 4th byte
 *    for BC4 at pitch 4 is not: BC4 writes 1 byte per texel), and in its
 *    order, so pitches shorter than a decoded row (overlapping rows) give the
 *    reference's contents too;
 *  - BC6H outputs RGB triplets; is_signed selects the signed-format decode;
 *  - decompressed_len (in elements) must be at least
 *    bc_decode_block_min_len(kind, pitch), where the reference's slice
 *    indexing would panic (BC_ERR_DST_SIZE); compressed_len must cover the
 *    block (BC_ERR_SRC_SIZE).
 * Host buffers, synchronous (the block is staged through the current device). */
#define BC_BLOCK_BC1 0
#define BC_BLOCK_BC2 1
#define BC_BLOCK_BC3 2
#define BC_BLOCK_BC4 3
#define BC_BLOCK_BC5 4
#define BC_BLOCK_BC6H 5       /* binary16 output (decode_block_bc6h) */
#define BC_BLOCK_BC6H_FLOAT 6 /* f32 output (decode_block_bc6h_float) */
#define BC_BLOCK_BC7 7
size_t bc_decode_block_min_len(int kind, size_t destination_pitch);
int bc_decode_block_bc1(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
int bc_decode_block_bc2(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
int bc_decode_block_bc3(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
int bc_decode_block_bc4(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
int bc_decode_block_bc5(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
int bc_decode_block_bc6h(const uint8_t* compressed_block, size_t compressed_len, uint16_t* decompressed_block,
                         size_t decompressed_len, size_t destination_pitch, int is_signed);
int bc_decode_block_bc6h_float(const uint8_t* compressed_block, size_t compressed_len, float* decompressed_block,
                               size_t decompressed_len, size_t destination_pitch, int is_signed);
int bc_decode_block_bc7(const uint8_t* compressed_block, size_t compressed_len, uint8_t* decompressed_block,
                        size_t decompressed_len, size_t destination_pitch);
/* Device form, stream-ordered: nblocks consecutive blocks of `kind` from
 * blocks_dev; block i is decoded as above into out_dev starting at element
 * i * out_block_stride (out_len elements in all). The output ranges of
 * different blocks must not overlap (their write order is not defined). */
int bc_decode_blocks_device(int kind, int is_signed, const uint8_t* blocks_dev, size_t nblocks, void* out_dev,
                            size_t out_len, size_t destination_pitch, size_t out_block_stride, void* stream);

/* ---- GpuBlockCompressor task interface (src/block_compressor.rs:44-590) ---- */
typedef struct bc_compressor bc_compressor;

/* GpuBlockCompressor::new (src/block_compressor.rs:66). `device` is a CUDA
 * device ordinal; -1 uses the current device. */
int bc_compressor_create(int device, bc_compressor** out);
int bc_compressor_destroy(bc_compressor* c);

/* GpuBlockCompressor::add_compression_task (src/block_compressor.rs:342-387).
 * src_dev: device pointer to row 0 of the source texture (RGBA8 for all
 *   variants but BC6H, RGBA16F for BC6H); src_pitch: bytes per texture row;
 *   src_len: bytes of the source allocation reachable from src_dev.
 * width/height: size of the region to compress; texture_y_offset: first
 *   texture row of the region (the reference's Option<u32>, 0 = None).
 * dst_dev/dst_len: destination buffer; blocks_offset: byte offset of the
 *   region's first block in it (the reference's Option<u32>, 0 = None; like the
 *   reference, which addresses the buffer in 4-byte words, the offset is
 *   rounded down to a multiple of 4).
 * settings: as for bc_compress_rgba8. The task keeps copies of the settings
 * and of the pointers (the buffers must stay alive until compress returns
 * work to the stream and that work completes). */
int bc_compressor_add_task(bc_compressor* c, int variant, const void* settings,
                           const void* src_dev, size_t src_pitch, size_t src_len, uint32_t width,
                           uint32_t height, uint32_t texture_y_offset, void* dst_dev,
                           size_t dst_len, uint32_t blocks_offset);

/* GpuBlockCompressor::compress (src/block_compressor.rs:540-590): enqueues
 * every pending task on `stream` as one launch per task and drains the queue. */
int bc_compressor_compress(bc_compressor* c, void* stream);

/* Number of pending tasks. */
int bc_compressor_task_count(const bc_compressor* c);

/* ---- batched compression (no counterpart in the reference: the reference
 * dispatches one compute shader per task, src/block_compressor.rs:550-589) --
 *
 * A bc_batch freezes every pending task of a compressor (the compressor's
 * queue is drained) into one device task table and one CUDA graph: one
 * persistent work-queue launch for all BC1-BC5 tiles, one pass of the BC7
 * kernel pipeline over the tiles of all BC7 tasks with the same settings,
 * one launch per BC6H task. bc_batch_launch replays the graph; the tasks'
 * buffers must stay valid while the batch exists.
 *
 * bc_tune is the launch shape. threads_per_cta: 128 or 256 (BC1-BC5 work
 * queue); ctas_per_sm: resident CTAs per SM of that queue (1-16);
 * tiles_per_claim: tiles of 32 blocks a warp takes per queue claim (1-64);
 * bc7_search_warps: 4 or 8 partition candidates per BC7 search CTA (one
 * staged tile shared by that many candidate warps). */
typedef struct bc_tune {
    uint32_t threads_per_cta;
    uint32_t ctas_per_sm;
    uint32_t tiles_per_claim;
    uint32_t bc7_search_warps;
} bc_tune;

typedef struct bc_batch bc_batch;

/* tune: explicit launch shape, or NULL. With NULL the shape comes from this
 * process's autotune cache for a batch of the same shape on the same device;
 * failing that, autotune != 0 times the candidate shapes on the batch itself
 * (running it several times on `stream`, writing the outputs) and caches the
 * winner, and autotune == 0 uses defaults. */
int bc_batch_create(bc_compressor* c, const bc_tune* tune, int autotune, void* stream, bc_batch** out);
int bc_batch_launch(bc_batch* b, void* stream);
int bc_batch_get_tune(const bc_batch* b, bc_tune* out);
int bc_batch_destroy(bc_batch* b);

/* One-shot: bc_batch_create (autotuned unless `tune` is given),
 * bc_batch_launch, synchronise `stream`, bc_batch_destroy. */
int bc_compressor_compress_batched(bc_compressor* c, void* stream, const bc_tune* tune);

/* ---- mip generation (no counterpart in the reference: callers supply mip
 * levels, src/block_compressor.rs:297-299) ------------------------------------
 * One mip level of an RGBA8 image: (sw, sh) -> (max(1, sw/2), max(1, sh/2)),
 * each pixel the 2x2 box average (coordinates clamped to the source,
 * (sum + 2) / 4 per channel), written padded up to multiples of 4 by edge
 * replication so the level can be block-compressed directly. dst_pitch >=
 * padded width * 4 bytes; all pointers and pitches 4-byte aligned. */
int bc_mip_level_rgba8_device(const uint8_t* src, size_t src_pitch, uint32_t sw, uint32_t sh,
                              uint8_t* dst, size_t dst_pitch, size_t dst_len, void* stream);

/* ---- differentiable decode and gradient endpoint refinement (no counterpart
 * in the reference) -------------------------------------------------------------
 * The relaxed decode replaces a block's quantised endpoints by continuous
 * endpoints in 8-bit units and drops the decoder's integer rounding, for a
 * fixed mode, partition, rotation, index selector and fixed indices:
 *   BC7: c = e0 + (e1 - e0) * w / 64, w the BPTC index weight
 *        (src/encode/common.rs:6-21), channels swapped by the block's rotation
 *        (src/decode/block.rs:1238-1243); modes 0-3 give alpha 255;
 *   BC1: c = e0 + (e1 - e0) * t, t = 0, 1, 1/3, 2/3 for indices 0..3 in the
 *        four-colour mode (block.rs:153-165), t = 0, 1, 1/2 and constant
 *        transparent black for index 3 in the three-colour mode (:166-175).
 * With the endpoints a parse returns, floor(c + 0.5) equals the decoder's
 * output. All buffers are device memory; calls are stream-ordered.
 *
 * Layouts per block:
 *   BC7 meta: 8 x uint32 (16-byte aligned), endpoints: 24 x float (slot
 *       (2 * subset + end) * 4 + channel, RGBA before the rotation swap,
 *       16-byte aligned);
 *   BC1 meta: 2 x uint32, endpoints: 6 x float (e0 RGB, e1 RGB);
 *   relaxed pixels and their gradients: 16 x 4 floats (pixel y * 4 + x,
 *       RGBA), 16-byte aligned.
 * A BC7 block with the reserved mode encoding decodes to zeros and has a zero
 * gradient. */
int bc_bc7_parse_device(const uint8_t* blocks, size_t nblocks, uint32_t* meta, float* endpoints,
                        void* stream);
int bc_bc7_decode_relaxed_device(const uint32_t* meta, const float* endpoints, size_t nblocks,
                                 float* out, void* stream);
/* Adjoint of the relaxed decode: grad_endpoints = (d out / d endpoints)^T grad_out. */
int bc_bc7_decode_adjoint_device(const uint32_t* meta, const float* grad_out, size_t nblocks,
                                 float* grad_endpoints, void* stream);
int bc_bc1_parse_device(const uint8_t* blocks, size_t nblocks, uint32_t* meta, float* endpoints,
                        void* stream);
int bc_bc1_decode_relaxed_device(const uint32_t* meta, const float* endpoints, size_t nblocks,
                                 float* out, void* stream);
int bc_bc1_decode_adjoint_device(const uint32_t* meta, const float* grad_out, size_t nblocks,
                                 float* grad_endpoints, void* stream);

/* Gradient endpoint refinement of encoded blocks against their RGBA8 source
 * (width x height, multiples of 4; src_stride in bytes). Per block: `steps`
 * Adam steps (beta1 0.9, beta2 0.999, eps 1e-8, learning rate `lr` in 8-bit
 * units) on the relaxed decode's squared error over the first `channels`
 * channels (BC1: RGB), each step followed by re-quantisation with the
 * encoder's quantisers and coding with the block's fixed indices
 * (src/encode/bc7.rs:97-276 and :381-515; src/encode/bc1_to_5.rs:268-278).
 * The best coded block replaces the input, in place, only if its exact
 * squared error (decoded texels against the source) is strictly lower.
 * stats (optional, 4 x uint64, added to, not cleared): blocks refined,
 * blocks replaced, summed exact error before, after.
 * endpoints_out (optional): the final continuous endpoints per block. */
int bc_bc7_refine_device(const uint8_t* src, size_t src_stride, uint32_t width, uint32_t height,
                         uint8_t* blocks, size_t blocks_len, uint32_t channels, uint32_t steps,
                         float lr, uint64_t* stats, float* endpoints_out, void* stream);
int bc_bc1_refine_device(const uint8_t* src, size_t src_stride, uint32_t width, uint32_t height,
                         uint8_t* blocks, size_t blocks_len, uint32_t steps, float lr,
                         uint64_t* stats, float* endpoints_out, void* stream);

/* Several images in one call (one launch per 16 images, so small images
 * still fill the GPU). `images` is a host array describing device buffers;
 * each entry as the arguments of bc_bc7_refine_device. */
typedef struct bc_refine_image {
    const uint8_t* src;     /* RGBA8 source rows (device) */
    size_t src_stride;      /* bytes per source row */
    uint32_t width, height; /* multiples of 4 */
    uint8_t* blocks;        /* encoded blocks (device), refined in place */
    size_t blocks_len;
    float* endpoints_out;   /* optional final continuous endpoints (device) */
} bc_refine_image;
int bc_bc7_refine_images_device(const bc_refine_image* images, uint32_t count, uint32_t channels,
                                uint32_t steps, float lr, uint64_t* stats, void* stream);
int bc_bc1_refine_images_device(const bc_refine_image* images, uint32_t count, uint32_t steps,
                                float lr, uint64_t* stats, void* stream);

/* ---- image-quality metric (the reference's test metric,
 * tests/metrics.rs:40-114, computed on the GPU) ----------------------------------
 * Per-channel sums of squared differences between two RGBA8 images a and b
 * (row pitches in bytes, 4-byte aligned) over the first `channels` channels,
 * in f64: RGB compared after sRGB -> linear (tests/common/mod.rs:17-24),
 * alpha as a / 255. sse_out: 4 doubles in device memory (unused channels are
 * 0). MSE = sse / (width * height); the reference's overall MSE is the mean of
 * the 4 channel MSEs over `channels`, PSNR = 20 log10(1 / sqrt(MSE)) (0 when
 * MSE is 0). The partial sums are added in a fixed order, so results do not
 * vary between runs; they may differ from a sequential sum in the last bits. */
int bc_image_sse_rgba8_device(const uint8_t* a, size_t pitch_a, const uint8_t* b, size_t pitch_b,
                              uint32_t width, uint32_t height, uint32_t channels, double* sse_out,
                              void* stream);

/* BC6H quality of encoded blocks against their RGBA16F source (the HDR
 * metric of the BC6H workload; the reference's own tests measure BC6H only
 * after an sRGB round trip to RGBA8). Both images are widened exactly to
 * f64; per texel the decoded RGB (the unsigned decoder of the image drivers,
 * src/decode.rs:397) is compared with the source RGB:
 *   sums_out[0] = sum over texels and R, G, B of (decoded - source)^2,
 *   sums_out[1] = sum over texels of (log2 L(decoded) - log2 L(source))^2,
 *                 L = 0.2126 R + 0.7152 G + 0.0722 B, floored at 2^-24;
 * the log-luminance RMSE is sqrt(sums_out[1] / (width * height)).
 * block_sse_out (optional, one double per block, row-major) receives each
 * block's squared RGB error. src_len_elems and src_stride_elems in f16
 * elements; device buffers; stream-ordered. The sums are added in a fixed
 * order. */
int bc_bc6h_error_device(const uint16_t* src_dev, size_t src_len_elems, size_t src_stride_elems,
                         const uint8_t* blocks_dev, size_t blocks_len, uint32_t width, uint32_t height,
                         double* sums_out, double* block_sse_out, void* stream);

/* ---- DDS container (the reference CLI's output, compressor/src/main.rs:313-353)
 * bc_dds_header writes the 148-byte header of a DX10-extended DDS file for one
 * 2D texture: "DDS " + DDS_HEADER + DDS_HEADER_DXT10, straight alpha, the
 * given mip count (the block data of every level follows the header, largest
 * first). srgb != 0 selects the _SRGB DXGI formats for BC1/BC2/BC3/BC7, as the
 * reference CLI does (:343-353); BC4/BC5 are UNORM, BC6H is UF16. */
#define BC_DDS_HEADER_BYTES 148u
int bc_dds_header(int variant, uint32_t width, uint32_t height, uint32_t mip_levels, int srgb,
                  uint8_t* out, size_t out_len);
uint32_t bc_dds_dxgi_format(int variant, int srgb);

/* ---- diagnostics -------------------------------------------------------- */
/* cudaError_t of the last CUDA failure seen on this thread (0 if none). */
int bc_last_cuda_error(void);
/* Bounds-checked debug build. libbcn_b200_check.so is the same library
 * compiled with every guarded index of the kernels (staged source rows and
 * columns, per-block scratch rows, output blocks, decoder shared-memory
 * slots) compared with its array's extent before the access; a failed guard
 * records (site, index, extent) and skips the access instead of trapping.
 * bc_check_enabled() is 1 in that build, 0 in the release build.
 * bc_check_read() copies the first recorded failure of each kernel file
 * since the last read into out (site, index, extent; site 0 = none) and
 * clears the records; it synchronises. bc_check_selftest() enqueues one
 * guard on (index, extent) that accesses no memory, to exercise the path. */
int bc_check_enabled(void);
int bc_check_read(uint64_t out[3]);
int bc_check_selftest(uint64_t index, uint64_t extent, void* stream);

/* Library version string, e.g. "bcn-b200 0.1.0 (sm_100a)". */
const char* bc_version(void);

#ifdef __cplusplus
}
#endif
#endif /* BC_CAPI_H */
