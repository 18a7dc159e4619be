/* CPU oracle — TEST INFRASTRUCTURE ONLY.
 *
 * C entry points of the CPU restatement of the reference crate's codec
 * (novacrazy/block_compression v0.3.0). Tests, the smoke check and the
 * bench's CPU-baseline leg load liboracle.so through ctypes to check and
 * time the CUDA product path; the product never links it.
 *
 * Variant ids follow the order of the reference enum CompressionVariant
 * (src/lib.rs:74-103): 0 BC1, 1 BC2, 2 BC3, 3 BC4, 4 BC5, 5 BC6H, 6 BC7.
 * Status codes: 0 ok, <0 the condition under which the Rust code panics.
 */
#ifndef BCN_ORACLE_H
#define BCN_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_OK 0
#define ORACLE_ERR_DIMS -1      /* width/height not a multiple of 4 */
#define ORACLE_ERR_DST -2       /* destination too small / wrong size */
#define ORACLE_ERR_SRC -3       /* source slice too short */
#define ORACLE_ERR_VARIANT -4   /* variant not supported by this entry point */

/* encode::compress_rgba8 (src/encode.rs:83). stride in bytes. */
int oracle_compress_rgba8(int variant, const void* settings, const uint8_t* src, size_t src_len,
                          uint8_t* dst, size_t dst_len, uint32_t width, uint32_t height,
                          uint32_t stride, int threads);
/* encode::compress_rgba16 (src/encode.rs:211). stride in f16 elements. */
int oracle_compress_rgba16(const void* bc6h_settings, const uint16_t* src, size_t src_len,
                           uint8_t* dst, size_t dst_len, uint32_t width, uint32_t height,
                           uint32_t stride, int threads);
/* decode::decompress_blocks_as_rgba8 / rgba16f / rgba32f (src/decode.rs:336, 397, 438). */
int oracle_decompress_rgba8(int variant, uint32_t width, uint32_t height, const uint8_t* blocks,
                            size_t blocks_len, uint8_t* out, size_t out_len, int threads);
int oracle_decompress_rgba16f(uint32_t width, uint32_t height, const uint8_t* blocks,
                              size_t blocks_len, uint16_t* out, size_t out_len);
int oracle_decompress_rgba32f(uint32_t width, uint32_t height, const uint8_t* blocks,
                              size_t blocks_len, float* out, size_t out_len);

/* Per-block decoders (src/decode/block.rs public functions).
 * which: 0 bc1, 1 bc2, 2 bc3, 3 bc4, 4 bc5, 5 bc6h (u16 out), 6 bc6h_float (f32 out), 7 bc7.
 * pitch in output elements. */
void oracle_decode_block(int which, const uint8_t* block, void* out, size_t pitch, int is_signed);

/* Per-block encoders on the planar f32[64] block (R 0..15, G 16..31, B 32..47, A 48..63). */
void oracle_encode_block_bc1(const float* block, uint32_t out[2]);
void oracle_encode_block_bc3_alpha(const float* block, uint32_t out[2]);
void oracle_encode_block_bc7(const float* block, const void* bc7_settings, uint32_t out[4]);
void oracle_encode_block_bc6h(const float* block, const void* bc6h_settings, uint32_t out[4]);

/* Shared primitives exposed for the differential tests against the
 * independent Python restatement (src/encode/common.rs). */
float oracle_block_quant(uint32_t qblock[2], const float* block, uint32_t bits, const float* ep,
                         uint32_t pattern, uint32_t channels);
void oracle_opt_endpoints(float* ep, const float* block, uint32_t bits, const uint32_t qblock[2],
                          uint32_t mask, uint32_t channels);
float oracle_block_pca_bound_split(const float* block, uint32_t mask, uint32_t channels);
void oracle_block_segment_core(float* ep, const float* block, uint32_t mask, uint32_t channels);
/* ep_quant_dequant of src/encode/bc7.rs:234 (24 endpoint values, mode 0-7). */
void oracle_ep_quant_dequant(int32_t qep[24], float ep[24], uint32_t mode, uint32_t channels);
uint32_t oracle_get_pattern(int32_t part_id);
uint32_t oracle_get_pattern_mask(int32_t part_id, uint32_t j);
uint32_t oracle_get_skip_packed(int32_t part_id);
uint32_t oracle_partition_set(uint32_t table_index, uint32_t k);

/* Conversions restated from the `half` crate / Rust std on the BC6H paths. */
uint16_t oracle_f32_to_f16(float f);
float oracle_f16_to_f32(uint16_t h);
uint8_t oracle_linear_to_srgb(float linear);

#ifdef __cplusplus
}
#endif
#endif
