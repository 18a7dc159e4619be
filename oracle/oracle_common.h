// CPU oracle — TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the reference crate's CPU codec
// (novacrazy/block_compression v0.3.0, Rust). It exists so that tests, the
// smoke check and the bench's CPU-baseline leg can check the CUDA product
// path against the reference algorithm. Nothing in the shipped library links
// or calls this code.
//
// Pinning: the decoders are pinned by the reference's 18 decoder known-answer
// tests (tests/golden/decoder_kat.json); the encoders are parity unpinned --
// the reference ships no encode golden vectors and cannot be built here (no
// Rust toolchain), so the encoder half rests on transcription fidelity plus
// round trips through the pinned decoders.
//
// Floating point rules that keep it bit-identical to the Rust source:
//   * built with -O2 -ffp-contract=off (no FMA contraction), no fast-math;
//   * every f32 operation is written in the Rust source order;
//   * Rust `as i32` / `as u32` from f32 saturate and map NaN to 0 (f2i/f2u);
//   * Rust `f32::min/max` are IEEE minNum/maxNum (std::fmin/fmax);
//   * Rust `f32::clamp` is "if x<lo x=lo; if x>hi x=hi" (NaN passes through).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

inline int32_t f2i(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

inline uint32_t f2u(float x) {
    if (std::isnan(x) || x <= -1.0f) return 0;
    if (x >= 4294967296.0f) return UINT32_MAX;
    if (x < 0.0f) return 0;
    return (uint32_t)x;
}

inline float fmin_r(float a, float b) { return std::fmin(a, b); }
inline float fmax_r(float a, float b) { return std::fmax(a, b); }

inline float clampf_r(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

inline int32_t clampi_r(int32_t x, int32_t lo, int32_t hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

inline uint32_t clampu_r(uint32_t x, uint32_t lo, uint32_t hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

inline float sq(float x) { return x * x; }

// The encoder sources compute in `real`: plain f32 here, an op-counting f32
// in the op-counting build (oracle_count.h, -DORACLE_COUNT_OPS) that measures
// the reference algorithm's arithmetic per block.
#ifdef ORACLE_COUNT_OPS
}  // namespace oracle
#include "oracle_count.h"
namespace oracle {
#else
using real = float;
inline float sqrt_r(float x) { return std::sqrt(x); }
inline float fabs_r(float x) { return std::fabs(x); }
#endif

// Settings structs: byte layout of the reference's #[repr(C)] structs
// (src/settings.rs:207-213 and :278-288).
struct BC6HSettings {
    uint32_t slow_mode;
    uint32_t fast_mode;
    uint32_t refine_iterations_1p;
    uint32_t refine_iterations_2p;
    uint32_t fast_skip_threshold;
};

struct BC7Settings {
    uint32_t refine_iterations[8];
    uint32_t mode_selection[4];
    uint32_t skip_mode2;
    uint32_t fast_skip_threshold_mode1;
    uint32_t fast_skip_threshold_mode3;
    uint32_t fast_skip_threshold_mode7;
    uint32_t mode45_channel0;
    uint32_t refine_iterations_channel;
    uint32_t channels;
};

// ---- shared BC6H/BC7 math: src/encode/common.rs -------------------------

int32_t get_unquant_value(uint32_t bits, int32_t index);           // common.rs:6
uint32_t get_pattern(int32_t part_id);                              // common.rs:23
uint32_t get_pattern_mask(int32_t part_id, uint32_t j);             // common.rs:49
void get_skips(int32_t part_id, uint32_t skips[3]);                 // common.rs:85
void put_bits(uint32_t data[5], uint32_t* pos, uint32_t bits, uint32_t v);  // common.rs:103
void data_shl_1bit_from(uint32_t data[5], uint32_t from_bits);      // common.rs:111
void partial_sort_list(int32_t* list, uint32_t length, uint32_t partial_count);  // :126
void opt_endpoints(real* ep, const real block[64], uint32_t bits, const uint32_t qblock[2],
                   uint32_t mask, uint32_t channels);               // common.rs:142
real get_pca_bound(const real covar[10], uint32_t channels);      // common.rs:208
void compute_axis(real axis[4], const real covar[10], uint32_t power_iterations,
                  uint32_t channels);                               // common.rs:260
void compute_stats_masked(real stats[15], const real block[64], uint32_t mask,
                          uint32_t channels);                       // common.rs:294
void covar_from_stats(real covar[10], const real stats[15], uint32_t channels);  // :334
void compute_covar_dc_masked(real covar[10], real dc[4], const real block[64], uint32_t mask,
                             uint32_t channels);                    // common.rs:352
void block_pca_axis(real axis[4], real dc[4], const real block[64], uint32_t mask,
                    uint32_t channels);                             // common.rs:370
real block_pca_bound_split(const real block[64], uint32_t mask, const real full_stats[15],
                            uint32_t channels);                     // common.rs:396
real block_quant(uint32_t qblock[2], const real block[64], uint32_t bits, const real* ep,
                  uint32_t pattern, uint32_t channels);             // common.rs:422
void block_segment_core(real* ep, const real block[64], uint32_t mask, uint32_t channels);
void bc7_ep_quant_dequant(int32_t* qep, real* ep, uint32_t mode, uint32_t channels);  // bc7.rs:234
void bc7_code_qblock(uint32_t data[5], uint32_t* qpos, const uint32_t qblock[2], uint32_t bits,
                     uint32_t flips);                               // common.rs:520
void bc7_code_adjust_skip_mode01237(uint32_t data[5], uint32_t mode, int32_t part_id);
void bc7_code_apply_swap_mode456(int32_t* qep, uint32_t channels, uint32_t qblock[2],
                                 uint32_t bits);                    // common.rs:564
uint32_t bc7_code_apply_swap_mode01237(int32_t qep[24], const uint32_t qblock[2], uint32_t mode,
                                       int32_t part_id);            // common.rs:583

// ---- per-block encoders ---------------------------------------------------

// BC1-BC5 (src/encode/bc1_to_5.rs). `block` is the planar f32[64] layout
// R=0..15, G=16..31, B=32..47, A=48..63.
void bc1_core(const real block[64], uint32_t out[2]);       // bc1_to_5.rs:386
void bc3_alpha(const real block[64], uint32_t out[2]);      // bc1_to_5.rs:431

// BC7 (src/encode/bc7.rs) and BC6H (src/encode/bc6h.rs).
void bc7_encode_block(const real block[64], const BC7Settings* s, uint32_t out[4]);
void bc6h_encode_block(const real block_in[64], const BC6HSettings* s, uint32_t out[4]);

}  // namespace oracle
