"""Pins the CPU oracle to the reference's own known-answer data (CPU only).

decoder_kat.json holds the 18 decoder known-answer tests of
src/decode/block.rs:1405-1841; decoder_tables.json / encoder_tables.json the
reference's BPTC tables; settings_presets.json its quality presets. All were
extracted from the reference sources by tests/golden/make_golden.py.
"""
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


KATS = _load("decoder_kat.json")


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_oracle_decoder_known_answers(oracle_lib, kat):
    c = np.array(kat["compressed"], dtype=np.uint8)
    if kat["kind"] == "bc6h_half":
        out = np.zeros(48, np.uint16)
        oracle_lib.decode_block("bc6h_half", c, out, kat["pitch"], kat["is_signed"])
        assert out.tolist() == kat["expected"]
    elif kat["kind"] == "bc6h_float":
        out = np.zeros(48, np.float32)
        oracle_lib.decode_block("bc6h_float", c, out, kat["pitch"], kat["is_signed"])
        assert out.view(np.uint32).tolist() == kat["expected_f32_bits"]
    else:
        # The reference compares a 64-byte scratch buffer (rows overlap for the
        # BC7 tests, which use pitch 8); the whole buffer must match.
        out = np.zeros(64, np.uint8)
        oracle_lib.decode_block(kat["kind"], c, out, kat["pitch"])
        assert out.tolist() == kat["expected"]


def test_oracle_partition_tables_match_decoder_tables(oracle_lib):
    t = _load("decoder_tables.json")
    L = oracle_lib.lib()
    for p in range(32):
        assert [L.oracle_partition_set(p, k) for k in range(16)] == t["bc6h_partition_sets"][p]
    for p in range(64):
        assert [L.oracle_partition_set(p, k) for k in range(16)] == t["bc7_partition_sets_2"][p]
        assert [L.oracle_partition_set(64 + p, k) for k in range(16)] == t["bc7_partition_sets_3"][p]


def test_oracle_encoder_tables(oracle_lib):
    t = _load("encoder_tables.json")
    L = oracle_lib.lib()
    assert [L.oracle_get_pattern(p) for p in range(128)] == t["pattern"]
    assert [L.oracle_get_skip_packed(p) for p in range(128)] == t["skip"]
    packed = t["pattern_mask"]
    for p in range(128):
        m0, m1 = packed[p] & 0xFFFF, packed[p] >> 16
        assert L.oracle_get_pattern_mask(p, 0) == m0
        assert L.oracle_get_pattern_mask(p, 1) == m1
        assert L.oracle_get_pattern_mask(p, 2) == (~m0 & ~m1) & 0xFFFFFFFF


def test_f16_conversions_match_numpy(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.uniform(-70000, 70000, 2000), rng.uniform(-1e-4, 1e-4, 2000),
                           np.array([0.0, -0.0, 65504.0, 65520.0, 6.1e-5, 5.96e-8, 2.98e-8, 1.0 / 3])]).astype(np.float32)
    for v in vals:
        assert L.oracle_f32_to_f16(float(v)) == int(np.array(v, np.float32).astype(np.float16).view(np.uint16))
    for h in range(0, 0x7C00, 7):
        assert L.oracle_f16_to_f32(h) == float(np.array(h, np.uint16).view(np.float16).astype(np.float32))


def test_round_trip_psnr_sanity(oracle_lib):
    """Oracle encode -> known-answer-pinned decode gives plausible quality."""
    from block_compression_b200 import synthetic
    img = synthetic.config1_image(seed=11, size=128)
    for v, floor in [(0, 28.0), (2, 28.0)]:
        blocks = oracle_lib.compress_rgba8(v, img, 128, 128)
        dec = oracle_lib.decompress_rgba8(v, blocks, 128, 128).reshape(img.shape)
        mse = np.mean((dec[..., :3].astype(np.float64) - img[..., :3]) ** 2)
        assert 10 * np.log10(255.0 ** 2 / mse) > floor


def test_count_division_shortcut_is_exact(oracle_lib):
    """The BC7 kernels divide integer pixel statistics by a pixel count with
    a reciprocal and one fused correction step; over every integer numerator
    in [0, 2^24] and every count 1..16 that must equal IEEE division."""
    assert oracle_lib.lib().oracle_check_div_count() == 0


@pytest.mark.parametrize("d", [31.0, 255.0, 65535.0])
def test_constant_division_shortcut_is_exact(oracle_lib, d):
    """The encoders' scale conversions divide by 31, 255 and 65535 with a
    reciprocal and one fused correction step; for every finite float
    numerator (all 2^32 bit patterns, -0 aside) that must equal IEEE
    division."""
    assert oracle_lib.lib().oracle_check_div_const(d, os.cpu_count() or 1) == 0


def test_integer_pair_division_shortcut_is_exact(oracle_lib):
    """The BC7 index fit divides integer sums of 8-bit products by each other
    with a reciprocal and one fused correction step; for every numerator and
    divisor in [1, 4 * 255^2] that must equal IEEE division."""
    assert oracle_lib.lib().oracle_check_div_int_pairs(os.cpu_count() or 1) == 0


def test_channel_division_shortcut_is_exact(oracle_lib):
    """The BC7 mode-4/5 scalar-channel fit divides an 8-bit difference by an
    8-bit difference plus 0.001 with a reciprocal and one fused correction
    step; every such pair must give the IEEE quotient."""
    assert oracle_lib.lib().oracle_check_div_channel() == 0
