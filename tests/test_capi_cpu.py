"""The C-ABI library loads, exports what include/bc_capi.h declares, and its
host-side logic (sizes, presets, argument checks that mirror the reference's
asserts) behaves like the reference -- all without a GPU."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = []
    for hdr in ("bc_capi.h",):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^[a-z_0-9 ]+?\**\s*\**(bc_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(bcn):
    names = _declared_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(bcn.lib, n), n
    # and the dynamic symbol table really carries them
    lib = ctypes.CDLL(os.path.join(ROOT, "block_compression_b200", "libbcn_b200.so"))
    for n in names:
        getattr(lib, n)


def test_sizes_match_reference(bcn):
    V = bcn.CompressionVariant
    s7 = bcn.BC7Settings.alpha_basic()
    s6 = bcn.BC6HSettings.basic()
    for w, h in [(0, 0), (4, 4), (5, 7), (1024, 1024), (2048, 13), (1, 1)]:
        bw, bh = (w + 3) // 4, (h + 3) // 4
        for v, bb in [(V.BC1, 8), (V.BC2, 16), (V.BC3, 16), (V.BC4, 8), (V.BC5, 16), (V.BC6H(s6), 16),
                      (V.BC7(s7), 16)]:
            assert v.blocks_byte_size(w, h) == bw * bh * bb
            assert v.bytes_per_row(w) == bw * bb


def test_variant_equality_ignores_settings(bcn):
    V = bcn.CompressionVariant
    a = V.BC7(bcn.BC7Settings.alpha_basic())
    b = V.BC7(bcn.BC7Settings.opaque_fast())
    assert a == b and hash(a) == hash(b)
    assert V.BC1 != V.BC2


def test_presets_match_reference(bcn):
    golden = json.load(open(os.path.join(ROOT, "tests", "golden", "settings_presets.json")))
    for name, f in golden["bc6h"].items():
        s = getattr(bcn.BC6HSettings, name)()
        assert s.as_list() == [f["slow_mode"], f["fast_mode"], f["refine_iterations_1p"], f["refine_iterations_2p"],
                               f["fast_skip_threshold"]], name
    for name, f in golden["bc7"].items():
        s = getattr(bcn.BC7Settings, name)()
        exp = (f["refine_iterations"] + f["mode_selection"] +
               [f["skip_mode2"], f["fast_skip_threshold_mode1"], f["fast_skip_threshold_mode3"],
                f["fast_skip_threshold_mode7"], f["mode45_channel0"], f["refine_iterations_channel"], f["channels"]])
        assert s.as_list() == exp, name
    assert ctypes.sizeof(bcn.BC6HSettings) == 20 and ctypes.sizeof(bcn.BC7Settings) == 76


def test_argument_checks_without_gpu(bcn):
    """Checks that the reference expresses as assert!/panic! surface as the
    same conditions here, before any CUDA work is attempted."""
    L = bcn.lib
    V = bcn.CompressionVariant
    buf = np.zeros(64 * 64 * 4, np.uint8)
    out = np.zeros(4096, np.uint8)
    P = lambda a: a.ctypes.data
    # width/height not a multiple of 4 (src/encode.rs:91-92)
    assert L.bc_compress_rgba8(0, None, P(buf), buf.size, P(out), out.size, 6, 8, 24) == -1
    assert L.bc_compress_rgba8(0, None, P(buf), buf.size, P(out), out.size, 8, 6, 32) == -1
    # destination too small (src/encode.rs:96-101)
    assert L.bc_compress_rgba8(2, None, P(buf), buf.size, P(out), 10, 16, 16, 64) == -2
    # source slice too short
    assert L.bc_compress_rgba8(0, None, P(buf), 100, P(out), out.size, 16, 16, 64) == -3
    # compress_rgba16 with a non-BC6H variant (src/encode.rs:247-249)
    s6 = bcn.BC6HSettings.basic()
    assert L.bc_compress_rgba16(6, ctypes.byref(s6), P(buf), buf.size // 2, P(out), out.size, 8, 8, 32) == -4
    # BC7 needs settings; invalid settings are rejected
    assert L.bc_compress_rgba8(6, None, P(buf), buf.size, P(out), out.size, 8, 8, 32) == -6
    s7 = bcn.BC7Settings.alpha_basic()
    s7.channels = 5
    assert L.bc_compress_rgba8(6, ctypes.byref(s7), P(buf), buf.size, P(out), out.size, 8, 8, 32) == -5
    s7 = bcn.BC7Settings.alpha_basic()
    s7.fast_skip_threshold_mode1 = 65
    assert L.bc_compress_rgba8(6, ctypes.byref(s7), P(buf), buf.size, P(out), out.size, 8, 8, 32) == -5
    s6.fast_skip_threshold = 33
    assert L.bc_compress_rgba16(5, ctypes.byref(s6), P(buf), buf.size // 2, P(out), out.size, 8, 8, 32) == -5
    # unknown variant
    assert L.bc_compress_rgba8(9, None, P(buf), buf.size, P(out), out.size, 8, 8, 32) == -4
    # zero-sized images are a no-op, as in the reference
    assert L.bc_compress_rgba8(0, None, P(buf), 0, P(out), 0, 0, 0, 0) == 0
    # decode size checks (src/decode.rs:343-355)
    rgba = np.zeros(16 * 16 * 4, np.uint8)
    blocks = np.zeros(V.BC1.blocks_byte_size(16, 16), np.uint8)
    assert L.bc_decompress_blocks_as_rgba8(0, 16, 16, P(blocks), blocks.size - 1, P(rgba), rgba.size) == -3
    assert L.bc_decompress_blocks_as_rgba8(0, 16, 16, P(blocks), blocks.size, P(rgba), rgba.size + 4) == -2
    # rgba16f / rgba32f decode only for BC6H (src/decode.rs:423-426)
    assert L.bc_decompress_blocks_as_rgba16f(0, 16, 16, P(blocks), blocks.size, P(rgba), rgba.size // 2) == -4
    # unknown preset names
    assert L.bc_bc7_settings_preset(b"nope", ctypes.byref(bcn.BC7Settings())) == -5


def test_python_api_raises_like_reference_panics(bcn):
    V = bcn.CompressionVariant
    with pytest.raises(bcn.BcError):
        bcn.encode.compress_rgba8(V.BC1, np.zeros(16 * 6 * 4, np.uint8), np.zeros(64, np.uint8), 6, 4, 24)
    with pytest.raises(bcn.BcError):
        bcn.decode.decompress_blocks_as_rgba8(V.BC1, 8, 8, np.zeros(31, np.uint8), np.zeros(256, np.uint8))


def test_block_decoder_length_rules_without_gpu(bcn):
    """The per-block decoders need the output length the reference's slice
    indexing needs (src/decode/block.rs); shorter buffers, short source blocks
    and is_signed on a non-BC6H kind are rejected before any CUDA work."""
    L = bcn.lib
    assert bcn.decode.block_min_len("bc1", 16) == 64
    assert bcn.decode.block_min_len("bc7", 8) == 40
    assert bcn.decode.block_min_len("bc4", 4) == 16
    assert bcn.decode.block_min_len("bc5", 8) == 32
    assert bcn.decode.block_min_len("bc6h", 12) == 48
    assert bcn.decode.block_min_len("bc6h_float", 12) == 48
    assert bcn.decode.block_min_len("bc6h_float", 20) == 80  # the slice advances by the pitch after row 4
    blk = np.zeros(16, np.uint8)
    out = np.zeros(64, np.uint8)
    P = lambda a: a.ctypes.data
    assert L.bc_decode_block_bc1(P(blk), 8, P(out), 63, 16) == -2
    assert L.bc_decode_block_bc7(P(blk), 15, P(out), 64, 16) == -3
    assert L.bc_decode_block_bc3(None, 16, P(out), 64, 16) == -6
    assert L.bc_decode_blocks_device(0, 1, P(blk), 1, P(out), 64, 16, 0, None) == -4
    assert L.bc_decode_blocks_device(8, 0, P(blk), 1, P(out), 64, 16, 0, None) == -4
    assert L.bc_decode_blocks_device(7, 0, P(blk), 2, P(out), 64, 8, 40, None) == -2
    assert L.bc_decode_blocks_device(7, 0, P(blk), 0, P(out), 0, 8, 40, None) == 0
