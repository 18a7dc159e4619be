"""DDS container header and the CLI's PNG reader (host code, no GPU)."""
import struct
import zlib

import numpy as np
import pytest

# DXGI formats the reference CLI maps each variant to (compressor/src/main.rs:343-353)
REFERENCE_DXGI = {"BC1": 72, "BC2": 75, "BC3": 78, "BC4": 80, "BC5": 83, "BC6H": 95, "BC7": 99}


def _variants(bcn):
    V = bcn.CompressionVariant
    return {"BC1": V.BC1, "BC2": V.BC2, "BC3": V.BC3, "BC4": V.BC4, "BC5": V.BC5,
            "BC6H": V.BC6H(bcn.BC6HSettings.basic()), "BC7": V.BC7(bcn.BC7Settings.alpha_basic())}


@pytest.mark.parametrize("mips", [1, 5])
def test_dds_header_layout(bcn, mips):
    from block_compression_b200 import dds
    for name, v in _variants(bcn).items():
        h = dds.dds_header(v, 320, 200, mips)
        assert len(h) == 148 and h[:4] == b"DDS "
        size, flags, height, width, linear, depth, mipc = struct.unpack_from("<7I", h, 4)
        assert (size, height, width, depth, mipc) == (124, 200, 320, 0, mips)
        assert flags == 0x1 | 0x2 | 0x4 | 0x1000 | 0x20000 | 0x80000
        assert linear == v.blocks_byte_size(320, 200)
        assert struct.unpack_from("<2I", h, 76) == (32, 0x4) and h[84:88] == b"DX10"
        caps = struct.unpack_from("<I", h, 108)[0]
        assert caps == (0x1000 | (0x400008 if mips > 1 else 0))
        assert struct.unpack_from("<5I", h, 128) == (REFERENCE_DXGI[name], 3, 0, 1, 1)
        assert dds.dxgi_format(v) == REFERENCE_DXGI[name]
    assert dds.dxgi_format(bcn.CompressionVariant.BC7(bcn.BC7Settings.alpha_basic()), srgb=False) == 98
    with pytest.raises(bcn.BcError):
        dds.dds_header(bcn.CompressionVariant.BC1, 0, 4)


def _png(img, filters):
    h, w, c = img.shape
    ctype = {1: 0, 2: 4, 3: 2, 4: 6}[c]
    raw = bytearray()
    prev = np.zeros(w * c, dtype=np.int32)
    for y in range(h):
        cur = img[y].reshape(-1).astype(np.int32)
        ft = filters[y % len(filters)]
        out = np.zeros_like(cur)
        for x in range(w * c):
            a = cur[x - c] if x >= c else 0
            b = prev[x]
            cc = prev[x - c] if x >= c else 0
            p = {0: 0, 1: a, 2: b, 3: (a + b) >> 1}.get(ft)
            if ft == 4:
                pa, pb, pc = abs(b - cc), abs(a - cc), abs(a + b - 2 * cc)
                p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else cc)
            out[x] = (cur[x] - p) & 0xFF
        raw.append(ft)
        raw += out.astype(np.uint8).tobytes()
        prev = cur

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, ctype, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(bytes(raw))) + chunk(b"IEND", b""))


@pytest.mark.parametrize("chans", [1, 2, 3, 4])
def test_png_reader_all_filters(tmp_path, chans):
    from block_compression_b200.cli import read_png
    rng = np.random.default_rng(chans)
    img = rng.integers(0, 256, size=(9, 7, chans), dtype=np.uint8)
    p = tmp_path / "t.png"
    p.write_bytes(_png(img, [0, 1, 2, 3, 4]))
    got = read_png(str(p))
    exp = np.empty((9, 7, 4), dtype=np.uint8)
    if chans in (1, 2):
        exp[..., :3] = img[..., :1]
        exp[..., 3] = img[..., 1] if chans == 2 else 255
    else:
        exp[..., :3] = img[..., :3]
        exp[..., 3] = img[..., 3] if chans == 4 else 255
    assert np.array_equal(got, exp)


def test_cli_bc6h_input_table():
    from block_compression_b200.cli import srgb8_to_linear_f16_table
    t = srgb8_to_linear_f16_table()
    assert t[0] == 0 and t[255] == 1.0
    v = 128 / 255.0
    assert t[128] == np.float16(((v + 0.055) / 1.055) ** 2.4)
