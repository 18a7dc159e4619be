"""Parity of the sm_100a kernels with the CPU oracle (the C++ restatement of
the reference codec), through the C ABI. Bit-exact for every variant: the
encoders keep the reference's float operation order, the decoders are
integer code.
"""
import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu

BC6H_PRESETS = ["very_fast", "fast", "basic", "slow", "very_slow"]
BC7_PRESETS = ["opaque_ultra_fast", "opaque_very_fast", "opaque_fast", "opaque_basic", "opaque_slow",
               "alpha_ultrafast", "alpha_very_fast", "alpha_fast", "alpha_basic", "alpha_slow"]


def _edge_blocks(rng, n_side=8):
    """A small image of hand-picked hard blocks: flat colours, two-colour
    blocks, single-channel ramps, extreme values, noise."""
    tiles = []
    for v in (0, 1, 127, 128, 254, 255):
        tiles.append(np.full((4, 4, 4), v, np.uint8))
    for a, b in [(0, 255), (10, 11), (200, 40), (255, 254)]:
        t = np.full((4, 4, 4), a, np.uint8)
        t[::2, ::2] = b
        tiles.append(t)
    for c in range(4):
        t = np.zeros((4, 4, 4), np.uint8)
        t[..., c] = np.arange(16, dtype=np.uint8).reshape(4, 4) * 17
        t[..., 3] = 255 if c != 3 else t[..., 3]
        tiles.append(t)
    while len(tiles) < n_side * n_side:
        tiles.append(rng.integers(0, 256, (4, 4, 4), dtype=np.uint8))
    rows = [np.concatenate(tiles[r * n_side:(r + 1) * n_side], axis=1) for r in range(n_side)]
    return np.ascontiguousarray(np.concatenate(rows, axis=0))


def _images(size=128):
    rng = np.random.default_rng(7)
    return {
        "textured": synthetic.config1_image(seed=5, size=size),
        "alpha": synthetic.config2_image(seed=6, size=size),
        "noise": rng.integers(0, 256, (size, size, 4), dtype=np.uint8),
        "edge": _edge_blocks(rng),
    }


def _gpu_encode(bcn, torch, variant, img):
    h, w = img.shape[:2]
    src = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    dst = torch.zeros(variant.blocks_byte_size(w, h), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba8(variant, src, dst, w, h, w * 4)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def _first_mismatch(a, b, bb):
    bad = np.nonzero((a.reshape(-1, bb) != b.reshape(-1, bb)).any(1))[0]
    return len(bad), (bad[:5].tolist() if len(bad) else [])


@pytest.mark.parametrize("vid", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("name", ["textured", "alpha", "noise", "edge"])
def test_bc1_to_bc5_encode_bit_exact(bcn, oracle_lib, cuda, vid, name):
    import torch
    img = _images()[name]
    h, w = img.shape[:2]
    v = bcn.CompressionVariant(vid)
    got = _gpu_encode(bcn, torch, v, img)
    exp = oracle_lib.compress_rgba8(vid, img, w, h)
    n, first = _first_mismatch(got, exp, v.block_byte_size())
    assert n == 0, "%d mismatching blocks, first %s" % (n, first)


@pytest.mark.parametrize("preset", BC7_PRESETS)
def test_bc7_encode_bit_exact(bcn, oracle_lib, cuda, preset):
    import torch
    s = getattr(bcn.BC7Settings, preset)()
    v = bcn.CompressionVariant.BC7(s)
    for name, img in _images(size=64).items():
        h, w = img.shape[:2]
        got = _gpu_encode(bcn, torch, v, img)
        exp = oracle_lib.compress_rgba8(6, img, w, h, settings=s.as_list())
        n, first = _first_mismatch(got, exp, 16)
        assert n == 0, "%s/%s: %d mismatching blocks, first %s" % (preset, name, n, first)


def _hdr_images(size=64):
    rng = np.random.default_rng(9)
    hdr = synthetic.config3_hdr(seed=8, size=size)
    flat = np.zeros((16, 16, 4), np.float16)
    flat[4:8] = 1.0
    flat[8:12] = 60000.0
    flat[12:] = np.float16(2.0 ** -20)
    rnd = rng.integers(0, 0x7C00, (32, 32, 4), dtype=np.uint16).view(np.float16)
    return {"hdr": hdr, "flat": flat, "random_bits": rnd}


@pytest.mark.parametrize("preset", BC6H_PRESETS)
def test_bc6h_encode_bit_exact(bcn, oracle_lib, cuda, preset):
    import torch
    s = getattr(bcn.BC6HSettings, preset)()
    v = bcn.CompressionVariant.BC6H(s)
    for name, img in _hdr_images().items():
        h, w = img.shape[:2]
        src = torch.from_numpy(np.ascontiguousarray(img).view(np.int16)).cuda()
        dst = torch.zeros(v.blocks_byte_size(w, h), dtype=torch.uint8, device="cuda")
        bcn.encode.compress_rgba16(v, src, dst, w, h, w * 4)
        torch.cuda.synchronize()
        got = dst.cpu().numpy()
        exp = oracle_lib.compress_rgba16(img.view(np.uint16), w, h, s.as_list())
        n, first = _first_mismatch(got, exp, 16)
        assert n == 0, "%s/%s: %d mismatching blocks, first %s" % (preset, name, n, first)


def test_bc6h_from_rgba8_bit_exact(bcn, oracle_lib, cuda):
    """compress_rgba8 with BC6H: sRGB->linear->f16 input conversion
    (src/encode/bc6h.rs:45-71)."""
    import torch
    img = _images(size=64)["textured"]
    s = bcn.BC6HSettings.basic()
    v = bcn.CompressionVariant.BC6H(s)
    got = _gpu_encode(bcn, torch, v, img)
    exp = oracle_lib.compress_rgba8(5, img, 64, 64, settings=s.as_list())
    n, first = _first_mismatch(got, exp, 16)
    assert n == 0, "%d mismatching blocks, first %s" % (n, first)


@pytest.mark.parametrize("vid", [0, 1, 2, 3, 4, 5, 6])
def test_decode_random_blocks_bit_exact(bcn, oracle_lib, cuda, vid):
    """Random block bytes exercise every mode, partition and the reserved /
    invalid encodings of the decoders."""
    import torch
    rng = np.random.default_rng(100 + vid)
    w, h = 128, 64
    v = bcn.CompressionVariant(vid, bcn.BC6HSettings.basic() if vid == 5 else
                               (bcn.BC7Settings.alpha_basic() if vid == 6 else None))
    blocks = rng.integers(0, 256, v.blocks_byte_size(w, h), dtype=np.uint8)
    if vid == 6:
        # make every BC7 mode (and the invalid all-zero mode byte) frequent
        modes = rng.integers(0, 9, blocks.size // 16)
        first = np.where(modes < 8, (1 << modes) & 0xFF, 0).astype(np.uint8)
        blocks.reshape(-1, 16)[:, 0] = first | (blocks.reshape(-1, 16)[:, 0] & ~((2 << modes) - 1).astype(np.uint8))
    b_dev = torch.from_numpy(blocks).cuda()
    out = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
    bcn.decode.decompress_blocks_as_rgba8(v, w, h, b_dev, out)
    torch.cuda.synchronize()
    exp = oracle_lib.decompress_rgba8(vid, blocks, w, h)
    assert np.array_equal(out.cpu().numpy(), exp)
    if vid == 5:
        o16 = torch.full((w * h * 4,), 0x1234, dtype=torch.int16, device="cuda")
        bcn.decode.decompress_blocks_as_rgba16f(v, w, h, b_dev, o16)
        exp16 = np.full(w * h * 4, 0x1234, np.uint16)
        oracle_lib.decompress_rgba16f(blocks, w, h, out=exp16)
        assert np.array_equal(o16.cpu().numpy().view(np.uint16), exp16)
        o32 = torch.full((w * h * 4,), -7.0, dtype=torch.float32, device="cuda")
        bcn.decode.decompress_blocks_as_rgba32f(v, w, h, b_dev, o32)
        exp32 = np.full(w * h * 4, -7.0, np.float32)
        oracle_lib.decompress_rgba32f(blocks, w, h, out=exp32)
        assert np.array_equal(o32.cpu().numpy().view(np.uint32), exp32.view(np.uint32))


def test_host_entry_points_match_device_ones(bcn, oracle_lib, cuda):
    """bc_compress_rgba8 / bc_decompress_* with host buffers (the drop-in for
    the reference's CPU functions) give the same bytes."""
    img = _images(size=64)["alpha"]
    for vid in range(7):
        s = bcn.BC6HSettings.fast() if vid == 5 else (bcn.BC7Settings.alpha_fast() if vid == 6 else None)
        v = bcn.CompressionVariant(vid, s)
        blocks = np.zeros(v.blocks_byte_size(64, 64), np.uint8)
        bcn.encode.compress_rgba8(v, img, blocks, 64, 64, 256)
        exp = oracle_lib.compress_rgba8(vid, img, 64, 64, settings=s.as_list() if s is not None else None)
        assert np.array_equal(blocks, exp), vid
        out = np.zeros(64 * 64 * 4, np.uint8)
        bcn.decode.decompress_blocks_as_rgba8(v, 64, 64, blocks, out)
        assert np.array_equal(out, oracle_lib.decompress_rgba8(vid, blocks, 64, 64)), vid


def test_padded_stride_and_unaligned_buffers(bcn, oracle_lib, cuda):
    import torch
    img = _images(size=64)["textured"]
    stride = 64 * 4 + 12  # not a multiple of 16: exercises the byte-wise loads
    padded = np.zeros((64, stride), np.uint8)
    padded[:, :256] = img.reshape(64, 256)
    for vid in (0, 2, 6):
        s = bcn.BC7Settings.alpha_fast() if vid == 6 else None
        v = bcn.CompressionVariant(vid, s)
        src = torch.from_numpy(padded.reshape(-1)).cuda()
        n = v.blocks_byte_size(64, 64)
        dst = torch.zeros(n + 4, dtype=torch.uint8, device="cuda")
        bcn.encode.compress_rgba8(v, src, dst[4:], 64, 64, stride)
        torch.cuda.synchronize()
        exp = oracle_lib.compress_rgba8(vid, padded.reshape(-1), 64, 64, stride=stride,
                                        settings=s.as_list() if s is not None else None)
        assert np.array_equal(dst[4:].cpu().numpy(), exp), vid


def test_multi_task_compression(bcn, oracle_lib, cuda):
    """Four tasks in one compress(), split by texture_y_offset and
    blocks_offset as tests/multi_tasks.rs does; every region must equal the
    oracle's encode of that half."""
    import torch
    a = synthetic.config1_image(seed=21, size=64)
    b = synthetic.config2_image(seed=22, size=96)[:, :64].copy()
    for vid in range(7):
        s = bcn.BC6HSettings.very_fast() if vid == 5 else (bcn.BC7Settings.opaque_ultra_fast() if vid == 6 else None)
        v = bcn.CompressionVariant(vid, s)
        if vid == 5:
            ta = torch.from_numpy(a.astype(np.float16).view(np.int16)).cuda()
            tb = torch.from_numpy(b.astype(np.float16).view(np.int16)).cuda()
        else:
            ta, tb = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
        ha, hb = (a.shape[0] // 2) & ~3, (b.shape[0] // 2) & ~3
        sa, sb = v.blocks_byte_size(64, ha), v.blocks_byte_size(64, hb)
        buf = torch.zeros(2 * sa + 2 * sb, dtype=torch.uint8, device="cuda")
        c = bcn.GpuBlockCompressor()
        c.add_compression_task(v, ta, 64, ha, buf)
        c.add_compression_task(v, ta, 64, ha, buf, texture_y_offset=ha, blocks_offset=sa)
        c.add_compression_task(v, tb, 64, hb, buf, blocks_offset=2 * sa)
        c.add_compression_task(v, tb, 64, hb, buf, texture_y_offset=hb, blocks_offset=2 * sa + sb)
        assert c.task_count() == 4
        c.compress()
        assert c.task_count() == 0
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
        parts = []
        for img, hh in ((a, ha), (b, hb)):
            for y0 in (0, hh):
                reg = np.ascontiguousarray(img[y0:y0 + hh])
                if vid == 5:
                    parts.append(oracle_lib.compress_rgba16(reg.astype(np.float16).view(np.uint16), 64, hh,
                                                            s.as_list()))
                else:
                    parts.append(oracle_lib.compress_rgba8(vid, reg, 64, hh,
                                                           settings=s.as_list() if s is not None else None))
        assert np.array_equal(got, np.concatenate(parts)), vid
