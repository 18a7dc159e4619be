"""Bit-exact parity at the benchmark workloads' full sizes: every block of every
configuration the benchmark measures is compared with the CPU oracle.

  C1  1024x1024 RGBA8 (gradients + value noise + 32 triangles): BC1 encode,
      then decode of the encoded blocks;
  C2  2048x2048 RGBA8 with alpha: BC7 alpha_basic, BC3, BC4 (R); 2048x2048
      normal map: BC5;
  C3  1024x1024 RGBA16F HDR: BC6H basic through compress_rgba16;
  C4  the mixed mip-chain workload at reduced texture count (the first 6 of
      the 64 textures, every mip level), batched and per-task paths;
  C5  8 images 512x512 BC7 opaque_basic, plus the 20-step endpoint refinement
      of one whole image against the oracle's sequential restatement.
"""
import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def _encode(bcn, torch, variant, img):
    h, w = img.shape[:2]
    src = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    dst = torch.zeros(variant.blocks_byte_size(w, h), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba8(variant, src, dst, w, h, w * 4)
    torch.cuda.synchronize()
    return dst.cpu().numpy()


def _assert_blocks_equal(got, exp, bb, what):
    bad = np.nonzero((got.reshape(-1, bb) != exp.reshape(-1, bb)).any(1))[0]
    assert bad.size == 0, "%s: %d of %d blocks differ, first %s" % (what, bad.size, got.size // bb, bad[:5].tolist())


def test_c1_bc1_encode_decode_1024(bcn, oracle_lib, cuda):
    import torch
    img = synthetic.config1_image(seed=1, size=1024)
    got = _encode(bcn, torch, bcn.CompressionVariant.BC1, img)
    _assert_blocks_equal(got, oracle_lib.compress_rgba8(0, img, 1024, 1024), 8, "C1 BC1 encode")
    out = torch.zeros(1024 * 1024 * 4, dtype=torch.uint8, device="cuda")
    bcn.decode.decompress_blocks_as_rgba8(bcn.CompressionVariant.BC1, 1024, 1024, torch.from_numpy(got).cuda(), out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle_lib.decompress_rgba8(0, got, 1024, 1024))


@pytest.mark.parametrize("name", ["bc7_alpha_basic", "bc3", "bc4", "bc5"])
def test_c2_2048(bcn, oracle_lib, cuda, name):
    import torch
    V = bcn.CompressionVariant
    s7 = bcn.BC7Settings.alpha_basic()
    variant = {"bc7_alpha_basic": V.BC7(s7), "bc3": V.BC3, "bc4": V.BC4, "bc5": V.BC5}[name]
    img = synthetic.normal_map(seed=2, size=2048) if name == "bc5" else synthetic.config2_image(seed=2, size=2048)
    got = _encode(bcn, torch, variant, img)
    exp = oracle_lib.compress_rgba8(variant.id, img, 2048, 2048,
                                    settings=s7.as_list() if name.startswith("bc7") else None)
    _assert_blocks_equal(got, exp, 16 if variant.id != 3 else 8, "C2 " + name)


def test_c3_bc6h_basic_1024(bcn, oracle_lib, cuda):
    import torch
    hdr = synthetic.config3_hdr(seed=3, size=1024)
    s6 = bcn.BC6HSettings.basic()
    v = bcn.CompressionVariant.BC6H(s6)
    src = torch.from_numpy(hdr.view(np.int16)).cuda()
    dst = torch.zeros(v.blocks_byte_size(1024, 1024), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba16(v, src, dst, 1024, 1024, 1024 * 4)
    torch.cuda.synchronize()
    exp = oracle_lib.compress_rgba16(hdr.view(np.uint16), 1024, 1024, s6.as_list())
    _assert_blocks_equal(dst.cpu().numpy(), exp, 16, "C3 BC6H basic")


def test_c4_mip_chains_batched_and_per_task(bcn, oracle_lib, cuda):
    import torch

    from block_compression_b200 import mips
    V = bcn.CompressionVariant
    variants = [V.BC1, V.BC5, V.BC7(bcn.BC7Settings.alpha_basic())]
    shapes = synthetic.config4_textures(seed=4, count=64)[:6]
    chains = [mips.generate_mip_chain(synthetic.rgba8_textured_torch(4000 + i, h, w, cuda))
              for i, (h, w) in enumerate(shapes)]
    tasks, total = [], 0
    for i, chain in enumerate(chains):
        v = variants[i % 3]
        for lv in chain:
            n = v.blocks_byte_size(lv.padded_width, lv.padded_height)
            tasks.append((lv, v, total, n))
            total += n
    outs = []
    for batched in (False, True):
        c = bcn.GpuBlockCompressor()
        buf = torch.zeros(total, dtype=torch.uint8, device="cuda")
        for lv, v, off, n in tasks:
            c.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, buf, blocks_offset=off)
        c.compress_batched() if batched else c.compress()
        torch.cuda.synchronize()
        outs.append(buf.cpu().numpy())
    assert np.array_equal(outs[0], outs[1]), "batched and per-task outputs differ"
    for lv, v, off, n in tasks:
        img = lv.data.cpu().numpy()
        s = v.settings.as_list() if v.settings is not None else None
        exp = oracle_lib.compress_rgba8(v.id, img, lv.padded_width, lv.padded_height, settings=s)
        _assert_blocks_equal(outs[1][off:off + n], exp, 8 if v.id == 0 else 16,
                             "C4 %r %dx%d" % (v, lv.padded_width, lv.padded_height))


def test_c5_bc7_eight_images_and_refinement(bcn, oracle_lib, cuda):
    import torch

    from block_compression_b200 import refine
    s = bcn.BC7Settings.opaque_basic()
    v = bcn.CompressionVariant.BC7(s)
    imgs = [synthetic.config1_image(100 + i, 512) for i in range(8)]
    encoded = []
    for i, img in enumerate(imgs):
        got = _encode(bcn, torch, v, img)
        _assert_blocks_equal(got, oracle_lib.compress_rgba8(6, img, 512, 512, settings=s.as_list()), 16,
                             "C5 image %d" % i)
        encoded.append(got)
    # the refinement of image 0, whole, against the sequential restatement
    blocks = torch.from_numpy(encoded[0].copy()).cuda()
    refine.refine_bc7(torch.from_numpy(imgs[0]).cuda(), blocks, channels=3, steps=20, lr=0.5)
    torch.cuda.synchronize()
    exp, _, _ = oracle_lib.refine_blocks("bc7", encoded[0].reshape(-1, 16), oracle_lib.image_blocks(imgs[0], 512, 512),
                                         20, 0.5, 3)
    _assert_blocks_equal(blocks.cpu().numpy(), exp, 16, "C5 refinement")
