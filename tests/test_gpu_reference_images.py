"""The reference's own PSNR cases (tests/metrics.rs:255-526) on 128x128 crops
of its test images, through the CUDA path: the blocks equal the oracle's, the
decoded images equal the oracle's, and the GPU metric's PSNR
(bc_image_sse_rgba8_device) is within the reference's tolerance (0.0025 dB,
tests/metrics.rs:245) of the committed oracle PSNR for that case."""
import json

import numpy as np
import pytest

import reference_images as ri

pytestmark = pytest.mark.gpu
TABLE = json.load(open(ri.TABLE))


@pytest.mark.parametrize("case", ri.CASES, ids=[ri.case_id(c) for c in ri.CASES])
def test_reference_image_round_trip(bcn, oracle_lib, cuda, case):
    import torch

    from block_compression_b200 import metrics
    im, vid, preset, ch = case
    img = ri.load(im)
    s = ri.settings_list(bcn, vid, preset)
    settings = (getattr(bcn.BC6HSettings, preset)() if vid == 5 else
                getattr(bcn.BC7Settings, preset)() if vid == 6 else None)
    v = bcn.CompressionVariant(vid, settings)
    blocks = np.zeros(v.blocks_byte_size(128, 128), np.uint8)
    bcn.encode.compress_rgba8(v, img, blocks, 128, 128, 128 * 4)  # host entry point
    exp = oracle_lib.compress_rgba8(vid, img, 128, 128, settings=s)
    assert np.array_equal(blocks, exp)
    src = torch.from_numpy(img.copy()).cuda()
    dec = torch.zeros(128 * 128 * 4, dtype=torch.uint8, device="cuda")
    bcn.decode.decompress_blocks_as_rgba8(v, 128, 128, torch.from_numpy(blocks).cuda(), dec)
    torch.cuda.synchronize()
    assert np.array_equal(dec.cpu().numpy(), oracle_lib.decompress_rgba8(vid, exp, 128, 128))
    gpu = metrics.calculate_image_metrics_rgba8(src, dec, 128, 128, ch)
    assert abs(gpu.overall_psnr - TABLE[ri.case_id(case)]) <= 0.0025
