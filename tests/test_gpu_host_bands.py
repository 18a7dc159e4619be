"""The host-buffer encode entry points cut images into bands of block rows
and overlap each band's copies with its neighbours' kernels. Bands are a
host-side schedule only: their blocks must equal the single device-buffer
encode of the whole image, including a short last band and a row stride
wider than the image."""
import numpy as np
import pytest
import torch

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def _variants(bcn):
    V, S = bcn.CompressionVariant, bcn.BC7Settings
    return [("bc1", V.BC1), ("bc3", V.BC3), ("bc4", V.BC4), ("bc5", V.BC5), ("bc7", V.BC7(S.alpha_basic()))]


@pytest.mark.parametrize("name", ["bc1", "bc3", "bc4", "bc5", "bc7"])
def test_banded_host_encode_equals_device_encode(bcn, cuda, name):
    variant = dict(_variants(bcn))[name]
    # 1040 px wide with a 1088-px row stride: 4,352 bytes per row, so the
    # 4 MiB bands hold 960 rows; 2052 rows give three bands, the last of 132
    w, h, sw = 1040, 2052, 1088
    full = synthetic.config2_image(seed=5, size=2304)
    img = np.ascontiguousarray(full[:h, :sw])
    stride = sw * 4
    nbytes = variant.blocks_byte_size(w, h)
    host_out = np.zeros(nbytes, np.uint8)
    bcn.encode.compress_rgba8(variant, img, host_out, w, h, stride)
    dev_out = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba8(variant, torch.from_numpy(img).cuda(), dev_out, w, h, stride)
    torch.cuda.synchronize()
    assert np.array_equal(host_out, dev_out.cpu().numpy())


def test_banded_host_encode_bc6h_equals_device_encode(bcn, cuda):
    variant = bcn.CompressionVariant.BC6H(bcn.BC6HSettings.very_fast())
    # 8 bytes per pixel: 1024 px rows are 8 KiB, 512-row bands; 1032 rows
    # give three bands, the last of 8 rows
    w, h = 1024, 1032
    rng = np.random.default_rng(3)
    img = rng.uniform(0.0, 8.0, size=(h, w, 4)).astype(np.float16)
    nbytes = variant.blocks_byte_size(w, h)
    host_out = np.zeros(nbytes, np.uint8)
    bcn.encode.compress_rgba16(variant, img.view(np.uint16), host_out, w, h, w * 4)
    dev_out = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba16(variant, torch.from_numpy(img.view(np.int16)).cuda(), dev_out, w, h, w * 4)
    torch.cuda.synchronize()
    assert np.array_equal(host_out, dev_out.cpu().numpy())
