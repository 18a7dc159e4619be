"""GPU image metric against an f64 numpy restatement of the reference's
calculate_image_metrics_rgba8, and the CLI end to end (PNG in, DDS out)."""
import struct

import numpy as np
import pytest

from block_compression_b200 import synthetic

from test_tools_cpu import _png

pytestmark = pytest.mark.gpu


def _ref_metrics(a, b, channels):
    """tests/metrics.rs:40-114 in numpy f64 (sequential per-channel sums)."""
    def lin(x):
        v = x.astype(np.float64) / 255.0
        return np.where(v <= 0.04045, v / 12.92, ((v + 0.055) / 1.055) ** 2.4)
    mse = np.zeros(4)
    for c in range(channels):
        if c < 3:
            d = lin(a[..., c]) - lin(b[..., c])
        else:
            d = a[..., c].astype(np.float64) / 255.0 - b[..., c].astype(np.float64) / 255.0
        mse[c] = (d * d).sum() / (a.shape[0] * a.shape[1])
    return mse


@pytest.mark.parametrize("channels", [3, 4])
def test_gpu_metrics_match_reference_formula(bcn, cuda, channels):
    import torch
    from block_compression_b200 import metrics
    a = synthetic.config2_image(2, 256)
    v = bcn.CompressionVariant.BC7(bcn.BC7Settings.alpha_basic())
    ta = torch.from_numpy(a).cuda()
    blocks = torch.zeros(v.blocks_byte_size(256, 256), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba8(v, ta, blocks, 256, 256, 1024)
    out = torch.zeros(256 * 256 * 4, dtype=torch.uint8, device="cuda")
    bcn.decode.decompress_blocks_as_rgba8(v, 256, 256, blocks, out)
    r = metrics.calculate_image_metrics_rgba8(ta, out, 256, 256, channels)
    exp = _ref_metrics(a, out.view(256, 256, 4).cpu().numpy(), channels)
    got = np.array([r.red.mse, r.green.mse, r.blue.mse, r.alpha.mse])
    np.testing.assert_allclose(got, exp, rtol=1e-12, atol=0)
    assert r.overall_mse == pytest.approx(exp.sum() / channels, rel=1e-12)
    assert r.overall_psnr == pytest.approx(20 * np.log10(1 / np.sqrt(exp.sum() / channels)), rel=1e-12)
    same = metrics.calculate_image_metrics_rgba8(ta, ta, 256, 256, channels)
    assert same.overall_mse == 0.0 and same.overall_psnr == 0.0
    # deterministic across calls
    s1 = metrics.image_sse_rgba8(ta, out, 256, 256, channels).cpu().numpy()
    s2 = metrics.image_sse_rgba8(ta, out, 256, 256, channels).cpu().numpy()
    assert np.array_equal(s1, s2)


@pytest.mark.parametrize("name", ["bc1", "bc7", "bc6h"])
def test_cli_png_to_dds(bcn, oracle_lib, cuda, tmp_path, name):
    from block_compression_b200 import cli
    img = synthetic.config2_image(5, 64)[:62, :58]  # not multiples of 4: padded by edge replication
    p = tmp_path / "in.png"
    p.write_bytes(_png(img, [0, 1, 4]))
    out = cli.compress_file(name, str(p), log=lambda *a: None)
    assert out.endswith("in.dds")
    data = open(out, "rb").read()
    assert data[:4] == b"DDS " and struct.unpack_from("<2I", data, 12) == (64, 60)
    padded = synthetic.pad_to_multiple_of_4(img)
    v = cli._variant(name)
    if name == "bc6h":
        half = cli.srgb8_to_linear_f16_table()[padded]
        exp = oracle_lib.compress_rgba16(half.view(np.uint16), 60, 64, v.settings.as_list())
    else:
        exp = oracle_lib.compress_rgba8(v.id, padded, 60, 64,
                                        settings=v.settings.as_list() if v.settings is not None else None)
    assert np.array_equal(np.frombuffer(data[148:], dtype=np.uint8), exp)
