"""BC6H quality on the HDR workload (1024x1024 RGBA16F, BC6H basic):
log-luminance RMSE and per-block squared error in FP64.

The GPU metric (bc_bc6h_error_device) is checked against a numpy float64
restatement: per-block squared RGB errors bit for bit (both add the 48
squared differences of exactly widened f16 values in the same order, with
no fused multiply-add), the image sums to 1e-12 relative (CUDA's and numpy's
log2 may differ in the last bit, and the reductions add in different
orders). Then every block the GPU encoder wrote is checked against the
oracle's block by an FP64 recomputation of both blocks' errors: none may be
worse than the reference's by more than 1e-6 relative, and all are expected
to be bit-identical.
"""
import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def decoded_rgb(oracle_lib, blocks, w, h):
    """(h, w, 3) float64 of the decoded image (decompress_blocks_as_rgba16f,
    src/decode.rs:397, writes each block row's 4 RGB triplets packed at the
    start of the block's 16-element span)."""
    out = oracle_lib.decompress_rgba16f(blocks, w, h).reshape(h, w // 4, 16)[:, :, :12]
    return out.reshape(h, w // 4, 4, 3).reshape(h, w, 3).view(np.float16).astype(np.float64)


def numpy_metric(src_rgb, dec_rgb):
    """(per-block squared RGB error, squared log2-luminance error per block),
    texels of a block in row-major order, channels R, G, B."""
    h, w = src_rgb.shape[:2]
    s = src_rgb.reshape(h // 4, 4, w // 4, 4, 3).transpose(0, 2, 1, 3, 4).reshape(-1, 16, 3)
    d = dec_rgb.reshape(h // 4, 4, w // 4, 4, 3).transpose(0, 2, 1, 3, 4).reshape(-1, 16, 3)
    sse = np.zeros(s.shape[0])
    for k in range(16):
        for c in range(3):
            t = d[:, k, c] - s[:, k, c]
            sse = sse + t * t
    lum = lambda x: np.log2(np.maximum(0.2126 * x[..., 0] + 0.7152 * x[..., 1] + 0.0722 * x[..., 2], 2.0 ** -24))
    lg = ((lum(d) - lum(s)) ** 2).sum(1)
    return sse, lg


def test_hdr_workload_log_luminance_and_fp64_block_errors(bcn, oracle_lib, cuda):
    import torch

    from block_compression_b200 import metrics
    n = 1024
    hdr = synthetic.config3_hdr(seed=3, size=n)
    s6 = bcn.BC6HSettings.basic()
    v = bcn.CompressionVariant.BC6H(s6)
    src = torch.from_numpy(hdr.view(np.int16)).cuda()
    blocks = torch.zeros(v.blocks_byte_size(n, n), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba16(v, src, blocks, n, n, n * 4)
    block_sse = torch.zeros((n // 4) ** 2, dtype=torch.float64, device="cuda")
    sums = metrics.bc6h_error(src, blocks, n, n, block_sse=block_sse).cpu().numpy()
    got = blocks.cpu().numpy()

    src_rgb = hdr.reshape(n, n, 4)[..., :3].astype(np.float64)
    sse_np, log_np = numpy_metric(src_rgb, decoded_rgb(oracle_lib, got, n, n))
    assert np.array_equal(block_sse.cpu().numpy().view(np.uint64), sse_np.view(np.uint64))
    assert sums[0] == pytest.approx(sse_np.sum(), rel=1e-12)
    assert sums[1] == pytest.approx(log_np.sum(), rel=1e-12)
    rmse = metrics.log_luminance_rmse(src, blocks, n, n)
    assert rmse == pytest.approx(np.sqrt(log_np.sum() / (n * n)), rel=1e-12)
    assert 0.0 < rmse < 0.1  # BC6H basic keeps luminance within a few percent on this content

    # FP64 recomputation of every block's error: the GPU's blocks against the oracle's
    exp = oracle_lib.compress_rgba16(hdr.view(np.uint16), n, n, s6.as_list())
    sse_ref, _ = numpy_metric(src_rgb, decoded_rgb(oracle_lib, exp, n, n))
    assert np.all(sse_np <= sse_ref * (1 + 1e-6))
    identical = (got.reshape(-1, 16) == exp.reshape(-1, 16)).all(1)
    assert identical.mean() >= 0.999
    assert identical.all()


def test_metric_argument_checks(bcn, cuda):
    import torch
    src = torch.zeros(16 * 4, dtype=torch.int16, device="cuda")
    blocks = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    L = bcn.lib
    assert L.bc_bc6h_error_device(src.data_ptr(), 64, 16, blocks.data_ptr(), 16, 4, 4, out.data_ptr(), None,
                                  None) == 0
    assert L.bc_bc6h_error_device(src.data_ptr(), 63, 16, blocks.data_ptr(), 16, 4, 4, out.data_ptr(), None,
                                  None) == -3
    assert L.bc_bc6h_error_device(src.data_ptr(), 64, 16, blocks.data_ptr(), 15, 4, 4, out.data_ptr(), None,
                                  None) == -3
    assert L.bc_bc6h_error_device(src.data_ptr(), 64, 16, blocks.data_ptr(), 16, 6, 4, out.data_ptr(), None,
                                  None) == -1
