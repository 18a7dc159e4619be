"""Image-quality metrics on the GPU, the reference's test metric
(tests/metrics.rs:40-114): per-channel MSE and PSNR of two RGBA8 images, RGB
compared in linear light (sRGB decoded, tests/common/mod.rs:17-24), alpha as
a / 255."""
import math

from . import _buffers
from ._lib import check, lib


class ChannelMetrics:
    __slots__ = ("psnr", "mse")

    def __init__(self, mse):
        self.mse = mse
        self.psnr = _psnr(mse)

    def __repr__(self):
        return "ChannelMetrics(psnr=%.4f, mse=%.9g)" % (self.psnr, self.mse)


class PsnrResult:
    """overall_psnr, overall_mse and per-channel results (red, green, blue,
    alpha), computed as calculate_image_metrics_rgba8 computes them."""
    __slots__ = ("overall_psnr", "overall_mse", "red", "green", "blue", "alpha", "sse")

    def __init__(self, sse, pixel_count, channels):
        self.sse = list(sse)
        mse = [v / pixel_count for v in sse]
        self.overall_mse = sum(mse) / channels
        self.overall_psnr = _psnr(self.overall_mse)
        self.red, self.green, self.blue, self.alpha = (ChannelMetrics(m) for m in mse)

    def __repr__(self):
        return "PsnrResult(overall_psnr=%.4f, overall_mse=%.9g)" % (self.overall_psnr, self.overall_mse)


def _psnr(mse):
    return 0.0 if mse == 0.0 else 20.0 * math.log10(1.0 / math.sqrt(mse))


def image_sse_rgba8(a, b, width, height, channels=4, pitch_a=None, pitch_b=None, out=None, stream=None):
    """Per-channel sums of squared differences (CUDA float64 tensor of 4) of
    two CUDA uint8 RGBA8 images. Stream-ordered; nothing is synchronised."""
    import torch

    va, vb = _buffers.view(a), _buffers.view(b)
    if not (va.cuda and vb.cuda):
        raise ValueError("images must be CUDA tensors")
    if out is None:
        out = torch.zeros(4, dtype=torch.float64, device=a.device)
    s = stream if stream is not None else _buffers.current_stream_ptr()
    check("bc_image_sse_rgba8_device",
          lib.bc_image_sse_rgba8_device(va.ptr, pitch_a or width * 4, vb.ptr, pitch_b or width * 4, width, height,
                                        channels, out.data_ptr(), s))
    return out


def calculate_image_metrics_rgba8(original, compressed, width, height, channels=4):
    """calculate_image_metrics_rgba8 (tests/metrics.rs:40-114) on the GPU.
    Returns a PsnrResult (synchronises to read the four sums)."""
    sse = image_sse_rgba8(original, compressed, width, height, channels)
    return PsnrResult(sse.cpu().tolist(), float(width * height), channels)


def bc6h_error(src, blocks, width, height, stride=None, block_sse=None, stream=None):
    """FP64 quality of BC6H `blocks` against their RGBA16F source `src` (CUDA
    buffers; stride in f16 elements, default width * 4). Returns a CUDA
    float64 tensor of 2: the squared RGB error and the squared log2-luminance
    error summed over the image; `block_sse` (CUDA float64, one per block)
    receives each block's squared RGB error. Stream-ordered."""
    import torch

    vs, vb = _buffers.view(src), _buffers.view(blocks)
    if not (vs.cuda and vb.cuda):
        raise ValueError("bc6h_error takes CUDA buffers")
    out = torch.zeros(2, dtype=torch.float64, device=blocks.device)
    bp = None
    if block_sse is not None:
        bp = _buffers.view(block_sse, writable=True)
        if bp.nbytes < (width // 4) * (height // 4) * 8:
            check("bc_bc6h_error_device", -2)
    s = stream if stream is not None else _buffers.current_stream_ptr()
    check("bc_bc6h_error_device",
          lib.bc_bc6h_error_device(vs.ptr, vs.nbytes // 2, stride or width * 4, vb.ptr, vb.nbytes, width, height,
                                   out.data_ptr(), bp.ptr if bp is not None else None, s))
    return out


def log_luminance_rmse(src, blocks, width, height, stride=None):
    """Root-mean-square error of log2 luminance (Rec. 709 weights) of the
    decoded BC6H image against its RGBA16F source (synchronises)."""
    sums = bc6h_error(src, blocks, width, height, stride).cpu().tolist()
    return math.sqrt(sums[1] / (width * height))
