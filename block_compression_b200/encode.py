"""Encoding entry points mirroring the reference's `encode` module
(src/encode.rs:83-251), executed by the sm_100a kernels.

Host buffers (numpy arrays, bytes-like objects, CPU tensors) go through the
synchronous host entry points; CUDA tensors go through the stream-ordered
device entry points on torch's current stream. Where the reference panics,
these raise BcError with the C ABI status.
"""
import ctypes

from . import _buffers
from ._lib import check, lib
from .settings import BC6HSettings, CompressionVariant


def compress_rgba8(variant, rgba_data, blocks_buffer, width, height, stride, stream=None):
    """encode::compress_rgba8 (src/encode.rs:83): RGBA8 rows of `stride` bytes
    -> blocks written into `blocks_buffer`."""
    src = _buffers.view(rgba_data)
    dst = _buffers.view(blocks_buffer, writable=True)
    sp = variant.settings_ptr()
    if src.cuda != dst.cuda:
        raise ValueError("source and destination must both be host or both be CUDA buffers")
    if src.cuda:
        s = stream if stream is not None else _buffers.current_stream_ptr()
        check("bc_compress_rgba8_device",
              lib.bc_compress_rgba8_device(variant.id, sp, src.ptr, src.nbytes, dst.ptr, dst.nbytes,
                                           width, height, stride, s))
    else:
        check("bc_compress_rgba8",
              lib.bc_compress_rgba8(variant.id, sp, src.ptr, src.nbytes, dst.ptr, dst.nbytes,
                                    width, height, stride))


def compress_rgba16(variant, rgba_data, blocks_buffer, width, height, stride, stream=None):
    """encode::compress_rgba16 (src/encode.rs:211): RGBA binary16 rows of
    `stride` f16 elements -> BC6H blocks. Only BC6H is accepted."""
    src = _buffers.view(rgba_data)
    dst = _buffers.view(blocks_buffer, writable=True)
    if src.cuda != dst.cuda:
        raise ValueError("source and destination must both be host or both be CUDA buffers")
    sp = variant.settings_ptr()
    if src.cuda:
        if variant.id != 5:
            check("bc_compress_rgba16_device", -4)
        s = stream if stream is not None else _buffers.current_stream_ptr()
        check("bc_compress_rgba16_device",
              lib.bc_compress_rgba16_device(sp, src.ptr, src.nbytes // 2, dst.ptr, dst.nbytes, width, height,
                                            stride, s))
    else:
        check("bc_compress_rgba16",
              lib.bc_compress_rgba16(variant.id, sp, src.ptr, src.nbytes // 2, dst.ptr, dst.nbytes,
                                     width, height, stride))


__all__ = ["compress_rgba8", "compress_rgba16", "CompressionVariant", "BC6HSettings"]
