"""Decoding entry points mirroring the reference's `decode` module
(src/decode.rs:326-468), executed by the sm_100a kernels.

Host buffers use the synchronous host entry points, CUDA tensors the
stream-ordered device entry point on torch's current stream.
"""
from . import _buffers
from ._lib import check, lib

_FMT = {"rgba8": 0, "rgba16f": 1, "rgba32f": 2}


def _decompress(fmt, variant, width, height, blocks_data, out, esize, host_fn, name, stream):
    src = _buffers.view(blocks_data)
    dst = _buffers.view(out, writable=True)
    if src.cuda != dst.cuda:
        raise ValueError("source and destination must both be host or both be CUDA buffers")
    if src.cuda:
        s = stream if stream is not None else _buffers.current_stream_ptr()
        check("bc_decompress_device",
              lib.bc_decompress_device(variant.id, width, height, src.ptr, src.nbytes, dst.ptr,
                                       dst.nbytes // esize, _FMT[fmt], s))
    else:
        check(name, host_fn(variant.id, width, height, src.ptr, src.nbytes, dst.ptr, dst.nbytes // esize))


def decompress_blocks_as_rgba8(variant, width, height, blocks_data, rgba_data, stream=None):
    """decode::decompress_blocks_as_rgba8 (src/decode.rs:336)."""
    _decompress("rgba8", variant, width, height, blocks_data, rgba_data, 1, lib.bc_decompress_blocks_as_rgba8,
                "bc_decompress_blocks_as_rgba8", stream)


def decompress_blocks_as_rgba16f(variant, width, height, blocks_data, rgba_data, stream=None):
    """decode::decompress_blocks_as_rgba16f (src/decode.rs:397), BC6H only;
    rgba_data holds binary16 values (uint16 / float16 elements)."""
    _decompress("rgba16f", variant, width, height, blocks_data, rgba_data, 2,
                lib.bc_decompress_blocks_as_rgba16f, "bc_decompress_blocks_as_rgba16f", stream)


def decompress_blocks_as_rgba32f(variant, width, height, blocks_data, rgba_data, stream=None):
    """decode::decompress_blocks_as_rgba32f (src/decode.rs:438), BC6H only."""
    _decompress("rgba32f", variant, width, height, blocks_data, rgba_data, 4,
                lib.bc_decompress_blocks_as_rgba32f, "bc_decompress_blocks_as_rgba32f", stream)
