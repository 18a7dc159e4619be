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


# ---- per-block decoders (src/decode/block.rs:50-119, 262, 774, 801) ----------

BLOCK_KINDS = {"bc1": 0, "bc2": 1, "bc3": 2, "bc4": 3, "bc5": 4, "bc6h": 5, "bc6h_float": 6, "bc7": 7}
_BLOCK_ELEM = {"bc6h": 2, "bc6h_float": 4}


def block_min_len(kind, destination_pitch):
    """Output elements the reference's decode_block_<kind> needs at this pitch."""
    return lib.bc_decode_block_min_len(BLOCK_KINDS[kind], destination_pitch)


def _decode_block(kind, compressed_block, decompressed_block, destination_pitch, is_signed=False):
    src = _buffers.view(compressed_block)
    dst = _buffers.view(decompressed_block, writable=True)
    if src.cuda != dst.cuda:
        raise ValueError("source and destination must both be host or both be CUDA buffers")
    esize = _BLOCK_ELEM.get(kind, 1)
    if src.cuda:
        decode_blocks(kind, compressed_block, decompressed_block, destination_pitch, 0, 1, is_signed)
        return
    if kind.startswith("bc6h"):
        fn = getattr(lib, "bc_decode_block_" + kind)
        check("bc_decode_block_" + kind,
              fn(src.ptr, src.nbytes, dst.ptr, dst.nbytes // esize, destination_pitch, int(bool(is_signed))))
    else:
        fn = getattr(lib, "bc_decode_block_" + kind)
        check("bc_decode_block_" + kind, fn(src.ptr, src.nbytes, dst.ptr, dst.nbytes, destination_pitch))


def decode_block_bc1(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc1 (src/decode/block.rs:50): RGBA8 rows `destination_pitch` bytes apart."""
    _decode_block("bc1", compressed_block, decompressed_block, destination_pitch)


def decode_block_bc2(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc2 (src/decode/block.rs:61)."""
    _decode_block("bc2", compressed_block, decompressed_block, destination_pitch)


def decode_block_bc3(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc3 (src/decode/block.rs:76)."""
    _decode_block("bc3", compressed_block, decompressed_block, destination_pitch)


def decode_block_bc4(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc4 (src/decode/block.rs:95): R8 texels."""
    _decode_block("bc4", compressed_block, decompressed_block, destination_pitch)


def decode_block_bc5(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc5 (src/decode/block.rs:106): RG8 texels."""
    _decode_block("bc5", compressed_block, decompressed_block, destination_pitch)


def decode_block_bc6h(compressed_block, decompressed_block, destination_pitch, is_signed):
    """decode::decode_block_bc6h (src/decode/block.rs:262): RGB binary16
    triplets (uint16 / float16 elements), rows `destination_pitch` elements apart."""
    _decode_block("bc6h", compressed_block, decompressed_block, destination_pitch, is_signed)


def decode_block_bc6h_float(compressed_block, decompressed_block, destination_pitch, is_signed):
    """decode::decode_block_bc6h_float (src/decode/block.rs:774): RGB f32 triplets."""
    _decode_block("bc6h_float", compressed_block, decompressed_block, destination_pitch, is_signed)


def decode_block_bc7(compressed_block, decompressed_block, destination_pitch):
    """decode::decode_block_bc7 (src/decode/block.rs:801)."""
    _decode_block("bc7", compressed_block, decompressed_block, destination_pitch)


def decode_blocks(kind, blocks, out, destination_pitch, out_block_stride, nblocks=None, is_signed=False,
                  stream=None):
    """Device form of the per-block decoders: `nblocks` consecutive blocks of
    CUDA memory, block i written from element i * out_block_stride of `out`
    (a CUDA buffer), stream-ordered on torch's current stream."""
    src = _buffers.view(blocks)
    dst = _buffers.view(out, writable=True)
    if not (src.cuda and dst.cuda):
        raise ValueError("decode_blocks takes CUDA buffers")
    bsz = 8 if kind in ("bc1", "bc4") else 16
    n = src.nbytes // bsz if nblocks is None else nblocks
    if n * bsz > src.nbytes:
        check("bc_decode_blocks_device", -3)
    s = stream if stream is not None else _buffers.current_stream_ptr()
    check("bc_decode_blocks_device",
          lib.bc_decode_blocks_device(BLOCK_KINDS[kind], int(bool(is_signed)), src.ptr, n, dst.ptr,
                                      dst.nbytes // _BLOCK_ELEM.get(kind, 1), destination_pitch, out_block_stride, s))
