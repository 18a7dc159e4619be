"""DDS container output, as the reference's example CLI writes it
(compressor/src/main.rs:313-353): a DX10-extended header for one 2D texture
with straight alpha, then the block data of each mip level, largest first."""
import ctypes

from ._lib import check, lib

HEADER_BYTES = 148


def dxgi_format(variant, srgb=True):
    """DXGI format of a variant: the reference CLI's mapping (_SRGB for
    BC1/BC2/BC3/BC7, UNORM for BC4/BC5, UF16 for BC6H) when srgb is True."""
    return int(lib.bc_dds_dxgi_format(variant.id, 1 if srgb else 0))


def dds_header(variant, width, height, mip_levels=1, srgb=True):
    buf = (ctypes.c_uint8 * HEADER_BYTES)()
    check("bc_dds_header", lib.bc_dds_header(variant.id, width, height, mip_levels, 1 if srgb else 0,
                                             ctypes.addressof(buf), HEADER_BYTES))
    return bytes(buf)


def write_dds(path, variant, width, height, levels, srgb=True):
    """Writes `levels` (a list of block buffers -- bytes, numpy arrays or
    tensors -- one per mip level, largest first) as a DDS file."""
    import numpy as np

    with open(path, "wb") as f:
        f.write(dds_header(variant, width, height, len(levels), srgb))
        for lv in levels:
            if hasattr(lv, "cpu"):
                lv = lv.cpu().numpy()
            f.write(np.ascontiguousarray(lv, dtype=np.uint8).tobytes())
    return path
