"""GPU mip-chain generation (box filter) feeding the batched encoder.

Each level is written padded up to whole 4x4 blocks by edge replication, so
every level can be added as a compression task directly.
"""
from . import _buffers
from ._lib import check, lib


class MipLevel:
    __slots__ = ("data", "width", "height")

    def __init__(self, data, width, height):
        self.data = data      # CUDA uint8 tensor (padded_h, padded_w, 4)
        self.width = width    # valid size of the level
        self.height = height

    @property
    def padded_width(self):
        return self.data.shape[1]

    @property
    def padded_height(self):
        return self.data.shape[0]


def generate_mip_chain(texture, stream=None):
    """texture: CUDA uint8 tensor (h, w, 4) with h, w multiples of 4. Returns
    the full chain down to 1x1 as MipLevel objects (level 0 = the input)."""
    import torch

    h, w = int(texture.shape[0]), int(texture.shape[1])
    if h % 4 or w % 4:
        raise ValueError("level 0 must be a multiple of 4 in both dimensions")
    s = stream if stream is not None else _buffers.current_stream_ptr()
    levels = [MipLevel(texture, w, h)]
    while levels[-1].width > 1 or levels[-1].height > 1:
        prev = levels[-1]
        dw, dh = max(1, prev.width // 2), max(1, prev.height // 2)
        pw, ph = (dw + 3) & ~3, (dh + 3) & ~3
        out = torch.empty((ph, pw, 4), dtype=torch.uint8, device=texture.device)
        check("bc_mip_level_rgba8_device",
              lib.bc_mip_level_rgba8_device(prev.data.data_ptr(), prev.padded_width * 4, prev.width, prev.height,
                                            out.data_ptr(), pw * 4, out.numel(), s))
        levels.append(MipLevel(out, dw, dh))
    return levels
