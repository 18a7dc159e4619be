"""Differentiable BC1/BC7 decode and gradient endpoint refinement (no
counterpart in the reference crate).

The relaxed decode treats a block's endpoints as continuous values in 8-bit
units with its mode, partition, rotation, index selector and indices fixed:
`c = e0 + (e1 - e0) * w / 64` for BC7 (w the BPTC index weight), and
`c = e0 + (e1 - e0) * t` with t = 0, 1, 1/3, 2/3 (four-colour) or 0, 1, 1/2
and transparent black (three-colour) for BC1. Parsed endpoints reproduce the
decoder exactly after rounding (floor(c + 0.5)).

All tensors are CUDA tensors; calls run on torch's current stream.
  parse_bc7(blocks)              -> (meta int32 (n, 8), endpoints float32 (n, 24))
  decode_relaxed_bc7(meta, ep)   -> float32 (n, 16, 4)
  decode_adjoint_bc7(meta, grad) -> float32 (n, 24)
  parse_bc1 / decode_relaxed_bc1 / decode_adjoint_bc1: the same with
    meta (n, 2) and endpoints (n, 6).
  refine_bc7(src, blocks, ...) / refine_bc1(src, blocks, ...): Adam endpoint
    refinement in place; a block is replaced only if its exact error drops.
"""
import ctypes

from . import _buffers
from ._lib import check, lib


def _torch():
    import torch
    return torch


def _cuda_contig(t, name, dtype=None):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("%s must be a CUDA tensor" % name)
    if dtype is not None and t.dtype != dtype:
        raise TypeError("%s must be %s" % (name, dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    return t


def _nblocks(blocks, block_bytes):
    n = blocks.numel() * blocks.element_size()
    if n % block_bytes:
        raise ValueError("blocks buffer is not a whole number of %d-byte blocks" % block_bytes)
    return n // block_bytes


def _stream():
    return _buffers.current_stream_ptr()


def parse_bc7(blocks):
    torch = _torch()
    _cuda_contig(blocks, "blocks")
    n = _nblocks(blocks, 16)
    meta = torch.empty((n, 8), dtype=torch.int32, device=blocks.device)
    ep = torch.empty((n, 24), dtype=torch.float32, device=blocks.device)
    check("bc_bc7_parse_device", lib.bc_bc7_parse_device(blocks.data_ptr(), n, meta.data_ptr(), ep.data_ptr(),
                                                         _stream()))
    return meta, ep


def decode_relaxed_bc7(meta, endpoints):
    torch = _torch()
    _cuda_contig(meta, "meta", torch.int32)
    _cuda_contig(endpoints, "endpoints", torch.float32)
    n = meta.shape[0]
    if tuple(meta.shape) != (n, 8) or tuple(endpoints.shape) != (n, 24):
        raise ValueError("meta must be (n, 8) and endpoints (n, 24)")
    out = torch.empty((n, 16, 4), dtype=torch.float32, device=meta.device)
    check("bc_bc7_decode_relaxed_device",
          lib.bc_bc7_decode_relaxed_device(meta.data_ptr(), endpoints.data_ptr(), n, out.data_ptr(), _stream()))
    return out


def decode_adjoint_bc7(meta, grad_out):
    torch = _torch()
    _cuda_contig(meta, "meta", torch.int32)
    _cuda_contig(grad_out, "grad_out", torch.float32)
    n = meta.shape[0]
    if tuple(grad_out.shape) != (n, 16, 4):
        raise ValueError("grad_out must be (n, 16, 4)")
    gep = torch.empty((n, 24), dtype=torch.float32, device=meta.device)
    check("bc_bc7_decode_adjoint_device",
          lib.bc_bc7_decode_adjoint_device(meta.data_ptr(), grad_out.data_ptr(), n, gep.data_ptr(), _stream()))
    return gep


def parse_bc1(blocks):
    torch = _torch()
    _cuda_contig(blocks, "blocks")
    n = _nblocks(blocks, 8)
    meta = torch.empty((n, 2), dtype=torch.int32, device=blocks.device)
    ep = torch.empty((n, 6), dtype=torch.float32, device=blocks.device)
    check("bc_bc1_parse_device", lib.bc_bc1_parse_device(blocks.data_ptr(), n, meta.data_ptr(), ep.data_ptr(),
                                                         _stream()))
    return meta, ep


def decode_relaxed_bc1(meta, endpoints):
    torch = _torch()
    _cuda_contig(meta, "meta", torch.int32)
    _cuda_contig(endpoints, "endpoints", torch.float32)
    n = meta.shape[0]
    if tuple(meta.shape) != (n, 2) or tuple(endpoints.shape) != (n, 6):
        raise ValueError("meta must be (n, 2) and endpoints (n, 6)")
    out = torch.empty((n, 16, 4), dtype=torch.float32, device=meta.device)
    check("bc_bc1_decode_relaxed_device",
          lib.bc_bc1_decode_relaxed_device(meta.data_ptr(), endpoints.data_ptr(), n, out.data_ptr(), _stream()))
    return out


def decode_adjoint_bc1(meta, grad_out):
    torch = _torch()
    _cuda_contig(meta, "meta", torch.int32)
    _cuda_contig(grad_out, "grad_out", torch.float32)
    n = meta.shape[0]
    if tuple(grad_out.shape) != (n, 16, 4):
        raise ValueError("grad_out must be (n, 16, 4)")
    gep = torch.empty((n, 6), dtype=torch.float32, device=meta.device)
    check("bc_bc1_decode_adjoint_device",
          lib.bc_bc1_decode_adjoint_device(meta.data_ptr(), grad_out.data_ptr(), n, gep.data_ptr(), _stream()))
    return gep


class RefineStats:
    __slots__ = ("blocks", "replaced", "err_before", "err_after")

    def __init__(self, vals):
        self.blocks, self.replaced, self.err_before, self.err_after = (int(v) for v in vals)

    def as_dict(self):
        return {k: getattr(self, k) for k in self.__slots__}


def _refine(kind, src, blocks, width, height, stride, steps, lr, channels, want_endpoints, stats):
    torch = _torch()
    _cuda_contig(src, "src")
    _cuda_contig(blocks, "blocks")
    h = int(src.shape[0]) if height is None else int(height)
    w = int(src.shape[1]) if width is None else int(width)
    stride = w * 4 if stride is None else int(stride)
    n = (w // 4) * (h // 4)
    per = 24 if kind == "bc7" else 6
    ep_out = torch.empty((n, per), dtype=torch.float32, device=blocks.device) if want_endpoints else None
    own_stats = stats is None
    if own_stats:
        stats = torch.zeros(4, dtype=torch.int64, device=blocks.device)
    args = (src.data_ptr(), stride, w, h, blocks.data_ptr(), blocks.numel() * blocks.element_size())
    tail = (stats.data_ptr(), ep_out.data_ptr() if ep_out is not None else None, _stream())
    if kind == "bc7":
        check("bc_bc7_refine_device", lib.bc_bc7_refine_device(*args, channels, steps, float(lr), *tail))
    else:
        check("bc_bc1_refine_device", lib.bc_bc1_refine_device(*args, steps, float(lr), *tail))
    result = RefineStats(stats.cpu().tolist()) if own_stats else None
    return (result, ep_out) if want_endpoints else result


class _Image(ctypes.Structure):
    _fields_ = [("src", ctypes.c_void_p), ("src_stride", ctypes.c_size_t), ("width", ctypes.c_uint32),
                ("height", ctypes.c_uint32), ("blocks", ctypes.c_void_p), ("blocks_len", ctypes.c_size_t),
                ("endpoints_out", ctypes.c_void_p)]


def _refine_many(kind, images, steps, lr, channels, stats):
    """images: list of (src (h, w, 4) CUDA uint8, blocks CUDA uint8)."""
    torch = _torch()
    arr = (_Image * len(images))()
    for e, (src, blocks) in zip(arr, images):
        _cuda_contig(src, "src")
        _cuda_contig(blocks, "blocks")
        e.src, e.src_stride = src.data_ptr(), int(src.shape[1]) * 4
        e.width, e.height = int(src.shape[1]), int(src.shape[0])
        e.blocks, e.blocks_len = blocks.data_ptr(), blocks.numel() * blocks.element_size()
        e.endpoints_out = None
    own = stats is None
    if own:
        dev = images[0][1].device if images else "cuda"
        stats = torch.zeros(4, dtype=torch.int64, device=dev)
    if kind == "bc7":
        check("bc_bc7_refine_images_device", lib.bc_bc7_refine_images_device(
            ctypes.addressof(arr), len(images), channels, steps, float(lr), stats.data_ptr(), _stream()))
    else:
        check("bc_bc1_refine_images_device", lib.bc_bc1_refine_images_device(
            ctypes.addressof(arr), len(images), steps, float(lr), stats.data_ptr(), _stream()))
    return RefineStats(stats.cpu().tolist()) if own else None


def refine_bc7_images(images, channels=4, steps=20, lr=0.5, stats=None):
    """refine_bc7 over a list of (src, blocks) pairs in as few launches as
    possible (16 images per launch)."""
    return _refine_many("bc7", images, steps, lr, channels, stats)


def refine_bc1_images(images, steps=20, lr=0.5, stats=None):
    return _refine_many("bc1", images, steps, lr, 3, stats)


def refine_bc7(src, blocks, channels=4, steps=20, lr=0.5, width=None, height=None, stride=None,
               return_endpoints=False, stats=None):
    """Refines BC7 `blocks` (CUDA uint8, row-major blocks of the image) in
    place against the RGBA8 source `src` (CUDA uint8 (h, w, 4) or a flat
    buffer with width/height/stride given). channels: 3 = RGB error, 4 = RGBA
    (use the BC7 settings' channel count). Returns RefineStats (synchronises),
    or nothing when a caller-owned int64[4] `stats` tensor accumulates them."""
    return _refine("bc7", src, blocks, width, height, stride, steps, lr, channels, return_endpoints, stats)


def refine_bc1(src, blocks, steps=20, lr=0.5, width=None, height=None, stride=None, return_endpoints=False,
               stats=None):
    """BC1 counterpart of refine_bc7 (RGB error)."""
    return _refine("bc1", src, blocks, width, height, stride, steps, lr, 3, return_endpoints, stats)
