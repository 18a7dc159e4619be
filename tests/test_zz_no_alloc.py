"""The allocation-free BC7 entry point (bc_compress_bc7_device_noalloc).

Callers that may not allocate device memory during an encode -- engines that
budget every byte of GPU memory through their own allocator, frame-critical
threads, processes running with the device nearly full -- use this entry
point; its scratch is a fixed array inside the library. This file checks,
through the C ABI, that it produces the same blocks as the regular entry
point, twice in a row (the array keeps the previous call's contents, which
must not leak into the next result), and that it rejects images whose
scratch would not fit.

Named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu

P, S, U32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32


def _entry_points(bcn):
    lib = ctypes.CDLL(bcn._lib.LIB_PATH)
    noalloc = lib.bc_compress_bc7_device_noalloc
    noalloc.argtypes = [P, P, S, P, S, U32, U32, S, P]
    noalloc.restype = ctypes.c_int
    regular = lib.bc_compress_rgba8_device
    regular.argtypes = [ctypes.c_int, P, P, S, P, S, U32, U32, S, P]
    regular.restype = ctypes.c_int
    return noalloc, regular


def test_noalloc_matches_regular_entry_point_twice(bcn, cuda):
    import torch

    noalloc, regular = _entry_points(bcn)
    cases = [
        (bcn.BC7Settings.alpha_basic(), synthetic.config2_image(seed=31, size=256)),
        (bcn.BC7Settings.opaque_fast(), synthetic.config1_image(seed=32, size=192)),
    ]
    for settings, img in cases:  # two calls in a row, different inputs and settings
        h, w = img.shape[:2]
        src = torch.from_numpy(img).cuda()
        n = (w // 4) * (h // 4) * 16
        want = torch.zeros(n, dtype=torch.uint8, device="cuda")
        got = torch.full((n,), 0xAB, dtype=torch.uint8, device="cuda")
        sp = ctypes.byref(settings)
        assert regular(6, ctypes.cast(sp, P), src.data_ptr(), src.numel(), want.data_ptr(), n, w, h, w * 4,
                       None) == 0
        assert noalloc(sp, src.data_ptr(), src.numel(), got.data_ptr(), n, w, h, w * 4, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_noalloc_rejects_images_beyond_its_scratch(bcn, cuda):
    import torch

    noalloc, _ = _entry_points(bcn)
    s = bcn.BC7Settings.alpha_slow()
    w, h = 2048, 2048  # ~4x the scratch of the largest supported image
    src = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
    dst = torch.zeros((w // 4) * (h // 4) * 16, dtype=torch.uint8, device="cuda")
    assert noalloc(ctypes.byref(s), src.data_ptr(), src.numel(), dst.data_ptr(), dst.numel(), w, h, w * 4,
                   None) == -10
    # the largest advertised size fits with the most scratch-hungry preset,
    # and gives the regular entry point's blocks
    _, regular = _entry_points(bcn)
    w = h = 1024
    img = torch.from_numpy(synthetic.config2_image(seed=33, size=w)).cuda()
    n = (w // 4) * (h // 4) * 16
    want = torch.zeros(n, dtype=torch.uint8, device="cuda")
    got = torch.full((n,), 0xCD, dtype=torch.uint8, device="cuda")
    assert regular(6, ctypes.cast(ctypes.byref(s), P), img.data_ptr(), img.numel(), want.data_ptr(), n, w, h, w * 4,
                   None) == 0
    assert noalloc(ctypes.byref(s), img.data_ptr(), img.numel(), got.data_ptr(), n, w, h, w * 4, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(got, want)
