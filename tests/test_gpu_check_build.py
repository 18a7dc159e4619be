"""The bounds-checked debug build on the GPU: the encoders and decoders of
libbcn_b200_check.so give the release library's bytes with no guard firing,
and a guard that sees an index outside its extent (the self-test launch,
which accesses no memory) is reported with its site, index and extent."""
import ctypes
import os

import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
P, S, U32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32


@pytest.fixture(scope="module")
def check_lib():
    path = os.path.join(ROOT, "block_compression_b200", "libbcn_b200_check.so")
    if not os.path.exists(path):
        pytest.fail("libbcn_b200_check.so is not built (build() makes it)")
    L = ctypes.CDLL(path)
    L.bc_compress_rgba8_device.argtypes = [ctypes.c_int, P, P, S, P, S, U32, U32, S, P]
    L.bc_compress_rgba16_device.argtypes = [P, P, S, P, S, U32, U32, S, P]
    L.bc_decompress_device.argtypes = [ctypes.c_int, U32, U32, P, S, P, S, ctypes.c_int, P]
    L.bc_check_read.argtypes = [P]
    L.bc_check_selftest.argtypes = [ctypes.c_uint64, ctypes.c_uint64, P]
    assert L.bc_check_enabled() == 1
    return L


def _read(L):
    out = (ctypes.c_uint64 * 3)()
    assert L.bc_check_read(out) == 0
    return list(out)


def test_checked_kernels_match_release_and_record_nothing(bcn, check_lib, cuda):
    import torch
    L = check_lib
    _read(L)  # clear
    w = h = 256
    img = torch.from_numpy(synthetic.config2_image(seed=41, size=w)).cuda()
    V = bcn.CompressionVariant
    s7 = bcn.BC7Settings.alpha_basic()
    for v in (V.BC1, V.BC2, V.BC3, V.BC4, V.BC5, V.BC7(s7)):
        n = v.blocks_byte_size(w, h)
        want = torch.zeros(n, dtype=torch.uint8, device="cuda")
        got = torch.zeros(n, dtype=torch.uint8, device="cuda")
        bcn.encode.compress_rgba8(v, img, want, w, h, w * 4)
        sp = v.settings_ptr()
        assert L.bc_compress_rgba8_device(v.id, sp, img.data_ptr(), img.numel(), got.data_ptr(), n, w, h, w * 4,
                                          None) == 0
        dec_want = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
        dec_got = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
        bcn.decode.decompress_blocks_as_rgba8(v, w, h, want, dec_want)
        assert L.bc_decompress_device(v.id, w, h, got.data_ptr(), n, dec_got.data_ptr(), w * h * 4, 0, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, want), v
        assert torch.equal(dec_got, dec_want), v
    hdr = torch.from_numpy(synthetic.config3_hdr(seed=42, size=128).view(np.int16)).cuda()
    s6 = bcn.BC6HSettings.basic()
    v6 = V.BC6H(s6)
    n = v6.blocks_byte_size(128, 128)
    want = torch.zeros(n, dtype=torch.uint8, device="cuda")
    got = torch.zeros(n, dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba16(v6, hdr, want, 128, 128, 128 * 4)
    assert L.bc_compress_rgba16_device(ctypes.byref(s6), hdr.data_ptr(), hdr.numel(), got.data_ptr(), n, 128, 128,
                                       128 * 4, None) == 0
    dec = torch.zeros(128 * 128 * 4, dtype=torch.int16, device="cuda")
    assert L.bc_decompress_device(5, 128, 128, got.data_ptr(), n, dec.data_ptr(), dec.numel(), 1, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    assert _read(L) == [0, 0, 0]


def test_failed_guard_is_recorded_not_trapped(check_lib, cuda):
    import torch
    L = check_lib
    _read(L)
    assert L.bc_check_selftest(3, 4, None) == 0  # inside: nothing recorded
    torch.cuda.synchronize()
    assert _read(L) == [0, 0, 0]
    assert L.bc_check_selftest(9, 4, None) == 0  # outside
    torch.cuda.synchronize()
    assert _read(L) == [11, 9, 4]  # site CHECK_SELFTEST, index, extent
    assert _read(L) == [0, 0, 0]   # reading clears
    # the context is still usable
    x = torch.ones(16, device="cuda")
    assert float(x.sum()) == 16.0
