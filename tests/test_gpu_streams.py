"""The device BC7 path forks its stage chains onto library-owned streams and
joins them back into the caller's stream. Work the caller orders after the
call on its own stream -- here a device-to-host copy on a non-default
stream, and a second encode reusing the scratch pool -- must see the
finished blocks."""
import numpy as np
import pytest
import torch

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_bc7_on_user_stream_is_ordered_before_later_work(bcn, oracle_lib, cuda):
    size = 256
    s7 = bcn.BC7Settings.alpha_basic()
    v = bcn.CompressionVariant.BC7(s7)
    img_a = synthetic.config2_image(seed=4, size=size)
    img_b = synthetic.config2_image(seed=5, size=size)
    exp_a = oracle_lib.compress_rgba8(v.id, img_a, size, size, settings=s7.as_list())
    exp_b = oracle_lib.compress_rgba8(v.id, img_b, size, size, settings=s7.as_list())
    nbytes = v.blocks_byte_size(size, size)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        src_a = torch.from_numpy(img_a).cuda()
        src_b = torch.from_numpy(img_b).cuda()
        dst_a = torch.full((nbytes,), 0xAB, dtype=torch.uint8, device="cuda")
        dst_b = torch.full((nbytes,), 0xAB, dtype=torch.uint8, device="cuda")
        for _ in range(3):
            bcn.encode.compress_rgba8(v, src_a, dst_a, size, size, size * 4)
            bcn.encode.compress_rgba8(v, src_b, dst_b, size, size, size * 4)
            host_a = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
            host_b = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
            host_a.copy_(dst_a, non_blocking=True)
            host_b.copy_(dst_b, non_blocking=True)
            stream.synchronize()
            assert np.array_equal(host_a.numpy(), exp_a)
            assert np.array_equal(host_b.numpy(), exp_b)
            dst_a.fill_(0xAB)
            dst_b.fill_(0xAB)
