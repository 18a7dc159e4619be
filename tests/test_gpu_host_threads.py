"""The host-buffer entry points from several host threads at once (as the
benchmark's end-to-end step and an application encoding several textures
use them): each thread's blocks equal the single-threaded encode's. The
library keeps its staging buffers and streams per thread, so the calls
overlap on the GPU."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_concurrent_host_encodes_match_serial(bcn, cuda):
    import torch
    V = bcn.CompressionVariant
    jobs = [(V.BC7(bcn.BC7Settings.alpha_basic()), synthetic.config2_image(seed=51, size=512)),
            (V.BC3, synthetic.config2_image(seed=52, size=512)),
            (V.BC1, synthetic.config1_image(seed=53, size=512)),
            (V.BC5, synthetic.normal_map(seed=54, size=512)),
            (V.BC7(bcn.BC7Settings.opaque_fast()), synthetic.config1_image(seed=55, size=256))]

    def encode(job):
        v, img = job
        h, w = img.shape[:2]
        torch.cuda.set_device(0)
        out = np.zeros(v.blocks_byte_size(w, h), np.uint8)
        bcn.encode.compress_rgba8(v, img, out, w, h, w * 4)
        return out

    serial = [encode(j) for j in jobs]
    with ThreadPoolExecutor(len(jobs)) as ex:
        for _ in range(3):
            parallel = list(ex.map(encode, jobs))
            for a, b in zip(serial, parallel):
                assert np.array_equal(a, b)
