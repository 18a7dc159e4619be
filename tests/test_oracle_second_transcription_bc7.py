"""Pins the BC7 half of the C++ oracle -- mode orchestration, candidate
lists, tie-breaking, the mode-4/5 rotations and scalar channel, and the bit
coding -- with a second, independent transcription of the reference BC7
encoder (oracle/numpy_bc7.py, written in numpy from src/encode/bc7.rs and
src/encode/common.rs:520-613): every block of every preset must agree bit for
bit, on the alpha-texture generator, uniform noise, hand-picked edge blocks
and a crop of the reference's own brick-alpha image. CPU only."""
import numpy as np
import pytest

import reference_images as ri
from block_compression_b200 import synthetic

PRESETS = ["opaque_ultra_fast", "opaque_very_fast", "opaque_fast", "opaque_basic", "opaque_slow",
           "alpha_ultrafast", "alpha_very_fast", "alpha_fast", "alpha_basic", "alpha_slow"]


def _images():
    from test_gpu_parity import _edge_blocks
    rng = np.random.default_rng(5)
    return {"alpha_texture": synthetic.config2_image(seed=21, size=64),
            "noise": rng.integers(0, 256, (32, 64, 4), dtype=np.uint8),
            "edge": _edge_blocks(np.random.default_rng(7)),
            "brick_alpha": np.ascontiguousarray(ri.load("brick-alpha")[:32, :64])}


@pytest.mark.parametrize("preset", PRESETS)
def test_bc7_encoder_matches_second_transcription(bcn, oracle_lib, preset):
    from oracle import numpy_bc7
    s = getattr(bcn.BC7Settings, preset)().as_list()
    for name, img in _images().items():
        h, w = img.shape[:2]
        with np.errstate(all="ignore"):
            got = numpy_bc7.compress_bc7(img, s)
        exp = oracle_lib.compress_rgba8(6, img, w, h, settings=s)
        bad = np.nonzero((got.reshape(-1, 16) != exp.reshape(-1, 16)).any(1))[0]
        assert bad.size == 0, "%s on %s: %d blocks differ, first %s" % (preset, name, bad.size, bad[:5].tolist())
