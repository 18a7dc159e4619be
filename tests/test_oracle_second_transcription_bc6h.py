"""Pins the BC6H half of the C++ oracle -- the mode tests and their margins,
the quantisation bounds, the 2-region partition search and refinement, the
1-region encode and the per-mode endpoint packing -- with a second,
independent transcription of the reference BC6H encoder
(oracle/numpy_bc6h.py, written in numpy from src/encode/bc6h.rs): every block
of every preset must agree bit for bit on the HDR workload's generator,
random f16 bit patterns (infinities and NaN codes included), flat blocks and
two-level blocks. CPU only."""
import numpy as np
import pytest

from block_compression_b200 import synthetic

PRESETS = ["very_fast", "fast", "basic", "slow", "very_slow"]


def _images():
    rng = np.random.default_rng(9)
    flat = rng.integers(0, 0x7C00, (8, 16, 1, 1, 4)).astype(np.uint16)
    flat = np.repeat(np.repeat(flat, 4, axis=2), 4, axis=3).transpose(0, 2, 1, 3, 4).reshape(32, 64, 4)
    two = np.where(rng.random((32, 64, 1)) < 0.5, np.uint16(0x3C00), np.uint16(0x5000)).repeat(4, 2)
    return {"hdr": synthetic.config3_hdr(seed=3, size=64).view(np.uint16),
            "random_bits": rng.integers(0, 65536, (32, 64, 4)).astype(np.uint16),
            "flat": np.ascontiguousarray(flat), "two_level": np.ascontiguousarray(two.astype(np.uint16))}


@pytest.mark.parametrize("preset", PRESETS)
def test_bc6h_encoder_matches_second_transcription(bcn, oracle_lib, preset):
    from oracle import numpy_bc6h
    s = getattr(bcn.BC6HSettings, preset)().as_list()
    for name, img in _images().items():
        h, w = img.shape[:2]
        with np.errstate(all="ignore"):
            got = numpy_bc6h.compress_bc6h(img, s)
        exp = oracle_lib.compress_rgba16(img, w, h, s)
        bad = np.nonzero((got.reshape(-1, 16) != exp.reshape(-1, 16)).any(1))[0]
        assert bad.size == 0, "%s on %s: %d blocks differ, first %s" % (preset, name, bad.size, bad[:5].tolist())
