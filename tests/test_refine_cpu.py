"""Relaxed (differentiable) BC1/BC7 decode and endpoint refinement: the CPU
restatement in the oracle, checked against the pinned oracle decoders and
against finite differences. These pin the checker the GPU tests use."""
import numpy as np
import pytest

from block_compression_b200 import synthetic
from block_compression_b200.settings import BC7Settings


def random_bc7_blocks(rng, per_mode=64):
    """Random 16-byte blocks with the mode prefix forced to each of modes 0-7
    (every bit pattern after the prefix is a valid block of that mode), plus
    reserved-encoding blocks (first byte 0)."""
    out = []
    for mode in range(8):
        b = rng.integers(0, 256, size=(per_mode, 16), dtype=np.uint8)
        b[:, 0] = (b[:, 0] & ~np.uint8((1 << (mode + 1)) - 1)) | np.uint8(1 << mode)
        out.append(b)
    r = rng.integers(0, 256, size=(4, 16), dtype=np.uint8)
    r[:, 0] = 0
    out.append(r)
    return np.concatenate(out)


def test_bc7_parse_roundtrip_equals_decoder(oracle_lib):
    rng = np.random.default_rng(11)
    blocks = random_bc7_blocks(rng)
    meta, ep = oracle_lib.parse("bc7", blocks)
    assert np.bincount(meta[:, 0] & 15, minlength=9).tolist() == [64] * 8 + [4]
    rel = oracle_lib.relaxed_f64("bc7", meta, ep)
    for i, blk in enumerate(blocks):
        dec = np.zeros(64, dtype=np.uint8)
        oracle_lib.decode_block("bc7", blk, dec, 16)
        assert np.array_equal(np.floor(rel[i] + 0.5).reshape(-1).astype(np.int64), dec.astype(np.int64)), i


@pytest.mark.parametrize("preset", ["alpha_basic", "opaque_basic"])
def test_bc7_encoded_roundtrip(oracle_lib, preset):
    img = synthetic.config2_image(2, 64)
    blocks = oracle_lib.compress_rgba8(6, img, 64, 64, settings=getattr(BC7Settings, preset)().as_list())
    meta, ep = oracle_lib.parse("bc7", blocks)
    rel = oracle_lib.relaxed_f64("bc7", meta, ep)
    dec = oracle_lib.image_blocks(oracle_lib.decompress_rgba8(6, blocks, 64, 64), 64, 64)
    assert np.array_equal(np.floor(rel + 0.5), dec.astype(np.float64))


def test_bc1_parse_roundtrip_within_one(oracle_lib):
    """BC1's decoder interpolates the 5/6-bit values with its own integer
    formula, so the relaxed decode rounds to within one step of it; indices 0
    and 1 (the endpoints) and the three-colour black texel are exact."""
    rng = np.random.default_rng(3)
    blocks = rng.integers(0, 256, size=(512, 8), dtype=np.uint8)
    meta, ep = oracle_lib.parse("bc1", blocks)
    rel = oracle_lib.relaxed_f64("bc1", meta, ep)
    for i, blk in enumerate(blocks):
        dec = np.zeros(64, dtype=np.uint8)
        oracle_lib.decode_block("bc1", blk, dec, 16)
        d = np.abs(np.floor(rel[i] + 0.5).reshape(16, 4) - dec.reshape(16, 4))
        idx = (int(meta[i, 1]) >> (2 * np.arange(16))) & 3
        assert d.max() <= 1
        assert d[idx < 2].max() == 0


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_oracle_adjoint_matches_finite_differences(oracle_lib, kind):
    rng = np.random.default_rng(5)
    blocks = random_bc7_blocks(rng, 16) if kind == "bc7" else rng.integers(0, 256, size=(128, 8), dtype=np.uint8)
    meta, ep = oracle_lib.parse(kind, blocks)
    theta = ep.astype(np.float64) + rng.uniform(-4, 4, size=ep.shape)
    src = rng.integers(0, 256, size=(len(meta), 16, 4)).astype(np.float64)

    def loss(t):
        return ((oracle_lib.relaxed_f64(kind, meta, t) - src) ** 2).sum(axis=(1, 2))

    g = oracle_lib.adjoint_f64(kind, meta, 2.0 * (oracle_lib.relaxed_f64(kind, meta, theta) - src))
    eps = 1e-3
    fd = np.zeros_like(theta)
    for j in range(theta.shape[1]):
        e = np.zeros_like(theta)
        e[:, j] = eps
        fd[:, j] = (loss(theta + e) - loss(theta - e)) / (2 * eps)
    np.testing.assert_allclose(g, fd, rtol=1e-7, atol=1e-6)


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_oracle_refine_never_worse(oracle_lib, kind):
    img = synthetic.config1_image(1, 64)
    if kind == "bc7":
        blocks = oracle_lib.compress_rgba8(6, img, 64, 64, settings=BC7Settings.opaque_basic().as_list())
    else:
        blocks = oracle_lib.compress_rgba8(0, img, 64, 64)
    src = oracle_lib.image_blocks(img, 64, 64)
    out, theta, errs = oracle_lib.refine_blocks(kind, blocks, src, 20, 0.5, 3)
    assert (errs[:, 1] <= errs[:, 0]).all()
    assert (errs[:, 1] < errs[:, 0]).sum() > 0
    bsz = 16 if kind == "bc7" else 8
    changed = (out != blocks.reshape(-1, bsz)).any(axis=1)
    assert np.array_equal(changed, errs[:, 1] < errs[:, 0])
    # the recorded error is the decoded block's exact error
    variant = 6 if kind == "bc7" else 0
    dec = oracle_lib.image_blocks(oracle_lib.decompress_rgba8(variant, out.reshape(-1), 64, 64), 64, 64)
    exact = ((dec[..., :3].astype(np.int64) - src[..., :3]) ** 2).sum(axis=(1, 2))
    assert np.array_equal(exact, errs[:, 1].astype(np.int64))
    # zero steps change nothing
    out0, _, errs0 = oracle_lib.refine_blocks(kind, blocks, src, 0, 0.5, 3)
    assert np.array_equal(out0, blocks.reshape(-1, bsz)) and np.array_equal(errs0[:, 0], errs0[:, 1])
