"""Pins the encoder half of the C++ oracle with a second, independent
transcription of the reference (oracle/numpy_restatement.py, written in numpy
from the Rust sources): the two must agree bit for bit on ~10^4 random blocks
per function -- BC1 compress_block_bc1_core and BC3 compress_block_bc3_alpha
(src/encode/bc1_to_5.rs:157-472), whole-image BC1-BC5 encodes
(src/encode.rs:259-500), and the BC7/BPTC primitives block_quant,
opt_endpoints, block_pca_bound_split, block_segment_core
(src/encode/common.rs:142-518) and ep_quant_dequant (src/encode/bc7.rs:97-237).
A mistranscription in either restatement shows up as a difference. CPU only.
"""
import ctypes

import numpy as np
import pytest

from oracle import numpy_restatement as nr

N = 10000


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _blocks(rng, n, alpha=True):
    """Planar float32 blocks of byte values: uniform noise, smooth ramps,
    2-4 colour blocks, flat blocks and near-flat blocks (the degenerate
    branches of the encoders)."""
    kinds = rng.integers(0, 5, n)
    px = rng.integers(0, 256, (n, 16, 4)).astype(np.float64)
    t = np.linspace(0, 1, 16)[None, :, None]
    a, b = rng.integers(0, 256, (n, 1, 4)), rng.integers(0, 256, (n, 1, 4))
    ramp = np.round(a + (b - a) * t)
    pal = rng.integers(0, 256, (n, 4, 4))
    sel = rng.integers(0, rng.integers(2, 5, n)[:, None], (n, 16))
    few = np.take_along_axis(pal, sel[..., None].repeat(4, -1), 1)
    flat = np.repeat(a, 16, 1)
    near = np.clip(flat + rng.integers(-1, 2, (n, 16, 4)), 0, 255)
    out = np.select([kinds[:, None, None] == k for k in range(5)], [px, ramp, few, flat, near])
    if not alpha:
        out[..., 3] = 255
    return np.ascontiguousarray(out.transpose(0, 2, 1).reshape(n, 64)).astype(np.float32)


def _bits_equal(a, b):
    a, b = np.asarray(a, np.float32), np.asarray(b, np.float32)
    return np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_bc1_core_and_bc3_alpha(oracle_lib):
    rng = np.random.default_rng(11)
    blk = _blocks(rng, N)
    got1, got3 = nr.bc1_core(blk), nr.bc3_alpha(blk)
    L = oracle_lib.lib()
    exp1 = np.zeros((N, 2), np.uint32)
    exp3 = np.zeros((N, 2), np.uint32)
    for i in range(N):
        b = np.ascontiguousarray(blk[i])
        L.oracle_encode_block_bc1(_ptr(b), _ptr(exp1[i]))
        L.oracle_encode_block_bc3_alpha(_ptr(b), _ptr(exp3[i]))
    assert np.array_equal(got1, exp1), np.nonzero((got1 != exp1).any(1))[0][:10]
    assert np.array_equal(got3, exp3), np.nonzero((got3 != exp3).any(1))[0][:10]


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_whole_image_bc1_to_bc5(oracle_lib, variant):
    from block_compression_b200 import synthetic
    rng = np.random.default_rng(12)
    imgs = [synthetic.config2_image(seed=21, size=256), synthetic.config1_image(seed=22, size=128),
            rng.integers(0, 256, (64, 96, 4), dtype=np.uint8)]
    for img in imgs:
        h, w = img.shape[:2]
        assert np.array_equal(nr.compress_bc15(variant, img), oracle_lib.compress_rgba8(variant, img, w, h))


def _patterns(rng, n, subsets_max=3):
    """2-bit-per-pixel subset maps: the BPTC partition patterns and random maps."""
    L = __import__("oracle").lib()
    table = np.array([L.oracle_get_pattern(p) for p in range(128)], np.uint32)
    pat = table[rng.integers(0, 128, n)]
    rnd = rng.integers(0, subsets_max, (n, 16)).astype(np.uint64)
    rnd = (rnd << (2 * np.arange(16, dtype=np.uint64))).sum(1).astype(np.uint32)
    return np.where(rng.random(n) < 0.5, pat, rnd).astype(np.uint32)


def _endpoints(rng, n):
    ep = rng.uniform(-20.0, 275.0, (n, 24)).astype(np.float32)
    ints = rng.random((n, 1)) < 0.4  # integer endpoints, as after quantisation
    ep = np.where(ints, np.clip(np.round(ep), 0, 255), ep).astype(np.float32)
    same = rng.random(n) < 0.05  # collapsed pairs: the 0 / 0 projection
    ep[same, 4:8] = ep[same, 0:4]
    return ep


@pytest.mark.parametrize("bits", [2, 3, 4])
@pytest.mark.parametrize("channels", [3, 4])
def test_block_quant(oracle_lib, bits, channels):
    rng = np.random.default_rng(100 * bits + channels)
    blk, ep, pat = _blocks(rng, N), _endpoints(rng, N), _patterns(rng, N)
    q, err = nr.block_quant(blk, bits, ep, pat, channels)
    L = oracle_lib.lib()
    eq = np.zeros((N, 2), np.uint32)
    ee = np.zeros(N, np.float32)
    for i in range(N):
        b, e = np.ascontiguousarray(blk[i]), np.ascontiguousarray(ep[i])
        ee[i] = L.oracle_block_quant(_ptr(eq[i]), _ptr(b), bits, _ptr(e), int(pat[i]), channels)
    assert np.array_equal(q, eq), np.nonzero((q != eq).any(1))[0][:10]
    assert _bits_equal(err, ee)


@pytest.mark.parametrize("bits", [2, 3, 4])
@pytest.mark.parametrize("channels", [3, 4])
def test_opt_endpoints(oracle_lib, bits, channels):
    rng = np.random.default_rng(200 * bits + channels)
    blk = _blocks(rng, N)
    q = rng.integers(0, 1 << bits, (N, 16)).astype(np.uint64)
    q[rng.random(N) < 0.05] = 0  # all indices equal: the flattened fit
    qb = np.stack([(q[:, :8] << (4 * np.arange(8, dtype=np.uint64))).sum(1),
                   (q[:, 8:] << (4 * np.arange(8, dtype=np.uint64))).sum(1)], 1).astype(np.uint32)
    mask = rng.integers(1, 1 << 16, N).astype(np.uint32)
    ep0 = rng.uniform(0, 255, (N, 8)).astype(np.float32)
    got = nr.opt_endpoints(ep0, blk, bits, qb, mask, channels)
    L = oracle_lib.lib()
    exp = ep0.copy()
    for i in range(N):
        b, e, qq = np.ascontiguousarray(blk[i]), exp[i], np.ascontiguousarray(qb[i])
        L.oracle_opt_endpoints(_ptr(e), _ptr(b), bits, _ptr(qq), int(mask[i]), channels)
    assert _bits_equal(got, exp), np.nonzero((got.view(np.uint32) != exp.view(np.uint32)).any(1))[0][:10]


@pytest.mark.parametrize("mode", range(8))
@pytest.mark.parametrize("channels", [3, 4])
def test_ep_quant_dequant(oracle_lib, mode, channels):
    rng = np.random.default_rng(300 * mode + channels)
    ep = _endpoints(rng, N)
    q, e = nr.ep_quant_dequant(ep, mode, channels)
    L = oracle_lib.lib()
    eq = np.zeros((N, 24), np.int32)
    ee = ep.copy()
    for i in range(N):
        L.oracle_ep_quant_dequant(_ptr(eq[i]), _ptr(ee[i]), mode, channels)
    m = 8 * nr.PAIRS[mode]
    assert np.array_equal(q[:, :m], eq[:, :m])
    assert _bits_equal(e, ee)


@pytest.mark.parametrize("channels", [3, 4])
def test_pca_bound_and_segment(oracle_lib, channels):
    rng = np.random.default_rng(400 + channels)
    blk = _blocks(rng, N)
    mask = rng.integers(1, 1 << 16, N).astype(np.uint32)
    full = rng.random(N) < 0.1
    mask[full] = 0xFFFF
    bound = nr.block_pca_bound_split(blk, mask, channels)
    seg = nr.block_segment_core(blk, mask, channels)
    L = oracle_lib.lib()
    eb = np.zeros(N, np.float32)
    es = np.zeros((N, 8), np.float32)
    for i in range(N):
        b = np.ascontiguousarray(blk[i])
        eb[i] = L.oracle_block_pca_bound_split(_ptr(b), int(mask[i]), channels)
        L.oracle_block_segment_core(_ptr(es[i]), _ptr(b), int(mask[i]), channels)
    assert _bits_equal(bound, eb)
    cols = [p for p in range(8) if p % 4 < channels]
    assert _bits_equal(seg[:, cols], es[:, cols]), np.nonzero(
        (seg[:, cols].view(np.uint32) != es[:, cols].view(np.uint32)).any(1))[0][:10]
