"""Batched path (one task table, one CUDA graph) and GPU mip generation,
checked against the per-task path and the CPU oracle."""
import ctypes

import numpy as np
import pytest

from block_compression_b200 import synthetic

pytestmark = pytest.mark.gpu


def _textures(torch):
    shapes = [(64, 48), (20, 36), (128, 128), (4, 4), (36, 100)]
    out = []
    for i, (h, w) in enumerate(shapes):
        out.append(torch.from_numpy(synthetic.config4_texture(7, i, h, w)).cuda())
    return out


def test_mip_chain_matches_numpy(bcn, cuda):
    import torch

    from block_compression_b200 import mips
    for h, w in [(64, 48), (12, 36), (4, 4), (100, 8)]:
        img = synthetic.config4_texture(3, h * 1000 + w, h, w)
        levels = mips.generate_mip_chain(torch.from_numpy(img).cuda())
        ref = synthetic.box_mip_chain(img)
        assert len(levels) == len(ref)
        for lv, r in zip(levels, ref):
            assert (lv.height, lv.width) == r.shape[:2]
            assert np.array_equal(lv.data.cpu().numpy(), synthetic.pad_to_multiple_of_4(r))


def _add_all(bcn, c, torch, textures, variants):
    """Every texture with its full mip chain, round-robin variants; returns
    the output buffer and the per-task (level, variant, offset) list."""
    from block_compression_b200 import mips
    tasks, total = [], 0
    chains = [mips.generate_mip_chain(t) for t in textures]
    for i, chain in enumerate(chains):
        v = variants[i % len(variants)]
        for lv in chain:
            n = v.blocks_byte_size(lv.padded_width, lv.padded_height)
            tasks.append((lv, v, total, n))
            total += n
    buf = torch.zeros(total, dtype=torch.uint8, device="cuda")
    for lv, v, off, n in tasks:
        c.add_compression_task(v, lv.data, lv.padded_width, lv.padded_height, buf, blocks_offset=off)
    return buf, tasks, chains


def _variants(bcn):
    V = bcn.CompressionVariant
    return [V.BC1, V.BC5, V.BC7(bcn.BC7Settings.alpha_basic()), V.BC3, V.BC7(bcn.BC7Settings.opaque_fast()), V.BC4]


def test_batched_equals_per_task_and_oracle(bcn, oracle_lib, cuda):
    import torch
    textures = _textures(torch)
    variants = _variants(bcn)
    c = bcn.GpuBlockCompressor()
    plain, tasks, _ = _add_all(bcn, c, torch, textures, variants)
    c.compress()
    torch.cuda.synchronize()
    c2 = bcn.GpuBlockCompressor()
    batched, _, _ = _add_all(bcn, c2, torch, textures, variants)
    c2.compress_batched()
    torch.cuda.synchronize()
    assert torch.equal(plain, batched)
    got = batched.cpu().numpy()
    for lv, v, off, n in tasks:
        img = lv.data.cpu().numpy()
        s = v.settings.as_list() if v.settings is not None else None
        exp = oracle_lib.compress_rgba8(v.id, img, lv.padded_width, lv.padded_height, settings=s)
        assert np.array_equal(got[off:off + n], exp), (v, lv.padded_width, lv.padded_height)


@pytest.mark.parametrize("tune", [(128, 2, 1, 4), (256, 8, 4, 8), (128, 1, 64, 8)])
def test_batch_graph_replay_and_explicit_tunes(bcn, cuda, tune):
    import torch
    textures = _textures(torch)
    variants = _variants(bcn)
    c = bcn.GpuBlockCompressor()
    plain, _, _ = _add_all(bcn, c, torch, textures, variants)
    c.compress()
    c2 = bcn.GpuBlockCompressor()
    out, _, chains = _add_all(bcn, c2, torch, textures, variants)
    t = bcn.Tune(*tune)
    b = c2.create_batch(tune=t)
    assert c2.task_count() == 0
    assert b.tune.as_dict() == t.as_dict()
    for _ in range(3):  # replays give identical results
        out.zero_()
        b.launch()
        torch.cuda.synchronize()
        assert torch.equal(out, plain)
    b.close()


def test_autotune_picks_a_valid_shape(bcn, cuda):
    import torch
    c = bcn.GpuBlockCompressor()
    _add_all(bcn, c, torch, _textures(torch), _variants(bcn))
    b = c.create_batch(autotune=True)
    t = b.tune.as_dict()
    assert t["threads_per_cta"] in (128, 256) and t["bc7_search_warps"] in (4, 8)
    assert 1 <= t["ctas_per_sm"] <= 16 and 1 <= t["tiles_per_claim"] <= 64
    b.launch()
    torch.cuda.synchronize()
    b.close()


def test_invalid_tune_rejected(bcn, cuda):
    c = bcn.GpuBlockCompressor()
    with pytest.raises(bcn.BcError):
        c.create_batch(tune=bcn.Tune(64, 4, 4, 8))
