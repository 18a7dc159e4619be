"""Differentiable BC1/BC7 decode and gradient endpoint refinement on the GPU,
checked against the oracle's restatement (bit-exact), against FP64 finite
differences (the adjoint), and against torch's own Adam through a
torch.autograd.Function that wraps the C-ABI kernels (test harness only)."""
import numpy as np
import pytest

from block_compression_b200 import synthetic
from block_compression_b200.settings import BC7Settings

from test_refine_cpu import random_bc7_blocks

pytestmark = pytest.mark.gpu


def _autograd_fn(torch, kind):
    from block_compression_b200 import refine

    fwd = refine.decode_relaxed_bc7 if kind == "bc7" else refine.decode_relaxed_bc1
    adj = refine.decode_adjoint_bc7 if kind == "bc7" else refine.decode_adjoint_bc1

    class RelaxedDecode(torch.autograd.Function):
        @staticmethod
        def forward(ctx, endpoints, meta):
            ctx.save_for_backward(meta)
            return fwd(meta, endpoints.contiguous())

        @staticmethod
        def backward(ctx, grad):
            (meta,) = ctx.saved_tensors
            return adj(meta, grad.contiguous()), None

    return RelaxedDecode.apply


def _enc(bcn, torch, variant, timg, w, h):
    out = torch.zeros(variant.blocks_byte_size(w, h), dtype=torch.uint8, device="cuda")
    bcn.encode.compress_rgba8(variant, timg, out, w, h, w * 4)
    return out


def _dec(bcn, torch, variant, blocks, w, h):
    out = torch.zeros(w * h * 4, dtype=torch.uint8, device="cuda")
    bcn.decode.decompress_blocks_as_rgba8(variant, w, h, blocks, out)
    return out.view(h, w, 4)


def _blocks(kind, rng):
    if kind == "bc7":
        return random_bc7_blocks(rng, 128)  # 1024 blocks over modes 0-7 + 4 reserved
    return rng.integers(0, 256, size=(1024, 8), dtype=np.uint8)


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_parse_matches_oracle(bcn, oracle_lib, cuda, kind):
    import torch
    from block_compression_b200 import refine
    rng = np.random.default_rng(21)
    blocks = _blocks(kind, rng)
    parse = refine.parse_bc7 if kind == "bc7" else refine.parse_bc1
    meta, ep = parse(torch.from_numpy(blocks.reshape(-1)).cuda())
    om, oe = oracle_lib.parse(kind, blocks)
    assert np.array_equal(meta.cpu().numpy().view(np.uint32), om)
    assert np.array_equal(ep.cpu().numpy(), oe)


def test_bc7_relaxed_rounds_to_decoder(bcn, oracle_lib, cuda):
    """At the parsed endpoints, floor(relaxed + 0.5) is the GPU decoder's
    output, bit for bit, for encoded blocks of every preset family."""
    import torch
    from block_compression_b200 import refine
    img = synthetic.config2_image(2, 256)
    timg = torch.from_numpy(img).cuda()
    for preset in ["alpha_basic", "opaque_basic", "alpha_slow", "opaque_ultra_fast"]:
        st = getattr(BC7Settings, preset)()
        blocks = _enc(bcn, torch, bcn.CompressionVariant.BC7(st), timg, 256, 256)
        meta, ep = refine.parse_bc7(blocks)
        rel = refine.decode_relaxed_bc7(meta, ep)
        dec = _dec(bcn, torch, bcn.CompressionVariant.BC7(st), blocks, 256, 256)
        decb = oracle_lib.image_blocks(dec.cpu().numpy(), 256, 256)
        assert np.array_equal(torch.floor(rel + 0.5).cpu().numpy(), decb.astype(np.float32)), preset


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_relaxed_and_adjoint_match_fp64(bcn, oracle_lib, cuda, kind):
    import torch
    from block_compression_b200 import refine
    rng = np.random.default_rng(22)
    blocks = _blocks(kind, rng)
    meta, ep = (refine.parse_bc7 if kind == "bc7" else refine.parse_bc1)(torch.from_numpy(blocks.reshape(-1)).cuda())
    theta = ep + torch.from_numpy(rng.uniform(-4, 4, size=tuple(ep.shape)).astype(np.float32)).cuda()
    fwd = refine.decode_relaxed_bc7 if kind == "bc7" else refine.decode_relaxed_bc1
    adj = refine.decode_adjoint_bc7 if kind == "bc7" else refine.decode_adjoint_bc1
    om = meta.cpu().numpy().view(np.uint32)
    th64 = theta.cpu().numpy().astype(np.float64)
    # FP32 relaxed decode vs FP64: a few FP32 ulps (values up to ~260)
    np.testing.assert_allclose(fwd(meta, theta).cpu().numpy(), oracle_lib.relaxed_f64(kind, om, th64), rtol=4e-7,
                               atol=1e-5)
    g = rng.normal(0, 10, size=(len(om), 16, 4)).astype(np.float32)
    got = adj(meta, torch.from_numpy(g).cuda()).cpu().numpy()
    np.testing.assert_allclose(got, oracle_lib.adjoint_f64(kind, om, g.astype(np.float64)), rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_autograd_gradient_vs_fp64_finite_differences(bcn, oracle_lib, cuda, kind):
    """MSE loss through the autograd.Function on 1,024 random blocks; the
    gradient from the adjoint kernel is checked against central differences
    (eps = 1e-3) of the FP64 relaxed decode. Tolerance: rtol 1e-4, atol 1e-2
    (FP32 forward rounding of ~1e-5 per texel over 64 terms)."""
    import torch
    from block_compression_b200 import refine
    rng = np.random.default_rng(23)
    blocks = _blocks(kind, rng)
    meta, ep = (refine.parse_bc7 if kind == "bc7" else refine.parse_bc1)(torch.from_numpy(blocks.reshape(-1)).cuda())
    theta0 = ep.cpu().numpy() + rng.uniform(-4, 4, size=tuple(ep.shape)).astype(np.float32)
    src = rng.integers(0, 256, size=(len(blocks), 16, 4)).astype(np.float32)
    theta = torch.from_numpy(theta0).cuda().requires_grad_(True)
    s = torch.from_numpy(src).cuda()
    f = _autograd_fn(torch, kind)
    loss = ((f(theta, meta) - s) ** 2).sum()
    loss.backward()
    grad = theta.grad.cpu().numpy().astype(np.float64)
    om = meta.cpu().numpy().view(np.uint32)
    th64 = theta0.astype(np.float64)
    s64 = src.astype(np.float64)

    def block_loss(t):
        return ((oracle_lib.relaxed_f64(kind, om, t) - s64) ** 2).sum(axis=(1, 2))

    eps = 1e-3
    fd = np.zeros_like(th64)
    for j in range(th64.shape[1]):
        e = np.zeros_like(th64)
        e[:, j] = eps
        fd[:, j] = (block_loss(th64 + e) - block_loss(th64 - e)) / (2 * eps)
    np.testing.assert_allclose(grad, fd, rtol=1e-4, atol=1e-2)
    assert np.abs(fd).max() > 100.0  # the check is not vacuous


def _encode_c5(bcn, torch, size=512, seed=1, preset="opaque_basic"):
    img = synthetic.config1_image(seed, size)
    timg = torch.from_numpy(img).cuda()
    blocks = _enc(bcn, torch, bcn.CompressionVariant.BC7(getattr(BC7Settings, preset)()), timg, size, size)
    return img, timg, blocks


@pytest.mark.parametrize("preset,channels", [("opaque_basic", 3), ("alpha_basic", 4)])
def test_bc7_refine_matches_oracle_bit_exact(bcn, oracle_lib, cuda, preset, channels):
    import torch
    from block_compression_b200 import refine
    img = synthetic.config2_image(2, 128) if channels == 4 else synthetic.config1_image(1, 128)
    timg = torch.from_numpy(img).cuda()
    blocks = _enc(bcn, torch, bcn.CompressionVariant.BC7(getattr(BC7Settings, preset)()), timg, 128, 128)
    orig = blocks.cpu().numpy().copy()
    stats, theta = refine.refine_bc7(timg, blocks, channels=channels, steps=20, lr=0.5, return_endpoints=True)
    out, oth, errs = oracle_lib.refine_blocks("bc7", orig, oracle_lib.image_blocks(img, 128, 128), 20, 0.5, channels)
    assert np.array_equal(blocks.cpu().numpy().reshape(-1, 16), out)
    assert np.array_equal(theta.cpu().numpy(), oth)
    d = stats.as_dict()
    assert d["blocks"] == 1024 and d["replaced"] == int((errs[:, 1] < errs[:, 0]).sum()) > 0
    assert d["err_before"] == int(errs[:, 0].sum()) and d["err_after"] == int(errs[:, 1].sum())


def test_bc1_refine_matches_oracle_bit_exact(bcn, oracle_lib, cuda):
    import torch
    from block_compression_b200 import refine
    img = synthetic.config1_image(1, 128)
    timg = torch.from_numpy(img).cuda()
    blocks = _enc(bcn, torch, bcn.CompressionVariant.BC1, timg, 128, 128)
    orig = blocks.cpu().numpy().copy()
    stats, theta = refine.refine_bc1(timg, blocks, steps=20, lr=0.5, return_endpoints=True)
    out, oth, errs = oracle_lib.refine_blocks("bc1", orig, oracle_lib.image_blocks(img, 128, 128), 20, 0.5)
    assert np.array_equal(blocks.cpu().numpy().reshape(-1, 8), out)
    assert np.array_equal(theta.cpu().numpy(), oth)
    assert stats.replaced == int((errs[:, 1] < errs[:, 0]).sum()) > 0
    assert stats.err_after == int(errs[:, 1].sum()) < stats.err_before


def test_c5_workload_never_worse_and_improves(bcn, oracle_lib, cuda):
    """8 RGBA8 images of 512x512 (the BC1 generator), BC7 basic, 20 Adam steps
    at lr 0.5: per block the exact error never rises, the replaced blocks are
    exactly the changed ones, and the summed error drops."""
    import torch
    from block_compression_b200 import refine
    total_before = total_after = 0
    for i in range(8):
        img, timg, blocks = _encode_c5(bcn, torch, 512, seed=100 + i)
        before = blocks.clone()
        stats = refine.refine_bc7(timg, blocks, channels=3, steps=20, lr=0.5)
        v = bcn.CompressionVariant.BC7(BC7Settings.opaque_basic())
        d0 = oracle_lib.image_blocks(_dec(bcn, torch, v, before, 512, 512).cpu().numpy(), 512, 512)
        d1 = oracle_lib.image_blocks(_dec(bcn, torch, v, blocks, 512, 512).cpu().numpy(), 512, 512)
        src = oracle_lib.image_blocks(img, 512, 512).astype(np.int64)
        e0 = ((d0[..., :3].astype(np.int64) - src[..., :3]) ** 2).sum(axis=(1, 2))
        e1 = ((d1[..., :3].astype(np.int64) - src[..., :3]) ** 2).sum(axis=(1, 2))
        assert (e1 <= e0).all()
        changed = (before != blocks).view(-1, 16).any(dim=1).cpu().numpy()
        assert np.array_equal(changed, e1 < e0)
        assert stats.replaced == int(changed.sum()) and stats.err_before == int(e0.sum())
        assert stats.err_after == int(e1.sum())
        total_before += int(e0.sum())
        total_after += int(e1.sum())
    assert total_after < total_before


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_torch_adam_through_autograd_function(bcn, cuda, kind):
    """torch.optim.Adam driving the autograd.Function reaches the same relaxed
    loss as the fused kernel's Adam (same hyper-parameters; the two differ only
    in rounding order)."""
    import torch
    from block_compression_b200 import refine
    img = synthetic.config1_image(1, 128)
    timg = torch.from_numpy(img).cuda()
    if kind == "bc7":
        blocks = _enc(bcn, torch, bcn.CompressionVariant.BC7(BC7Settings.opaque_basic()), timg, 128, 128)
        meta, ep = refine.parse_bc7(blocks)
        _, theta_k = refine.refine_bc7(timg, blocks.clone(), channels=3, steps=20, lr=0.5, return_endpoints=True)
    else:
        blocks = _enc(bcn, torch, bcn.CompressionVariant.BC1, timg, 128, 128)
        meta, ep = refine.parse_bc1(blocks)
        _, theta_k = refine.refine_bc1(timg, blocks.clone(), steps=20, lr=0.5, return_endpoints=True)
    src = timg.view(32, 4, 32, 4, 4).permute(0, 2, 1, 3, 4).reshape(-1, 16, 4).float()
    mask = torch.tensor([1.0, 1.0, 1.0, 0.0], device="cuda")
    f = _autograd_fn(torch, kind)
    theta = ep.clone().requires_grad_(True)
    opt = torch.optim.Adam([theta], lr=0.5, betas=(0.9, 0.999), eps=1e-8)
    for _ in range(20):
        opt.zero_grad()
        loss = (((f(theta, meta) - src) * mask) ** 2).sum()
        loss.backward()
        opt.step()
    with torch.no_grad():
        l_torch = float((((f(theta, meta) - src) * mask) ** 2).sum())
        l_kernel = float((((f(theta_k, meta) - src) * mask) ** 2).sum())
        l_start = float((((f(ep, meta) - src) * mask) ** 2).sum())
    assert l_kernel < l_start
    assert abs(l_torch - l_kernel) <= 1e-3 * l_start
    assert float((theta.detach() - theta_k).abs().median()) < 1e-3


def test_refine_argument_errors(bcn, cuda):
    import torch
    from block_compression_b200 import refine
    src = torch.zeros((8, 8, 4), dtype=torch.uint8, device="cuda")
    blocks = torch.zeros(4 * 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(bcn.BcError):
        refine.refine_bc7(src, blocks, channels=5)
    with pytest.raises(bcn.BcError):
        refine.refine_bc7(src, blocks[:32])
    with pytest.raises(bcn.BcError):
        refine.refine_bc7(src, blocks, lr=float("nan"))
    with pytest.raises(bcn.BcError):
        refine.refine_bc7(src, blocks, width=6, height=8)
    stats = refine.refine_bc7(src, blocks, steps=0)
    assert stats.replaced == 0


@pytest.mark.parametrize("kind", ["bc7", "bc1"])
def test_refine_images_equals_per_image(bcn, cuda, kind):
    """The multi-image entry point gives the same blocks and totals as one
    call per image (images of different sizes in one launch)."""
    import torch
    from block_compression_b200 import refine
    sizes = [(64, 64), (32, 96), (128, 40)]
    v = bcn.CompressionVariant.BC7(BC7Settings.opaque_basic()) if kind == "bc7" else bcn.CompressionVariant.BC1
    imgs, a, b = [], [], []
    for i, (h, w) in enumerate(sizes):
        t = torch.from_numpy(synthetic.config4_texture(11, i, h, w)).cuda()
        blk = _enc(bcn, torch, v, t, w, h)
        imgs.append(t)
        a.append(blk.clone())
        b.append(blk.clone())
    tot = [0, 0, 0, 0]
    for t, blk in zip(imgs, a):
        st = refine.refine_bc7(t, blk, channels=3) if kind == "bc7" else refine.refine_bc1(t, blk)
        tot = [x + y for x, y in zip(tot, [st.blocks, st.replaced, st.err_before, st.err_after])]
    if kind == "bc7":
        st = refine.refine_bc7_images(list(zip(imgs, b)), channels=3)
    else:
        st = refine.refine_bc1_images(list(zip(imgs, b)))
    assert [st.blocks, st.replaced, st.err_before, st.err_after] == tot
    for x, y in zip(a, b):
        assert torch.equal(x, y)
