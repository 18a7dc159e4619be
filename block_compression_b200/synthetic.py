"""Seeded synthetic textures for the benchmark configurations.

No public dataset is involved: these generators produce the content the
benchmark configurations describe (gradients + value noise + hard-edged
polygons for RGBA8, log-uniform HDR with spikes for RGBA16F, normal maps for
BC5, mip chains for the batched workload). Every generator is a pure function
of its seed (numpy PCG64).
"""
import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _bilinear_gradient(rng, h, w):
    """Per-channel smooth bilinear gradient from 4 random corner values."""
    c = rng.uniform(0, 255, size=(2, 2, 3))
    y = np.linspace(0.0, 1.0, h)[:, None, None]
    x = np.linspace(0.0, 1.0, w)[None, :, None]
    return (c[0, 0] * (1 - y) * (1 - x) + c[0, 1] * (1 - y) * x + c[1, 0] * y * (1 - x) + c[1, 1] * y * x)


def _value_noise(rng, h, w, octaves=4, channels=3, base_cells=4):
    """Sum of `octaves` bilinearly upsampled random lattices, in [-1, 1]."""
    out = np.zeros((h, w, channels))
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = base_cells * (2 ** o)
        lat = rng.uniform(-1, 1, size=(cells + 1, cells + 1, channels))
        ys = np.linspace(0, cells, h)
        xs = np.linspace(0, cells, w)
        y0 = np.minimum(ys.astype(int), cells - 1)
        x0 = np.minimum(xs.astype(int), cells - 1)
        fy = (ys - y0)[:, None, None]
        fx = (xs - x0)[None, :, None]
        a = lat[y0][:, x0]
        b = lat[y0][:, x0 + 1]
        c = lat[y0 + 1][:, x0]
        d = lat[y0 + 1][:, x0 + 1]
        out += amp * (a * (1 - fy) * (1 - fx) + b * (1 - fy) * fx + c * fy * (1 - fx) + d * fy * fx)
        total += amp
        amp *= 0.5
    return out / total


def _fill_polygons(rng, img, count, max_frac=0.25, sides=3):
    """Hard-edged filled convex polygons of uniform random colour."""
    h, w = img.shape[:2]
    for _ in range(count):
        n = sides if sides else int(rng.integers(3, 7))
        cx, cy = rng.uniform(0, w), rng.uniform(0, h)
        r = rng.uniform(0.03, max_frac) * min(h, w)
        ang = np.sort(rng.uniform(0, 2 * np.pi, n))
        px = cx + r * np.cos(ang)
        py = cy + r * np.sin(ang)
        x0, x1 = int(max(0, np.floor(px.min()))), int(min(w, np.ceil(px.max()) + 1))
        y0, y1 = int(max(0, np.floor(py.min()))), int(min(h, np.ceil(py.max()) + 1))
        if x1 <= x0 or y1 <= y0:
            continue
        yy, xx = np.mgrid[y0:y1, x0:x1]
        xx = xx + 0.5
        yy = yy + 0.5
        inside = np.ones(xx.shape, dtype=bool)
        for i in range(n):
            ax, ay, bx, by = px[i], py[i], px[(i + 1) % n], py[(i + 1) % n]
            inside &= (bx - ax) * (yy - ay) - (by - ay) * (xx - ax) >= 0
        img[y0:y1, x0:x1][inside] = rng.uniform(0, 255, size=3)


def rgba8_textured(seed, width, height, polygons=32, sides=3, alpha=None):
    """Gradients + 4-octave value noise (amplitude 40/255) + filled polygons.
    Returns uint8 (height, width, 4); alpha=255 unless an alpha plane is given."""
    rng = _rng(seed)
    rgb = _bilinear_gradient(rng, height, width) + 40.0 * _value_noise(rng, height, width)
    _fill_polygons(rng, rgb, polygons, sides=sides)
    out = np.empty((height, width, 4), dtype=np.uint8)
    out[..., :3] = np.clip(np.rint(rgb), 0, 255).astype(np.uint8)
    out[..., 3] = 255 if alpha is None else alpha
    return out


def config1_image(seed=1, size=1024):
    """BC1 workload: 1024x1024 RGBA8, alpha 255, 32 triangles."""
    return rgba8_textured(seed, size, size, polygons=32)


def config2_image(seed=2, size=2048):
    """BC7/BC3/BC4 workload: 2048x2048 RGBA8; RGB as config 1 with 64
    polygons; alpha = smooth radial ramp, 10% of the 4x4 blocks turned into
    binary 0/255 cutouts, and 5% of the pixels replaced by uniform noise."""
    rng = _rng(seed + 1000)
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float64)
    r = np.hypot(yy - size / 2, xx - size / 2) / (size / np.sqrt(2))
    alpha = np.clip(255.0 * (1.0 - r), 0, 255)
    nb = size // 4
    cut = rng.uniform(size=(nb, nb)) < 0.10
    cut_px = np.repeat(np.repeat(cut, 4, 0), 4, 1)
    alpha = np.where(cut_px, np.where(alpha >= 128, 255.0, 0.0), alpha)
    img = rgba8_textured(seed, size, size, polygons=64, sides=0, alpha=np.rint(alpha).astype(np.uint8))
    noise = rng.uniform(size=(size, size)) < 0.05
    img[noise] = rng.integers(0, 256, size=(int(noise.sum()), 4), dtype=np.uint8)
    return img


def normal_map(seed=2, size=2048):
    """BC5 workload: tangent-space normal map of a random height field,
    X/Y in the R/G channels of an RGBA8 image (B = Z, A = 255)."""
    rng = _rng(seed + 2000)
    hgt = _value_noise(rng, size, size, octaves=5, channels=1, base_cells=8)[..., 0] * 24.0
    gy, gx = np.gradient(hgt)
    n = np.stack([-gx, -gy, np.ones_like(hgt)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    out = np.empty((size, size, 4), dtype=np.uint8)
    out[..., :3] = np.clip(np.rint((n * 0.5 + 0.5) * 255.0), 0, 255).astype(np.uint8)
    out[..., 3] = 255
    return out


def config3_hdr(seed=3, size=1024):
    """BC6H workload: RGBA16F, values log-uniform in [2^-8, 2^8] with smooth
    log-space gradients, 2% specular spikes up to 6e4, alpha 1. Returns
    float16 (size, size, 4)."""
    rng = _rng(seed)
    y = np.linspace(0.0, 1.0, size)[:, None, None]
    x = np.linspace(0.0, 1.0, size)[None, :, None]
    c = rng.uniform(-8, 8, size=(2, 2, 3))
    grad = c[0, 0] * (1 - y) * (1 - x) + c[0, 1] * (1 - y) * x + c[1, 0] * y * (1 - x) + c[1, 1] * y * x
    log2v = np.clip(grad + 3.0 * _value_noise(rng, size, size), -8, 8)
    rgb = np.exp2(log2v)
    spikes = rng.uniform(size=(size, size)) < 0.02
    rgb[spikes] = rng.uniform(256.0, 6.0e4, size=(int(spikes.sum()), 1)) * rng.uniform(0.5, 1.0, size=(int(spikes.sum()), 3))
    out = np.empty((size, size, 4), dtype=np.float16)
    out[..., :3] = rgb.astype(np.float16)
    out[..., 3] = 1.0
    return out


def pad_to_multiple_of_4(img):
    """Edge-replicates an (h, w, c) image up to multiples of 4."""
    h, w = img.shape[:2]
    ph, pw = (-h) % 4, (-w) % 4
    if ph == 0 and pw == 0:
        return img
    return np.pad(img, ((0, ph), (0, pw), (0, 0)), mode="edge")


def box_mip_chain(img):
    """Full box-filtered mip chain of an RGBA8 image down to 1x1 (level sizes
    floor(w/2), floor(h/2), min 1; odd edges fold the last row/column in)."""
    levels = [img]
    cur = img.astype(np.uint32)
    while cur.shape[0] > 1 or cur.shape[1] > 1:
        h, w = cur.shape[:2]
        nh, nw = max(1, h // 2), max(1, w // 2)
        ys = np.minimum(np.arange(nh) * 2, h - 1)
        xs = np.minimum(np.arange(nw) * 2, w - 1)
        ys1 = np.minimum(ys + 1, h - 1)
        xs1 = np.minimum(xs + 1, w - 1)
        s = cur[ys][:, xs] + cur[ys][:, xs1] + cur[ys1][:, xs] + cur[ys1][:, xs1]
        cur = (s + 2) // 4
        levels.append(cur.astype(np.uint8))
    return levels


def config4_textures(seed=4, count=64, sides=None):
    """Batched workload: `count` RGBA8 textures with sides drawn uniformly from
    {16, 20, ..., 4096} (non-square allowed). Returns a list of (h, w) shapes;
    pixel content is generated on demand by config4_texture()."""
    rng = _rng(seed)
    choices = np.arange(16, 4097, 4) if sides is None else np.asarray(sides)
    return [(int(rng.choice(choices)), int(rng.choice(choices))) for _ in range(count)]


def config4_texture(seed, index, h, w):
    return rgba8_textured(seed * 1000 + index, w, h, polygons=16)


def rgba8_textured_torch(seed, height, width, device, polygons=16):
    """GPU version of rgba8_textured for large batches: bilinear gradients +
    4-octave value noise (amplitude 40/255) + filled triangles, alpha 255.
    Random parameters come from a seeded CPU generator, the pixels are made on
    `device`. Returns a uint8 tensor (height, width, 4)."""
    import torch
    import torch.nn.functional as F

    g = torch.Generator().manual_seed(int(seed))
    y = torch.linspace(0.0, 1.0, height, device=device)[:, None, None]
    x = torch.linspace(0.0, 1.0, width, device=device)[None, :, None]
    c = (torch.rand(2, 2, 3, generator=g) * 255.0).to(device)
    rgb = c[0, 0] * (1 - y) * (1 - x) + c[0, 1] * (1 - y) * x + c[1, 0] * y * (1 - x) + c[1, 1] * y * x
    noise = torch.zeros(1, 3, height, width, device=device)
    amp, total = 1.0, 0.0
    for o in range(4):
        cells = 4 * (2 ** o)
        lat = (torch.rand(1, 3, cells + 1, cells + 1, generator=g) * 2 - 1).to(device)
        noise += amp * F.interpolate(lat, size=(height, width), mode="bilinear", align_corners=True)
        total += amp
        amp *= 0.5
    rgb = rgb + 40.0 * (noise[0] / total).permute(1, 2, 0)
    yy = torch.arange(height, device=device, dtype=torch.float32)[:, None] + 0.5
    xx = torch.arange(width, device=device, dtype=torch.float32)[None, :] + 0.5
    for _ in range(polygons):
        cx, cy = float(torch.rand(1, generator=g)) * width, float(torch.rand(1, generator=g)) * height
        r = (0.03 + 0.22 * float(torch.rand(1, generator=g))) * min(height, width)
        ang = torch.sort(torch.rand(3, generator=g) * 6.283185307)[0]
        px = [cx + r * float(torch.cos(a)) for a in ang]
        py = [cy + r * float(torch.sin(a)) for a in ang]
        inside = torch.ones(height, width, dtype=torch.bool, device=device)
        for i in range(3):
            ax, ay, bx, by = px[i], py[i], px[(i + 1) % 3], py[(i + 1) % 3]
            inside &= (bx - ax) * (yy - ay) - (by - ay) * (xx - ax) >= 0
        col = (torch.rand(3, generator=g) * 255.0).to(device)
        rgb = torch.where(inside[..., None], col, rgb)
    out = torch.empty(height, width, 4, dtype=torch.uint8, device=device)
    out[..., :3] = rgb.round().clamp(0, 255).to(torch.uint8)
    out[..., 3] = 255
    return out
