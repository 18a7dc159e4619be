"""The PSNR cases of the reference's image-quality tests (tests/metrics.rs:255-526)
on the committed 128x128 crops of its test images (tests/golden/images/, made
by tests/golden/make_fixture_images.py), and the reference's metric restated in
numpy float64 (calculate_image_metrics_rgba8, tests/metrics.rs:40-114).
Shared by the CPU and GPU image tests."""
import os

import numpy as np

IMAGES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "images")

OPAQUE = ["brick", "marble", "blender"]
ALPHA = ["brick-alpha", "marble-alpha"]
BC6H_PRESETS = ["very_fast", "fast", "basic", "slow", "very_slow"]
BC7_ALPHA = ["alpha_ultrafast", "alpha_very_fast", "alpha_fast", "alpha_basic", "alpha_slow"]
BC7_OPAQUE = ["opaque_ultra_fast", "opaque_very_fast", "opaque_fast", "opaque_basic", "opaque_slow"]

# (image, variant id, preset name or None, channels compared): psnr_bc1,
# psnr_bc3, psnr_bc6h_*, psnr_bc7_alpha_* and psnr_bc7_opaque_* of metrics.rs
CASES = ([(im, 0, None, 3) for im in OPAQUE] + [(im, 2, None, 4) for im in ALPHA] +
         [(im, 5, p, 3) for p in BC6H_PRESETS for im in OPAQUE] +
         [(im, 6, p, 4) for p in BC7_ALPHA for im in ALPHA] +
         [(im, 6, p, 3) for p in BC7_OPAQUE for im in OPAQUE])


def case_id(case):
    im, vid, preset, ch = case
    return "%s-%s%s" % (im, ["bc1", "bc2", "bc3", "bc4", "bc5", "bc6h", "bc7"][vid], "-" + preset if preset else "")


def load(name):
    from PIL import Image
    return np.ascontiguousarray(np.asarray(Image.open(os.path.join(IMAGES, name + ".png")).convert("RGBA")))


def settings_list(bcn, vid, preset):
    """The preset's settings as the oracle's u32 list (None for BC1-BC5)."""
    if vid == 5:
        return getattr(bcn.BC6HSettings, preset)().as_list()
    if vid == 6:
        return getattr(bcn.BC7Settings, preset)().as_list()
    return None


def srgb_to_linear(v):
    """tests/common/mod.rs:17-24 in f64."""
    v = np.asarray(v, np.float64) / 255.0
    return np.where(v <= 0.04045, v / 12.92, ((v + 0.055) / 1.055) ** 2.4)


def psnr(original, decoded, channels):
    """(overall PSNR, per-channel MSE) of two RGBA8 images, tests/metrics.rs:40-114."""
    a = np.asarray(original, np.uint8).reshape(-1, 4)
    b = np.asarray(decoded, np.uint8).reshape(-1, 4)
    mse = np.zeros(4)
    for c in range(channels):
        if c < 3:
            d = srgb_to_linear(a[:, c]) - srgb_to_linear(b[:, c])
        else:
            d = a[:, c] / 255.0 - b[:, c] / 255.0
        mse[c] = np.sum(d * d) / a.shape[0]
    overall = mse.sum() / channels
    return (0.0 if overall == 0.0 else 20.0 * np.log10(1.0 / np.sqrt(overall))), mse


TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_images_psnr.json")


def oracle_psnr_table(bcn, oracle):
    """{case id: overall PSNR} of the oracle's encode -> decode round trip."""
    out = {}
    for case in CASES:
        im, vid, preset, ch = case
        img = load(im)
        blocks = oracle.compress_rgba8(vid, img, img.shape[1], img.shape[0], settings=settings_list(bcn, vid, preset))
        out[case_id(case)] = float(psnr(img, oracle.decompress_rgba8(vid, blocks, img.shape[1], img.shape[0]), ch)[0])
    return out


if __name__ == "__main__":
    # `python tests/reference_images.py` rewrites the committed PSNR table.
    import json
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import block_compression_b200 as bcn
    import oracle
    with open(TABLE, "w") as f:
        json.dump(oracle_psnr_table(bcn, oracle), f, indent=1)
    print("wrote", TABLE)
