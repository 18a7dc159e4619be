"""Cuts the image fixtures in tests/golden/images/ from the reference's test
images (tests/images/{brick,brick-alpha,marble,marble-alpha,blender}.png of
block_compression v0.3.0, the images of its PSNR tests, tests/metrics.rs).

    python tests/golden/make_fixture_images.py <reference checkout>

Each fixture is the 128x128 centre crop of one image, converted to RGBA8 as
the reference's tests load it (image::DynamicImage::to_rgba8, alpha 255 for
RGB images). The crops are committed; nothing at test time reads the
reference tree.
"""
import os
import sys

import numpy as np
from PIL import Image

NAMES = ["brick", "brick-alpha", "marble", "marble-alpha", "blender"]
SIZE = 128
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "images")


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BCN_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_fixture_images.py <reference checkout> (or set BCN_REFERENCE_DIR)")
    os.makedirs(HERE, exist_ok=True)
    for name in NAMES:
        img = np.asarray(Image.open(os.path.join(ref, "tests", "images", name + ".png")).convert("RGBA"))
        h, w = img.shape[:2]
        y, x = (h - SIZE) // 2 // 4 * 4, (w - SIZE) // 2 // 4 * 4
        crop = np.ascontiguousarray(img[y:y + SIZE, x:x + SIZE])
        Image.fromarray(crop, "RGBA").save(os.path.join(HERE, name + ".png"), optimize=True)
        print("%s: %dx%d crop at (%d, %d) of %dx%d" % (name, SIZE, SIZE, x, y, w, h))


if __name__ == "__main__":
    main()
