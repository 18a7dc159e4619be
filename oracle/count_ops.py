"""Measures the reference encoders' algorithmic work (FP32 ops per block,
op-counting build of the oracle) on the benchmark workloads' content.

    python -m oracle.count_ops [--blocks N]

Prints ops/block for BC1 (1024^2 textured image), BC3/BC4/BC5 and BC7
alpha_basic (2048^2 alpha image / normal map), BC6H basic (1024^2 HDR),
averaged over a seeded random sample of blocks. These are the per-block
figures the bench's rooflines use.
"""
import argparse
import json
import sys

import numpy as np

import oracle
from block_compression_b200 import synthetic


def blocks_of(img, idx):
    h, w = img.shape[:2]
    bw = w // 4
    out = []
    for i in idx:
        by, bx = divmod(int(i), bw)
        t = img[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4].reshape(16, -1).astype(np.float32)
        out.append(np.ascontiguousarray(t.T.reshape(-1)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--blocks", type=int, default=2048)
    args = ap.parse_args()
    rng = np.random.default_rng(0)
    img1 = synthetic.config1_image(seed=1, size=1024)
    img2 = synthetic.config2_image(seed=2, size=2048)
    nrm = synthetic.normal_map(seed=2, size=2048)
    hdr = synthetic.config3_hdr(seed=3, size=1024)
    a7 = [2, 2, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 12, 8, 8, 0, 2, 4]  # BC7Settings::alpha_basic()
    b6 = [0, 0, 2, 2, 4]                                               # BC6HSettings::basic()
    res = {}
    idx1 = rng.choice((1024 // 4) ** 2, args.blocks, replace=False)
    idx2 = rng.choice((2048 // 4) ** 2, args.blocks, replace=False)
    res["bc1_c1"] = float(np.mean([oracle.count_ops("bc1", b) for b in blocks_of(img1, idx1)]))
    blk2 = blocks_of(img2, idx2)
    res["bc3_c2"] = float(np.mean([oracle.count_ops("bc3_alpha", b) + oracle.count_ops("bc1", b) for b in blk2]))
    res["bc7_alpha_basic_c2"] = float(np.mean([oracle.count_ops("bc7", b, a7) for b in blk2]))
    red = []
    for b in blk2:
        r = b.copy()
        r[48:] = b[:16]
        red.append(r)
    res["bc4_c2"] = float(np.mean([oracle.count_ops("bc3_alpha", b) for b in red]))
    nb = []
    for b in blocks_of(nrm, idx2):
        r, g = b.copy(), b.copy()
        r[48:] = b[:16]
        g[48:] = b[16:32]
        nb.append((r, g))
    res["bc5_normal_c2"] = float(np.mean([oracle.count_ops("bc3_alpha", r) + oracle.count_ops("bc3_alpha", g) for r, g in nb]))
    hb = []
    for b in blocks_of(hdr.view(np.uint16), idx1):
        b = b.copy()
        b[48:] = 0.0
        hb.append(b)
    res["bc6h_basic_c3"] = float(np.mean([oracle.count_ops("bc6h", b, b6) for b in hb]))
    json.dump({"ops_per_block": res, "blocks_sampled": args.blocks}, sys.stdout, indent=1)
    print()


if __name__ == "__main__":
    main()
