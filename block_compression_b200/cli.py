"""Command-line compressor, the counterpart of the reference's example CLI
(compressor/src/main.rs): `python -m block_compression_b200.cli <variant>
<input_file>` reads an image, compresses it on the GPU through the task
interface and writes `<input_file stem>.dds` next to it.

Variants: bc1 bc2 bc3 bc4 bc5 bc6h bc7; bc6h uses BC6HSettings.very_slow()
and bc7 BC7Settings.alpha_slow(), as the reference CLI does. For bc6h each
8-bit channel is converted sRGB -> linear in f64 and rounded to f16
(compressor/src/main.rs:136-143). Inputs: 8-bit PNG (grey, grey+alpha, RGB,
RGBA; not interlaced) or a .npy array of shape (h, w, 4) uint8. Sizes that
are not multiples of 4 are padded by repeating the last row / column.
"""
import struct
import sys
import time
import zlib

import numpy as np


def read_png(path):
    """Minimal PNG reader: 8-bit grey / grey+alpha / RGB / RGBA, no
    interlacing. Returns uint8 (h, w, 4)."""
    with open(path, "rb") as f:
        data = f.read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat, hdr = 8, [], None
    while pos < len(data):
        n, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if typ == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif typ == b"IDAT":
            idat.append(body)
        elif typ == b"IEND":
            break
    if hdr is None:
        raise ValueError("PNG without IHDR")
    w, h, depth, ctype, _, _, interlace = hdr
    chans = {0: 1, 2: 3, 4: 2, 6: 4}.get(ctype)
    if depth != 8 or chans is None or interlace != 0:
        raise ValueError("only 8-bit non-interlaced grey/RGB/RGBA PNGs are supported")
    raw = zlib.decompress(b"".join(idat))
    stride = w * chans
    out = np.zeros((h, stride), dtype=np.uint8)
    prev = np.zeros(stride, dtype=np.int32)
    for y in range(h):
        ft = raw[y * (stride + 1)]
        line = np.frombuffer(raw, dtype=np.uint8, count=stride, offset=y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, dtype=np.int32)
        if ft == 0:
            cur = line
        elif ft == 2:
            cur = (line + prev) & 0xFF
        elif ft in (1, 3, 4):
            for x in range(stride):
                a = cur[x - chans] if x >= chans else 0
                b = prev[x]
                c = prev[x - chans] if x >= chans else 0
                if ft == 1:
                    p = a
                elif ft == 3:
                    p = (a + b) >> 1
                else:
                    pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
                    p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[x] = (line[x] + p) & 0xFF
        else:
            raise ValueError("bad PNG filter type %d" % ft)
        out[y] = cur
        prev = cur
    px = out.reshape(h, w, chans)
    rgba = np.empty((h, w, 4), dtype=np.uint8)
    if chans == 1:
        rgba[..., :3] = px
        rgba[..., 3] = 255
    elif chans == 2:
        rgba[..., :3] = px[..., :1]
        rgba[..., 3] = px[..., 1]
    elif chans == 3:
        rgba[..., :3] = px
        rgba[..., 3] = 255
    else:
        rgba[:] = px
    return rgba


def srgb8_to_linear_f16_table():
    """srgb_to_linear (compressor/src/main.rs:186-194) of every byte, in f64,
    rounded to f16 directly from f64 (half::f16::from_f64)."""
    v = np.arange(256, dtype=np.float64) / 255.0
    lin = np.where(v <= 0.04045, v / 12.92, ((v + 0.055) / 1.055) ** 2.4)
    return lin.astype(np.float16)


def _variant(name):
    import block_compression_b200 as bcn
    V = bcn.CompressionVariant
    table = {"bc1": V.BC1, "bc2": V.BC2, "bc3": V.BC3, "bc4": V.BC4, "bc5": V.BC5,
             "bc6h": V.BC6H(bcn.BC6HSettings.very_slow()), "bc7": V.BC7(bcn.BC7Settings.alpha_slow())}
    return table.get(name.lower())


def compress_file(variant_name, file_name, out_name=None, log=print):
    import torch

    import block_compression_b200 as bcn
    from block_compression_b200 import dds, synthetic

    variant = _variant(variant_name)
    if variant is None:
        raise ValueError("invalid compression variant %r" % variant_name)
    t0 = time.perf_counter()
    img = np.load(file_name) if file_name.endswith(".npy") else read_png(file_name)
    img = synthetic.pad_to_multiple_of_4(np.ascontiguousarray(img, dtype=np.uint8))
    h, w = img.shape[:2]
    if variant.id == 5:
        src = torch.from_numpy(srgb8_to_linear_f16_table()[img].view(np.int16)).cuda()
    else:
        src = torch.from_numpy(img).cuda()
    torch.cuda.synchronize()
    log("Image read and upload took: %.3f ms" % ((time.perf_counter() - t0) * 1e3))
    blocks = torch.zeros(variant.blocks_byte_size(w, h), dtype=torch.uint8, device="cuda")
    c = bcn.GpuBlockCompressor()
    c.add_compression_task(variant, src, w, h, blocks)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    c.compress()
    b.record()
    torch.cuda.synchronize()
    log("Compression took: %.3f ms" % a.elapsed_time(b))
    t0 = time.perf_counter()
    data = blocks.cpu().numpy()
    log("Block data download took: %.3f ms" % ((time.perf_counter() - t0) * 1e3))
    t0 = time.perf_counter()
    if out_name is None:
        out_name = file_name.rsplit(".", 1)[0] + ".dds" if "." in file_name.split("/")[-1] else file_name + ".dds"
    dds.write_dds(out_name, variant, w, h, [data])
    log("DDS output to disk took: %.3f ms" % ((time.perf_counter() - t0) * 1e3))
    return out_name


HELP = """Usage: python -m block_compression_b200.cli <compression_variant> <input_file>

Compression variants:
  bc1  - BC1 compression (RGB)
  bc2  - BC2 compression with sharp alpha (RGBA)
  bc3  - BC3 compression with smooth alpha (RGBA)
  bc4  - BC4 compression (R)
  bc5  - BC5 compression (RG)
  bc6h - BC6H compression (RGB HDR)
  bc7  - BC7 compression with smooth alpha (RGBA)"""


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 2 or "--help" in argv:
        print(HELP)
        return 1
    if _variant(argv[0]) is None:
        print("Error: Invalid compression variant")
        print(HELP)
        return 1
    compress_file(argv[0], argv[1])
    return 0


if __name__ == "__main__":
    sys.exit(main())
