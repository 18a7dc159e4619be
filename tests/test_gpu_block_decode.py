"""Per-block decoders on the GPU (decode::decode_block_*, src/decode/block.rs:50-119,
262, 774, 801) against the reference's own known-answer tests and the oracle.

The 18 known-answer tests of src/decode/block.rs:1405-1841 (tests/golden/decoder_kat.json)
run through the CUDA decoders exactly as the reference runs them: a zeroed
64-byte (or 48-element) buffer, the test's pitch -- 8 for BC7, so rows overlap
and later writes win -- and the whole buffer compared. Random blocks at several
pitches, both BC6H signednesses, go through the device form and must leave the
same buffer contents as the oracle's per-block decoder, untouched elements
included.
"""
import json
import os
import zlib

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KATS = json.load(open(os.path.join(GOLDEN, "decoder_kat.json")))

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kat", KATS, ids=[k["name"] for k in KATS])
def test_reference_known_answers_on_cuda(bcn, cuda, kat):
    c = np.array(kat["compressed"], dtype=np.uint8)
    d = bcn.decode
    if kat["kind"] == "bc6h_half":
        out = np.zeros(48, np.uint16)
        d.decode_block_bc6h(c, out, kat["pitch"], kat["is_signed"])
        assert out.tolist() == kat["expected"]
    elif kat["kind"] == "bc6h_float":
        out = np.zeros(48, np.float32)
        d.decode_block_bc6h_float(c, out, kat["pitch"], kat["is_signed"])
        assert out.view(np.uint32).tolist() == kat["expected_f32_bits"]
    else:
        out = np.zeros(64, np.uint8)
        getattr(d, "decode_block_" + kat["kind"])(c, out, kat["pitch"])
        assert out.tolist() == kat["expected"]


# (kind, pitches): pitches below a decoded row's width make rows overlap
CASES = [("bc1", [16, 8, 4, 20]), ("bc2", [16, 8, 20]), ("bc3", [16, 8, 12, 20]), ("bc4", [4, 2, 1, 7]),
         ("bc5", [8, 4, 3, 9]), ("bc6h", [12, 6, 3, 16]), ("bc6h_float", [12, 6, 16]), ("bc7", [16, 8, 4, 20])]
ORACLE_KIND = {"bc6h": "bc6h_half"}
DTYPE = {"bc6h": np.uint16, "bc6h_float": np.float32}


def _random_blocks(rng, kind, n):
    size = 8 if kind in ("bc1", "bc4") else 16
    b = rng.integers(0, 256, (n, size), dtype=np.uint8)
    if kind == "bc7":  # every mode and the reserved mode byte equally often
        modes = rng.integers(0, 9, n)
        first = np.where(modes < 8, (1 << modes) & 0xFF, 0).astype(np.uint8)
        b[:, 0] = first | (b[:, 0] & ~((2 << modes) - 1).astype(np.uint8))
    return b


@pytest.mark.parametrize("kind,pitches", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("is_signed", [False, True], ids=["unsigned", "signed"])
def test_random_blocks_device_form_matches_oracle(bcn, oracle_lib, cuda, kind, pitches, is_signed):
    import torch
    if is_signed and not kind.startswith("bc6h"):
        pytest.skip("signedness applies to BC6H only")
    rng = np.random.default_rng(zlib.crc32(("%s/%d" % (kind, is_signed)).encode()))
    n = 700
    blocks = _random_blocks(rng, kind, n)
    dt = DTYPE.get(kind, np.uint8)
    for pitch in pitches:
        need = bcn.decode.block_min_len(kind, pitch)
        stride = need + 3  # gaps between blocks stay untouched
        init = rng.integers(0, 1 << (8 * np.dtype(dt).itemsize - 1), n * stride).astype(dt)
        exp = init.copy()
        for i in range(n):
            oracle_lib.decode_block(ORACLE_KIND.get(kind, kind), blocks[i], exp[i * stride:(i + 1) * stride], pitch,
                                    is_signed)
        out = torch.from_numpy(init.view(np.int16) if dt == np.uint16 else init).cuda()
        bcn.decode.decode_blocks(kind, torch.from_numpy(blocks.reshape(-1)).cuda(), out, pitch, stride,
                                 is_signed=is_signed)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(dt)
        bad = np.nonzero(got.view(np.uint8 if dt == np.uint8 else (np.uint16 if dt == np.uint16 else np.uint32))
                         != exp.view(np.uint8 if dt == np.uint8 else (np.uint16 if dt == np.uint16 else np.uint32)))[0]
        assert bad.size == 0, "%s pitch %d: %d elements differ, first at block %d" % (
            kind, pitch, bad.size, bad[0] // stride)


def test_host_form_keeps_untouched_elements(bcn, oracle_lib, cuda):
    """BC4 at pitch 4 writes one byte per texel; every other byte of the
    caller's buffer keeps its value, as with the reference's slice writes."""
    rng = np.random.default_rng(7)
    blk = rng.integers(0, 256, 8, dtype=np.uint8)
    buf = rng.integers(0, 256, 40, dtype=np.uint8)
    exp = buf.copy()
    oracle_lib.decode_block("bc4", blk, exp, 9)
    bcn.decode.decode_block_bc4(blk, buf, 9)
    assert buf.tolist() == exp.tolist()
