"""Generates the golden fixtures in this folder from the reference sources.

Run where the reference crate (novacrazy/block_compression v0.3.0) is
checked out, giving its path as the first argument or in BCN_REFERENCE_DIR:
`python tests/golden/make_golden.py <reference checkout>`. The fixtures are
committed; nothing at test time reads the reference tree.

Outputs
  decoder_kat.json      the 18 known-answer tests of src/decode/block.rs:1405-1841
  decoder_tables.json   BPTC partition-set tables of the decoders (block.rs:279-312, :810-947)
  encoder_tables.json   packed pattern / mask / anchor tables (src/encode/common.rs:23-101)
  settings_presets.json BC6H/BC7 quality presets (src/settings.rs:207-442)
"""
import json
import os
import re
import struct
import sys

REF = None
HERE = os.path.dirname(os.path.abspath(__file__))


def _ints(text):
    return [int(v, 0) for v in re.findall(r"0x[0-9A-Fa-f]+|\b\d+\b", text)]


def decoder_kats(block_rs):
    tests_src = block_rs[block_rs.index("mod tests {"):]
    out = []
    for m in re.finditer(r"fn (test_\w+)\(\) \{(.*?)\n    \}\n", tests_src, re.S):
        name, body = m.group(1), m.group(2)
        comp = re.search(r"let compressed_block = \[(.*?)\];", body, re.S).group(1)
        rep = re.fullmatch(r"\s*(\w+?)(?:u8)?;\s*(\d+)\s*", comp)  # `[0u8; 8]` repeat form
        compressed = [int(rep.group(1), 0)] * int(rep.group(2)) if rep else _ints(comp)
        entry = {"name": name, "compressed": compressed}
        if "f16::from_bits" in body:
            exp = re.findall(r"f16::from_bits\((0x[0-9A-Fa-f]+)\)", body)
            entry.update(kind="bc6h_half", pitch=12, is_signed=True,
                         expected=[int(v, 16) for v in exp])
        elif "decode_block_bc6h_float" in body:
            arr = re.search(r"let expected_output: \[f32; 48\] = \[(.*?)\];", body, re.S).group(1)
            vals = [float(v) for v in re.findall(r"-?\d+\.\d+", arr)]
            # f32 bit patterns of the Rust literals (nearest f32 to the decimal text)
            bits = [struct.unpack("<I", struct.pack("<f", v))[0] for v in vals]
            entry.update(kind="bc6h_float", pitch=12, is_signed=True, expected_f32_bits=bits)
        else:
            arr = re.search(r"let expected_output = \[(.*?)\];", body, re.S).group(1)
            call = re.search(r"test_block\(\s*(decode_block_\w+),\s*(\d+),", body, re.S)
            entry.update(kind=call.group(1).replace("decode_block_", ""), pitch=int(call.group(2)),
                         expected=_ints(arr))
        out.append(entry)
    return out


def partition_sets(block_rs, start_marker, count):
    i = block_rs.index(start_marker)
    rows = re.findall(r"\[\[(\d+), (\d+), (\d+), (\d+)\], \[(\d+), (\d+), (\d+), (\d+)\], "
                      r"\[(\d+), (\d+), (\d+), (\d+)\], \[(\d+), (\d+), (\d+), (\d+)\]\]",
                      block_rs[i:])
    return [[int(v) for v in r] for r in rows[:count]]


def encoder_tables(common_rs):
    def arr(name):
        m = re.search(name + r": \[u32; 128\] = \[(.*?)\];", common_rs, re.S)
        vals = [int(v, 16) for v in re.findall(r"0x[0-9A-Fa-f]+", m.group(1))]
        assert len(vals) == 128
        return vals
    return {"pattern": arr("PATTERN_TABLE"), "pattern_mask": arr("PATTERN_MASK_TABLE"),
            "skip": arr("SKIP_TABLE")}


def presets(settings_rs):
    out = {}
    for m in re.finditer(r"pub const fn (\w+)\(\) -> Self \{\s*Self \{(.*?)\n        \}", settings_rs, re.S):
        name, body = m.group(1), m.group(2)
        fields = {}
        for f in re.finditer(r"(\w+): (\[[^\]]*\]|[^,\n]+),", body):
            key, val = f.group(1), f.group(2).strip()
            conv = lambda t: 1 if t.strip().startswith("true") else (0 if t.strip().startswith("false") else int(t))
            if val.startswith("["):
                fields[key] = [conv(t) for t in val[1:-1].split(",")]
            else:
                fields[key] = conv(val)
        kind = "bc6h" if "slow_mode" in fields else "bc7"
        out.setdefault(kind, {})[name] = fields
    return out


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BCN_REFERENCE_DIR")
    if not REF:
        sys.exit("usage: make_golden.py <reference checkout> (or set BCN_REFERENCE_DIR)")
    block_rs = open(os.path.join(REF, "src/decode/block.rs")).read()
    common_rs = open(os.path.join(REF, "src/encode/common.rs")).read()
    settings_rs = open(os.path.join(REF, "src/settings.rs")).read()
    kats = decoder_kats(block_rs)
    assert len(kats) == 18, len(kats)
    json.dump(kats, open(os.path.join(HERE, "decoder_kat.json"), "w"), indent=1)
    tables = {
        "bc6h_partition_sets": partition_sets(block_rs, "static PARTITION_SETS: &[[[u8; 4]; 4]; 32]", 32),
        "bc7_partition_sets_2": partition_sets(block_rs, "// Partition table for 2-subset BPTC", 64),
        "bc7_partition_sets_3": partition_sets(block_rs, "// Partition table for 3-subset BPTC", 64),
    }
    for k, v in tables.items():
        assert all(len(r) == 16 for r in v), k
    json.dump(tables, open(os.path.join(HERE, "decoder_tables.json"), "w"))
    json.dump(encoder_tables(common_rs), open(os.path.join(HERE, "encoder_tables.json"), "w"))
    p = presets(settings_rs)
    assert len(p["bc6h"]) == 5 and len(p["bc7"]) == 10, p.keys()
    json.dump(p, open(os.path.join(HERE, "settings_presets.json"), "w"), indent=1)
    print("wrote", len(kats), "decoder KATs and tables to", HERE)


if __name__ == "__main__":
    sys.exit(main())
