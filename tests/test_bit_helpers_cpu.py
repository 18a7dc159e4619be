"""Integer helpers of the device headers compiled for the host with nvcc and
checked against their per-field definitions (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "block_compression_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include "bc_common.cuh"

static uint32_t by_field(uint32_t map, uint32_t subset) {
    uint32_t m = 0;
    for (int k = 0; k < 16; k++) m |= (((map >> (2 * k)) & 3u) == subset ? 1u : 0u) << k;
    return m;
}

int main() {
    unsigned long long bad = 0, n = 0;
    // every field value at every position, the other fields held at each value
    for (uint32_t fill = 0; fill < 4; fill++)
        for (int pos = 0; pos < 16; pos++)
            for (uint32_t v = 0; v < 4; v++)
                for (uint32_t s = 0; s < 4; s++) {
                    uint32_t map = (fill * 0x55555555u & ~(3u << (2 * pos))) | (v << (2 * pos));
                    bad += bcn::subset_mask_from_map(map, s) != by_field(map, s);
                    n++;
                }
    // random maps (xorshift)
    uint32_t x = 2463534242u;
    for (int i = 0; i < 4000000; i++) {
        x ^= x << 13; x ^= x >> 17; x ^= x << 5;
        for (uint32_t s = 0; s < 4; s++) {
            bad += bcn::subset_mask_from_map(x, s) != by_field(x, s);
            n++;
        }
    }
    std::printf("%llu %llu\n", bad, n);
    return bad != 0;
}
"""


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    return None


def test_subset_mask_from_map_matches_per_field_definition(tmp_path):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    src = tmp_path / "mask_check.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "mask_check"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-I", CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    bad, n = map(int, r.stdout.split())
    assert r.returncode == 0 and bad == 0 and n == 1024 + 16000000
