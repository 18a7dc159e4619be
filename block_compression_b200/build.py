"""Builds the sm_100a shared library ``libbcn_b200.so`` in-tree.

Every kernel translation unit is compiled by nvcc for sm_100a with the float
flags the bit-exactness argument depends on:
  --fmad=false                    no FMA contraction (the reference never fuses)
  -prec-div=true -prec-sqrt=true  IEEE division and square root
  (no --use_fast_math, denormals kept)
`--check` builds the bounds-checked debug variant libbcn_b200_check.so
(-DBCN_CHECK: every guarded index compared with its array's extent, failures
recorded for bc_check_read() instead of trapping).
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbcn_b200.so")
BUILD_CHECK = os.path.join(HERE, "_build_check")
LIB_CHECK = os.path.join(HERE, "libbcn_b200_check.so")
SOURCES = ["bc15.cu", "bc7_encode.cu", "bc6h_encode.cu", "bc_decode.cu", "capi.cu", "batch.cu", "mips.cu", "refine.cu",
           "metrics.cu", "dds.cu"]
HEADERS = ["bc_common.cuh", "bptc_math.cuh", "bc_kernels.h", "bc7_device.cuh", "bptc_decode.cuh", "bc1_block.cuh",
           "bc_relaxed.cuh", "bc_check.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(force=False, verbose=False, check=False):
    """Compiles what changed and links the library; returns its path.
    check=True builds the bounds-checked debug variant
    (libbcn_b200_check.so, objects in _build_check/, -DBCN_CHECK)."""
    out_dir = BUILD_CHECK if check else BUILD
    lib_path = LIB_CHECK if check else LIB
    flags = NVCC_FLAGS + (["-DBCN_CHECK"] if check else [])
    os.makedirs(out_dir, exist_ok=True)
    include = os.path.join(os.path.dirname(HERE), "include")
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(include, "bc_capi.h")]
    hdr_time = _newest(hdrs)
    nvcc = _nvcc()
    jobs = []
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(out_dir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            jobs.append([nvcc] + flags + ["-I", include, "-c", s, "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
        return r.stderr

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not os.path.exists(lib_path) or os.path.getmtime(lib_path) < _newest(objs):
        tmp = lib_path + ".tmp"
        run([nvcc, "-shared", "-o", tmp] + objs + ["-lcudart"])
        os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, check="--check" in sys.argv))
