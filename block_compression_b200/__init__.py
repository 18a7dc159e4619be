"""block_compression_b200 — BCn (BC1-BC7) texture block compression on B200.

A drop-in for the per-4x4-block codec of the Rust crate block_compression
v0.3.0: the CPU encode/decode entry points (`encode`, `decode`), the BC6H/BC7
quality profiles, and the GpuBlockCompressor task interface, all executed by
hand-written sm_100a kernels in libbcn_b200.so behind a C ABI
(include/bc_capi.h). There is no CPU fallback: importing the package fails if
the library is missing.
"""
from ._lib import BcError, lib  # noqa: F401  (loads libbcn_b200.so or raises)
from .compressor import Batch, GpuBlockCompressor, Tune
from .settings import BC6HSettings, BC7Settings, CompressionVariant
from . import decode, encode

__all__ = ["BC6HSettings", "BC7Settings", "CompressionVariant", "GpuBlockCompressor", "Batch", "Tune", "BcError",
           "encode", "decode", "version"]


def version():
    return lib.bc_version().decode()
