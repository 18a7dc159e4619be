"""CPU oracle — TEST INFRASTRUCTURE ONLY.

ctypes binding of ``liboracle.so``, the C++ restatement of the reference
crate's CPU codec (novacrazy/block_compression v0.3.0). Only the tests, the
smoke check and the bench's CPU-baseline leg import this module, and only as
the checker / the timed CPU baseline. The product package never imports it.

Variant ids follow the reference enum order (src/lib.rs:74-103):
0 BC1, 1 BC2, 2 BC3, 3 BC4, 4 BC5, 5 BC6H, 6 BC7.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

BLOCK_BYTES = {0: 8, 1: 16, 2: 16, 3: 8, 4: 16, 5: 16, 6: 16}


def build(force=False):
    """Compiles liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    srcs = [f for f in os.listdir(_HERE) if f.endswith((".cpp", ".h"))] + ["Makefile"]
    newest = max(os.path.getmtime(os.path.join(_HERE, f)) for f in srcs)
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < newest:
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "liboracle.so"],
                       check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P, S, U32, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_int
        L.oracle_compress_rgba8.argtypes = [I, P, P, S, P, S, U32, U32, U32, I]
        L.oracle_compress_rgba16.argtypes = [P, P, S, P, S, U32, U32, U32, I]
        L.oracle_decompress_rgba8.argtypes = [I, U32, U32, P, S, P, S, I]
        L.oracle_decompress_rgba16f.argtypes = [U32, U32, P, S, P, S]
        L.oracle_decompress_rgba32f.argtypes = [U32, U32, P, S, P, S]
        L.oracle_decode_block.argtypes = [I, P, P, S, I]
        L.oracle_decode_block.restype = None
        for name in ("oracle_encode_block_bc1", "oracle_encode_block_bc3_alpha"):
            getattr(L, name).argtypes = [P, P]
            getattr(L, name).restype = None
        for name in ("oracle_encode_block_bc7", "oracle_encode_block_bc6h"):
            getattr(L, name).argtypes = [P, P, P]
            getattr(L, name).restype = None
        L.oracle_block_quant.argtypes = [P, P, U32, P, U32, U32]
        L.oracle_block_quant.restype = ctypes.c_float
        L.oracle_opt_endpoints.argtypes = [P, P, U32, P, U32, U32]
        L.oracle_opt_endpoints.restype = None
        L.oracle_block_pca_bound_split.argtypes = [P, U32, U32]
        L.oracle_block_pca_bound_split.restype = ctypes.c_float
        L.oracle_block_segment_core.argtypes = [P, P, U32, U32]
        L.oracle_block_segment_core.restype = None
        L.oracle_ep_quant_dequant.argtypes = [P, P, U32, U32]
        L.oracle_ep_quant_dequant.restype = None
        for name in ("oracle_get_pattern", "oracle_get_skip_packed"):
            getattr(L, name).argtypes = [ctypes.c_int32]
            getattr(L, name).restype = U32
        L.oracle_get_pattern_mask.argtypes = [ctypes.c_int32, U32]
        L.oracle_get_pattern_mask.restype = U32
        L.oracle_partition_set.argtypes = [U32, U32]
        L.oracle_partition_set.restype = U32
        L.oracle_f32_to_f16.argtypes = [ctypes.c_float]
        L.oracle_f32_to_f16.restype = ctypes.c_uint16
        L.oracle_f16_to_f32.argtypes = [ctypes.c_uint16]
        L.oracle_f16_to_f32.restype = ctypes.c_float
        L.oracle_linear_to_srgb.argtypes = [ctypes.c_float]
        L.oracle_linear_to_srgb.restype = ctypes.c_uint8
        for name in ("oracle_bc7_parse", "oracle_bc1_parse"):
            getattr(L, name).argtypes = [P, S, P, P]
            getattr(L, name).restype = None
        for name in ("oracle_bc7_relaxed_f64", "oracle_bc7_adjoint_f64", "oracle_bc1_relaxed_f64",
                     "oracle_bc1_adjoint_f64"):
            getattr(L, name).argtypes = [P, P, S, P]
            getattr(L, name).restype = None
        L.oracle_bc7_refine_block.argtypes = [P, P, U32, U32, ctypes.c_float, P, P]
        L.oracle_bc7_refine_block.restype = None
        L.oracle_bc1_refine_block.argtypes = [P, P, U32, ctypes.c_float, P, P]
        L.oracle_bc1_refine_block.restype = None
        L.oracle_check_div_count.argtypes = []
        L.oracle_check_div_count.restype = ctypes.c_uint64
        L.oracle_check_div_const.argtypes = [ctypes.c_float, ctypes.c_int]
        L.oracle_check_div_const.restype = ctypes.c_uint64
        L.oracle_check_div_int_pairs.argtypes = [ctypes.c_int]
        L.oracle_check_div_int_pairs.restype = ctypes.c_uint64
        L.oracle_check_div_channel.argtypes = []
        L.oracle_check_div_channel.restype = ctypes.c_uint64
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _settings_ptr(settings):
    if settings is None:
        return None, None
    arr = np.ascontiguousarray(np.asarray(settings, dtype=np.uint32))
    return arr, _ptr(arr)


def compress_rgba8(variant, rgba, width, height, stride=None, settings=None, threads=None):
    """encode::compress_rgba8 (src/encode.rs:83); rgba is a uint8 buffer."""
    rgba = np.ascontiguousarray(rgba, dtype=np.uint8).reshape(-1)
    stride = width * 4 if stride is None else stride
    n = ((width + 3) // 4) * ((height + 3) // 4) * BLOCK_BYTES[variant]
    out = np.zeros(n, dtype=np.uint8)
    keep, sp = _settings_ptr(settings)
    rc = lib().oracle_compress_rgba8(variant, sp, _ptr(rgba), rgba.size, _ptr(out), out.size,
                                     width, height, stride, threads or os.cpu_count())
    if rc != 0:
        raise ValueError("oracle_compress_rgba8 failed with status %d" % rc)
    return out


def compress_rgba16(rgba16, width, height, settings, stride=None, threads=None):
    """encode::compress_rgba16 (src/encode.rs:211); rgba16 holds f16 bit patterns (uint16)."""
    rgba16 = np.ascontiguousarray(rgba16).view(np.uint16).reshape(-1)
    stride = width * 4 if stride is None else stride
    n = ((width + 3) // 4) * ((height + 3) // 4) * 16
    out = np.zeros(n, dtype=np.uint8)
    keep, sp = _settings_ptr(settings)
    rc = lib().oracle_compress_rgba16(sp, _ptr(rgba16), rgba16.size, _ptr(out), out.size,
                                      width, height, stride, threads or os.cpu_count())
    if rc != 0:
        raise ValueError("oracle_compress_rgba16 failed with status %d" % rc)
    return out


def decompress_rgba8(variant, blocks, width, height, threads=None):
    blocks = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1)
    out = np.zeros(width * height * 4, dtype=np.uint8)
    rc = lib().oracle_decompress_rgba8(variant, width, height, _ptr(blocks), blocks.size, _ptr(out),
                                       out.size, threads or os.cpu_count())
    if rc != 0:
        raise ValueError("oracle_decompress_rgba8 failed with status %d" % rc)
    return out


def decompress_rgba16f(blocks, width, height, out=None):
    blocks = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1)
    out = np.zeros(width * height * 4, dtype=np.uint16) if out is None else out
    rc = lib().oracle_decompress_rgba16f(width, height, _ptr(blocks), blocks.size, _ptr(out), out.size)
    if rc != 0:
        raise ValueError("oracle_decompress_rgba16f failed with status %d" % rc)
    return out


def decompress_rgba32f(blocks, width, height, out=None):
    blocks = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1)
    out = np.zeros(width * height * 4, dtype=np.float32) if out is None else out
    rc = lib().oracle_decompress_rgba32f(width, height, _ptr(blocks), blocks.size, _ptr(out), out.size)
    if rc != 0:
        raise ValueError("oracle_decompress_rgba32f failed with status %d" % rc)
    return out


DECODE_KIND = {"bc1": 0, "bc2": 1, "bc3": 2, "bc4": 3, "bc5": 4, "bc6h_half": 5, "bc6h_float": 6, "bc7": 7}


def decode_block(kind, block, out, pitch, is_signed=False):
    """Per-block decoders of src/decode/block.rs; `out` is written in place."""
    block = np.ascontiguousarray(block, dtype=np.uint8)
    lib().oracle_decode_block(DECODE_KIND[kind], _ptr(block), _ptr(out), pitch, int(is_signed))
    return out


def planar_block(rgba16px):
    """4x4 RGBA pixels (uint8, shape (16, 4) row-major) -> planar f32[64]."""
    px = np.asarray(rgba16px, dtype=np.float32).reshape(16, 4)
    return np.ascontiguousarray(px.T.reshape(64))


def encode_block_bc1(block):
    out = np.zeros(2, dtype=np.uint32)
    lib().oracle_encode_block_bc1(_ptr(np.ascontiguousarray(block, np.float32)), _ptr(out))
    return out


def encode_block_bc3_alpha(block):
    out = np.zeros(2, dtype=np.uint32)
    lib().oracle_encode_block_bc3_alpha(_ptr(np.ascontiguousarray(block, np.float32)), _ptr(out))
    return out


def encode_block_bc7(block, settings):
    out = np.zeros(4, dtype=np.uint32)
    keep, sp = _settings_ptr(settings)
    lib().oracle_encode_block_bc7(_ptr(np.ascontiguousarray(block, np.float32)), sp, _ptr(out))
    return out


def encode_block_bc6h(block, settings):
    out = np.zeros(4, dtype=np.uint32)
    keep, sp = _settings_ptr(settings)
    lib().oracle_encode_block_bc6h(_ptr(np.ascontiguousarray(block, np.float32)), sp, _ptr(out))
    return out


_count_lib = None


def count_lib():
    """The op-counting build (liboracle_count.so): per-block FP32 op counts of
    the reference encoders, the algorithmic work of the BC6H/BC7 rooflines."""
    global _count_lib
    if _count_lib is None:
        path = os.path.join(_HERE, "liboracle_count.so")
        srcs = [f for f in os.listdir(_HERE) if f.endswith((".cpp", ".h"))] + ["Makefile"]
        newest = max(os.path.getmtime(os.path.join(_HERE, f)) for f in srcs)
        if not os.path.exists(path) or os.path.getmtime(path) < newest:
            subprocess.run(["make", "-s", "-C", _HERE, "liboracle_count.so"], check=True)
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        for name, args in (("oracle_count_bc7", [P, P]), ("oracle_count_bc6h", [P, P]),
                           ("oracle_count_bc1", [P]), ("oracle_count_bc3_alpha", [P])):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_uint64
        _count_lib = L
    return _count_lib


def count_ops(kind, block, settings=None):
    """FP32 ops of one block: kind in bc1, bc3_alpha, bc6h, bc7."""
    L = count_lib()
    b = np.ascontiguousarray(block, dtype=np.float32)
    if kind in ("bc1", "bc3_alpha"):
        return getattr(L, "oracle_count_" + kind)(_ptr(b))
    keep, sp = _settings_ptr(settings)
    return getattr(L, "oracle_count_" + kind)(_ptr(b), sp)


# ---- relaxed (differentiable) decode and endpoint refinement ----------------------
# Layouts: BC7 meta (n, 8) uint32 + endpoints (n, 24); BC1 meta (n, 2) +
# endpoints (n, 6); relaxed pixels and gradients (n, 16, 4).

_META_WORDS = {"bc7": 8, "bc1": 2}
_EP_COUNT = {"bc7": 24, "bc1": 6}
_BLOCK = {"bc7": 16, "bc1": 8}


def parse(kind, blocks):
    """Parses n blocks (uint8, n * 8 or n * 16 bytes) -> (meta uint32, endpoints float32)."""
    b = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1)
    n = b.size // _BLOCK[kind]
    meta = np.zeros((n, _META_WORDS[kind]), dtype=np.uint32)
    ep = np.zeros((n, _EP_COUNT[kind]), dtype=np.float32)
    getattr(lib(), "oracle_%s_parse" % kind)(_ptr(b), n, _ptr(meta), _ptr(ep))
    return meta, ep


def relaxed_f64(kind, meta, endpoints):
    """FP64 relaxed decode -> (n, 16, 4) float64."""
    meta = np.ascontiguousarray(meta, dtype=np.uint32)
    ep = np.ascontiguousarray(endpoints, dtype=np.float64)
    n = meta.shape[0]
    out = np.zeros((n, 16, 4), dtype=np.float64)
    getattr(lib(), "oracle_%s_relaxed_f64" % kind)(_ptr(meta), _ptr(ep), n, _ptr(out))
    return out


def adjoint_f64(kind, meta, grad):
    """FP64 adjoint of the relaxed decode -> (n, endpoints) float64."""
    meta = np.ascontiguousarray(meta, dtype=np.uint32)
    g = np.ascontiguousarray(grad, dtype=np.float64)
    n = meta.shape[0]
    out = np.zeros((n, _EP_COUNT[kind]), dtype=np.float64)
    getattr(lib(), "oracle_%s_adjoint_f64" % kind)(_ptr(meta), _ptr(g), n, _ptr(out))
    return out


def refine_blocks(kind, blocks, src_blocks, steps, lr, channels=4):
    """Sequential restatement of the refinement kernels, block by block.
    blocks: (n, 8|16) uint8 (copied); src_blocks: (n, 16, 4) uint8 source
    pixels per block. Returns (refined blocks, final endpoints, errors (n, 2))."""
    L = lib()
    out = np.array(blocks, dtype=np.uint8).reshape(-1, _BLOCK[kind]).copy()
    src = np.ascontiguousarray(src_blocks, dtype=np.uint8).reshape(-1, 64)
    n = out.shape[0]
    theta = np.zeros((n, _EP_COUNT[kind]), dtype=np.float32)
    errs = np.zeros((n, 2), dtype=np.uint32)
    for i in range(n):
        bi = out[i]
        if kind == "bc7":
            L.oracle_bc7_refine_block(_ptr(bi), _ptr(src[i]), channels, steps, lr, _ptr(theta[i]), _ptr(errs[i]))
        else:
            L.oracle_bc1_refine_block(_ptr(bi), _ptr(src[i]), steps, lr, _ptr(theta[i]), _ptr(errs[i]))
    return out, theta, errs


def image_blocks(rgba, width, height):
    """(h, w, 4) uint8 image -> (n, 16, 4) source pixels, blocks row-major."""
    img = np.asarray(rgba, dtype=np.uint8).reshape(height, width, 4)
    t = img.reshape(height // 4, 4, width // 4, 4, 4).transpose(0, 2, 1, 3, 4)
    return np.ascontiguousarray(t.reshape(-1, 16, 4))
