"""ctypes binding of libbcn_b200.so (the C ABI declared in include/bc_capi.h).

The shared library is the only implementation: there is no CPU fallback. If
it is missing or fails to load, importing the package raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbcn_b200.so")

BC_OK = 0
STATUS_NAMES = {
    -1: "BC_ERR_DIMS",
    -2: "BC_ERR_DST_SIZE",
    -3: "BC_ERR_SRC_SIZE",
    -4: "BC_ERR_VARIANT",
    -5: "BC_ERR_SETTINGS",
    -6: "BC_ERR_NULL",
    -7: "BC_ERR_CUDA",
    -8: "BC_ERR_TASKS",
    -9: "BC_ERR_NO_DEVICE",
    -10: "BC_ERR_TOO_LARGE",
}


class BcError(RuntimeError):
    """A C-ABI call returned a negative status (the reference would panic)."""

    def __init__(self, func, status, detail=""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        msg = "%s failed: %s" % (func, name)
        if detail:
            msg += " (%s)" % detail
        super().__init__(msg)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            "libbcn_b200.so is not built; run `python block_compression_b200/build.py` "
            "(nvcc with sm_100a support is required)")
    L = ctypes.CDLL(LIB_PATH)
    P, S, U32, I = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_int
    sig = {
        "bc_bc6h_settings_preset": ([ctypes.c_char_p, P], I),
        "bc_bc7_settings_preset": ([ctypes.c_char_p, P], I),
        "bc_bytes_per_row": ([I, U32], U32),
        "bc_blocks_byte_size": ([I, U32, U32], S),
        "bc_compress_rgba8": ([I, P, P, S, P, S, U32, U32, U32], I),
        "bc_compress_rgba16": ([I, P, P, S, P, S, U32, U32, U32], I),
        "bc_compress_rgba8_device": ([I, P, P, S, P, S, U32, U32, S, P], I),
        "bc_compress_rgba16_device": ([P, P, S, P, S, U32, U32, S, P], I),
        "bc_decompress_blocks_as_rgba8": ([I, U32, U32, P, S, P, S], I),
        "bc_decompress_blocks_as_rgba16f": ([I, U32, U32, P, S, P, S], I),
        "bc_decompress_blocks_as_rgba32f": ([I, U32, U32, P, S, P, S], I),
        "bc_decompress_device": ([I, U32, U32, P, S, P, S, I, P], I),
        "bc_decode_block_min_len": ([I, S], S),
        "bc_decode_block_bc1": ([P, S, P, S, S], I),
        "bc_decode_block_bc2": ([P, S, P, S, S], I),
        "bc_decode_block_bc3": ([P, S, P, S, S], I),
        "bc_decode_block_bc4": ([P, S, P, S, S], I),
        "bc_decode_block_bc5": ([P, S, P, S, S], I),
        "bc_decode_block_bc6h": ([P, S, P, S, S, I], I),
        "bc_decode_block_bc6h_float": ([P, S, P, S, S, I], I),
        "bc_decode_block_bc7": ([P, S, P, S, S], I),
        "bc_decode_blocks_device": ([I, I, P, S, P, S, S, S, P], I),
        "bc_compressor_create": ([I, ctypes.POINTER(P)], I),
        "bc_compressor_destroy": ([P], I),
        "bc_compressor_add_task": ([P, I, P, P, S, S, U32, U32, U32, P, S, U32], I),
        "bc_compressor_compress": ([P, P], I),
        "bc_compressor_task_count": ([P], I),
        "bc_batch_create": ([P, P, I, P, ctypes.POINTER(P)], I),
        "bc_batch_launch": ([P, P], I),
        "bc_batch_get_tune": ([P, P], I),
        "bc_batch_destroy": ([P], I),
        "bc_compressor_compress_batched": ([P, P, P], I),
        "bc_compress_bc7_device_noalloc": ([P, P, S, P, S, U32, U32, S, P], I),
        "bc_mip_level_rgba8_device": ([P, S, U32, U32, P, S, S, P], I),
        "bc_bc7_parse_device": ([P, S, P, P, P], I),
        "bc_bc7_decode_relaxed_device": ([P, P, S, P, P], I),
        "bc_bc7_decode_adjoint_device": ([P, P, S, P, P], I),
        "bc_bc1_parse_device": ([P, S, P, P, P], I),
        "bc_bc1_decode_relaxed_device": ([P, P, S, P, P], I),
        "bc_bc1_decode_adjoint_device": ([P, P, S, P, P], I),
        "bc_bc7_refine_device": ([P, S, U32, U32, P, S, U32, U32, ctypes.c_float, P, P, P], I),
        "bc_bc1_refine_device": ([P, S, U32, U32, P, S, U32, ctypes.c_float, P, P, P], I),
        "bc_bc7_refine_images_device": ([P, U32, U32, U32, ctypes.c_float, P, P], I),
        "bc_bc1_refine_images_device": ([P, U32, U32, ctypes.c_float, P, P], I),
        "bc_image_sse_rgba8_device": ([P, S, P, S, U32, U32, U32, P, P], I),
        "bc_bc6h_error_device": ([P, S, S, P, S, U32, U32, P, P, P], I),
        "bc_dds_header": ([I, U32, U32, U32, I, P, S], I),
        "bc_dds_dxgi_format": ([I, I], U32),
        "bc_last_cuda_error": ([], I),
        "bc_check_enabled": ([], I),
        "bc_check_read": ([P], I),
        "bc_check_selftest": ([ctypes.c_uint64, ctypes.c_uint64, P], I),
        "bc_version": ([], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L


lib = _load()


def check(func, status):
    if status != BC_OK:
        detail = ""
        if status == -7:
            detail = "cudaError %d" % lib.bc_last_cuda_error()
        raise BcError(func, status, detail)
    return status
