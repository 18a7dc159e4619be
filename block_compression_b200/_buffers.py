"""Raw-pointer views of the buffer types the Python API accepts: numpy arrays,
bytes/bytearray/memoryview (host) and torch tensors (host or CUDA)."""
import ctypes

import numpy as np


class Buf:
    __slots__ = ("ptr", "nbytes", "cuda", "keep")

    def __init__(self, ptr, nbytes, cuda, keep):
        self.ptr = ptr
        self.nbytes = nbytes
        self.cuda = cuda
        self.keep = keep


def view(obj, writable=False):
    """Returns a Buf for `obj`. CUDA tensors must be contiguous."""
    mod = type(obj).__module__
    if mod.startswith("torch"):
        if not obj.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return Buf(obj.data_ptr(), obj.numel() * obj.element_size(), obj.is_cuda, obj)
    if isinstance(obj, np.ndarray):
        if not obj.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        if writable and not obj.flags["WRITEABLE"]:
            raise ValueError("array is read-only")
        return Buf(obj.ctypes.data, obj.nbytes, False, obj)
    if isinstance(obj, bytes):
        if writable:
            raise ValueError("bytes is read-only")
        arr = np.frombuffer(obj, dtype=np.uint8)
        return Buf(arr.ctypes.data, arr.nbytes, False, arr)
    if isinstance(obj, (bytearray, memoryview)):
        arr = np.frombuffer(obj, dtype=np.uint8)
        return Buf(arr.ctypes.data, arr.nbytes, False, arr)
    raise TypeError("unsupported buffer type %r" % type(obj))


def current_stream_ptr():
    """cudaStream_t of torch's current stream (None if torch/CUDA absent)."""
    try:
        import torch
    except ImportError:
        return None
    if not torch.cuda.is_available():
        return None
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
