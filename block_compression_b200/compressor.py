"""GpuBlockCompressor: the reference's task interface
(src/block_compressor.rs:44-590) over CUDA device buffers.

Tasks are added one per texture / mip / row range, then `compress()` enqueues
them all on one CUDA stream and drains the queue, like the reference's
compress(&mut ComputePass).
"""
import ctypes

from . import _buffers
from ._lib import check, lib


class GpuBlockCompressor:
    def __init__(self, device=-1):
        """GpuBlockCompressor::new (src/block_compressor.rs:66). `device` is a
        CUDA ordinal (-1: the current device)."""
        h = ctypes.c_void_p()
        check("bc_compressor_create", lib.bc_compressor_create(int(device), ctypes.byref(h)))
        self._h = h
        self._keep = []  # keeps task buffers and settings alive until compress()

    def add_compression_task(self, variant, texture, width, height, buffer, texture_y_offset=None,
                             blocks_offset=None, row_pitch=None):
        """GpuBlockCompressor::add_compression_task (src/block_compressor.rs:342).

        texture: CUDA tensor holding the source texture (RGBA8 rows for
          BC1-BC5/BC7, RGBA16F rows for BC6H), row 0 first; row_pitch is its
          row size in bytes (default: the tensor's last two dims, i.e. rows of
          the full texture width when shaped (H, W, 4)).
        buffer: CUDA uint8 tensor receiving the blocks.
        texture_y_offset / blocks_offset: as the reference's Option<u32> (rows;
          bytes)."""
        src = _buffers.view(texture)
        dst = _buffers.view(buffer, writable=True)
        if not (src.cuda and dst.cuda):
            raise ValueError("texture and buffer must be CUDA tensors")
        if row_pitch is None:
            if texture.dim() >= 3:
                row_pitch = texture.shape[-2] * texture.shape[-1] * texture.element_size()
            else:
                row_pitch = width * (8 if variant.id == 5 else 4)
        self._keep.append((texture, buffer, variant.settings))
        check("bc_compressor_add_task",
              lib.bc_compressor_add_task(self._h, variant.id, variant.settings_ptr(), src.ptr, row_pitch, src.nbytes,
                                         width, height, texture_y_offset or 0, dst.ptr, dst.nbytes,
                                         blocks_offset or 0))

    def compress(self, stream=None):
        """GpuBlockCompressor::compress (src/block_compressor.rs:540): enqueue
        every pending task on `stream` (default: torch's current stream)."""
        s = stream if stream is not None else _buffers.current_stream_ptr()
        try:
            check("bc_compressor_compress", lib.bc_compressor_compress(self._h, s))
        finally:
            self._keep.clear()

    def task_count(self):
        return lib.bc_compressor_task_count(self._h)

    def close(self):
        if self._h:
            lib.bc_compressor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tune(ctypes.Structure):
    """Launch shape of a batch (include/bc_capi.h, bc_tune)."""

    _fields_ = [("threads_per_cta", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_uint32),
                ("tiles_per_claim", ctypes.c_uint32), ("bc7_search_warps", ctypes.c_uint32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Batch:
    """Every pending task of a GpuBlockCompressor frozen into one device task
    table and one CUDA graph (bc_batch). launch() replays it."""

    def __init__(self, compressor, tune=None, autotune=True, stream=None):
        s = stream if stream is not None else _buffers.current_stream_ptr()
        h = ctypes.c_void_p()
        tp = ctypes.byref(tune) if tune is not None else None
        check("bc_batch_create", lib.bc_batch_create(compressor._h, tp, int(bool(autotune)), s, ctypes.byref(h)))
        self._h = h
        self._keep = list(compressor._keep)  # the tasks' buffers must outlive the batch
        compressor._keep.clear()

    def launch(self, stream=None):
        s = stream if stream is not None else _buffers.current_stream_ptr()
        check("bc_batch_launch", lib.bc_batch_launch(self._h, s))

    @property
    def tune(self):
        t = Tune()
        check("bc_batch_get_tune", lib.bc_batch_get_tune(self._h, ctypes.byref(t)))
        return t

    def close(self):
        if self._h:
            lib.bc_batch_destroy(self._h)
            self._h = None
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _compress_batched(self, stream=None, tune=None):
    """All pending tasks in one batched graph launch (autotuned unless `tune`
    is given); synchronises the stream before returning."""
    s = stream if stream is not None else _buffers.current_stream_ptr()
    tp = ctypes.byref(tune) if tune is not None else None
    try:
        check("bc_compressor_compress_batched", lib.bc_compressor_compress_batched(self._h, s, tp))
    finally:
        self._keep.clear()


def _create_batch(self, tune=None, autotune=True, stream=None):
    return Batch(self, tune=tune, autotune=autotune, stream=stream)


GpuBlockCompressor.compress_batched = _compress_batched
GpuBlockCompressor.create_batch = _create_batch
