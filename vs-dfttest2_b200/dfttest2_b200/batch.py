"""Multi-clip batches: many device-resident clips, each with its own DFTTest
arguments, size, length and sample format, filtered by one CUDA graph launch
(dfttest2_b200_batch_create / _run of the C ABI).

    b = Batch([(flt_a, src_a, dst_a, FLOAT, 32), (flt_b, src_b, dst_b, INTEGER, 16), ...], tune=True)
    b.run()                      # on torch's current stream, asynchronous

``src`` and ``dst`` are CUDA tensors of shape (N, H, W) holding every frame of
one plane; a YUV clip contributes one entry per plane.  Tensors and filters
are kept alive by the batch.  With ``tune=True`` the kernel shape and unit
split of every group of jobs are timed on the batch itself at creation (the
timed runs write the outputs too); the choices are cached per process.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence

from . import _lib
from .plugin import Filter

__all__ = ["Batch"]


class Batch:
    def __init__(self, items: Sequence[tuple], tune: bool = True):
        import torch

        if not items:
            raise _lib.Error("empty clip list")
        self._lib = _lib.load()
        self._keep = []
        arr = (_lib.Clip * len(items))()
        for i, (flt, src, dst, sample_type, bits) in enumerate(items):
            if not isinstance(flt, Filter):
                raise TypeError("items must be (Filter, src, dst, sample_type, bits_per_sample)")
            if not (src.is_cuda and dst.is_cuda) or src.dim() != 3 or src.shape != dst.shape:
                raise ValueError("src and dst must be CUDA tensors of one (N, H, W) shape")
            if not (src.is_contiguous() and dst.is_contiguous()):
                raise ValueError("src and dst must be contiguous")
            n, h, w = src.shape
            es = src.element_size()
            c = arr[i]
            c.filter = flt.handle
            c.src = src.data_ptr()
            c.src_stride = w * es
            c.src_frame_bytes = h * w * es
            c.dst = dst.data_ptr()
            c.dst_stride = w * es
            c.dst_frame_bytes = h * w * es
            c.nframes, c.width, c.height = n, w, h
            c.sample_type, c.bits_per_sample = sample_type, bits
            self._keep.append((flt, src, dst))
        handle = ctypes.c_void_p()
        torch.cuda.current_stream().synchronize()  # inputs ready before the tuning runs read them
        _lib.check(self._lib.dfttest2_b200_batch_create(arr, len(items), _lib.BATCH_TUNE if tune else 0,
                                                        ctypes.byref(handle)))
        self.handle = handle.value

    def run(self, stream: int | None = None) -> None:
        import torch

        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        _lib.check(self._lib.dfttest2_b200_batch_run(self.handle, ctypes.c_void_p(stream)))

    def describe(self) -> tuple[int, str]:
        """(kernel launches per run, one line per group)."""
        buf = ctypes.create_string_buffer(1 << 16)
        n = self._lib.dfttest2_b200_batch_describe(self.handle, buf, len(buf))
        if n < 0:
            _lib.check(-n)
        return n, buf.value.decode()

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.dfttest2_b200_batch_free(self.handle)
            self.handle = None

    def __del__(self):
        self.close()
