"""The ``dfttest2_b200`` plugin namespace: DFTTest, RDFT and Version.

Mirrors the functions the reference's GPU plugins register
(nvrtc_source/source.cpp:940-985):

    DFTTest(clip, window, sigma, sigma2, pmin, pmax, filter_type,
            radius=, block_size=, block_step=, zero_mean=, window_freq=,
            planes=, device_id=, num_streams=) -> clip
    RDFT(data, shape) -> list[float]
    Version() -> {"version": ...}

Arguments keep the reference's names, meanings and defaults; errors raise
:class:`Error` with the reference's messages.  The clip is a
:class:`dfttest2_b200.clip.Clip`; host clips go through the whole-clip host
path of the C ABI (each frame uploaded once), CUDA clips (torch tensors)
through the device-resident batched path.  Filtering is evaluated when
DFTTest is called rather than lazily per frame.
"""
from __future__ import annotations

import ctypes
from collections.abc import Sequence

import numpy as np

from . import _lib
from .clip import Clip, plane_dims

Error = _lib.Error


def _opt(v, default=-1):
    return default if v is None else int(v)


class Filter:
    """An instance of the C-ABI filter (DFTTestCreate ... DFTTestFree)."""

    def __init__(self, window, sigma, sigma2, pmin, pmax, filter_type, radius=None, block_size=None, block_step=None,
                 zero_mean=None, window_freq=None, device_id=None, num_streams=None, synthesis_slice=None):
        lib = _lib.load()
        p = _lib.Params()
        lib.dfttest2_b200_params_init(ctypes.byref(p))
        self._keep = []
        w = _lib.as_double_array(list(window))
        s = _lib.as_double_array(list(sigma) if isinstance(sigma, Sequence) or hasattr(sigma, "__len__") else [sigma])
        self._keep += [w, s]
        p.window, p.window_len = w, len(w)
        p.sigma, p.sigma_len = s, len(s)
        p.sigma2, p.pmin, p.pmax = float(sigma2), float(pmin), float(pmax)
        p.filter_type = int(filter_type)
        p.radius = _opt(radius)
        p.block_size = _opt(block_size)
        p.block_step = _opt(block_step)
        p.zero_mean = _opt(zero_mean)
        if window_freq is not None:
            wf = _lib.as_double_array(list(window_freq))
            self._keep.append(wf)
            p.window_freq, p.window_freq_len = wf, len(wf)
        p.device_id = _opt(device_id)
        p.num_streams = _opt(num_streams)
        p.synthesis_slice = _opt(synthesis_slice)
        handle = ctypes.c_void_p()
        _lib.check(lib.dfttest2_b200_create(ctypes.byref(p), ctypes.byref(handle)))
        self.handle = handle
        self.radius = 0 if radius is None else int(radius)
        self._lib = lib

    def set_precision(self, mode: str) -> None:
        """Arithmetic of the block transforms: "fp32" (CUDA-core FFT codelets,
        the default) or a tensor-core form "tc_fp16x3", "tc_bf16x3", "tc_tf32", "tc_bf16"
        (dfttest2_b200_set_precision)."""
        if mode not in _lib.PRECISION:
            raise Error(f"unknown precision mode {mode!r}; one of {sorted(_lib.PRECISION)}")
        _lib.check(self._lib.dfttest2_b200_set_precision(self.handle, _lib.PRECISION[mode]))
        self.precision = mode

    def check(self) -> None:
        """Waits for the filter's queued work and raises :class:`Error` if a
        kernel reported an internal failure (dfttest2_b200_check)."""
        _lib.check(self._lib.dfttest2_b200_check(self.handle))

    def set_wait_limit(self, iterations: int) -> None:
        """Iteration limit of the kernels' bounded device waits; negative
        restores the default (dfttest2_b200_set_wait_limit, for failure-path
        tests)."""
        _lib.check(self._lib.dfttest2_b200_set_wait_limit(self.handle, int(iterations)))

    def close(self):
        if self.handle:
            self._lib.dfttest2_b200_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- planes --------------------------------------------------------------
    def process_plane_host(self, src_frames: Sequence[np.ndarray], sample_type: int, bits: int) -> np.ndarray:
        """One output plane from its 2r+1 source planes (host arrays)."""
        src = [np.ascontiguousarray(a) for a in src_frames]
        h, w = src[0].shape
        out = np.empty_like(src[0])
        pl = _lib.Plane()
        for t, a in enumerate(src):
            pl.src[t] = a.ctypes.data
        pl.src_stride = src[0].strides[0]
        pl.dst = out.ctypes.data
        pl.dst_stride = out.strides[0]
        pl.width, pl.height = w, h
        _lib.check(self._lib.dfttest2_b200_process_plane_host(self.handle, ctypes.byref(pl), sample_type, bits))
        return out

    def process_frame_host_cached(self, frames: np.ndarray, n: int, plane_index: int, sample_type: int,
                                  bits: int) -> np.ndarray:
        """Output frame n of one plane of a host clip (N, H, W), as a
        frame-by-frame host would request it: source planes are cached on the
        device by (frame number, plane index)."""
        frames = np.ascontiguousarray(frames)
        N, h, w = frames.shape
        r = self.radius
        ids = [min(max(n - r + t, 0), N - 1) for t in range(2 * r + 1)]
        out = np.empty((h, w), frames.dtype)
        pl = _lib.Plane()
        for t, k in enumerate(ids):
            pl.src[t] = frames[k].ctypes.data
        pl.src_stride = frames.strides[1]
        pl.dst = out.ctypes.data
        pl.dst_stride = out.strides[0]
        pl.width, pl.height = w, h
        arr = (ctypes.c_int * len(ids))(*ids)
        _lib.check(self._lib.dfttest2_b200_process_plane_host_cached(self.handle, ctypes.byref(pl), arr, plane_index,
                                                                     sample_type, bits))
        return out

    def process_frame_planes_host_cached(self, clips: Sequence[np.ndarray], n: int, sample_type: int,
                                         bits: int) -> list:
        """Output frame n of every plane of a host clip (one (N, H_i, W_i)
        array per plane), in one call: the frame-by-frame path with the device
        frame cache, all planes in one launch."""
        clips = [np.ascontiguousarray(c) for c in clips]
        N = clips[0].shape[0]
        r = self.radius
        ids = [min(max(n - r + t, 0), N - 1) for t in range(2 * r + 1)]
        arr = (_lib.Plane * len(clips))()
        outs = []
        for pl, c in zip(arr, clips):
            _, h, w = c.shape
            o = np.empty((h, w), c.dtype)
            for t, k in enumerate(ids):
                pl.src[t] = c[k].ctypes.data
            pl.src_stride, pl.dst, pl.dst_stride = c.strides[1], o.ctypes.data, o.strides[0]
            pl.width, pl.height = w, h
            outs.append(o)
        pidx = (ctypes.c_int * len(clips))(*range(len(clips)))
        fids = (ctypes.c_int * len(ids))(*ids)
        _lib.check(self._lib.dfttest2_b200_process_frame_host_cached(self.handle, arr, len(clips), pidx, fids,
                                                                     sample_type, bits))
        return outs

    def process_clip_host(self, frames: np.ndarray, sample_type: int, bits: int) -> np.ndarray:
        """All frames of one plane, (N, H, W) host array."""
        frames = np.ascontiguousarray(frames)
        n, h, w = frames.shape
        out = np.empty_like(frames)
        _lib.check(self._lib.dfttest2_b200_process_clip_host(
            self.handle, frames.ctypes.data, frames.strides[1], frames.strides[0], out.ctypes.data, out.strides[1],
            out.strides[0], n, w, h, sample_type, bits))
        return out

    def process_clip_planes_host(self, planes: Sequence[np.ndarray], sample_type: int, bits: int) -> list:
        """All frames of several planes of one clip (each an (N, H_i, W_i) host
        array, same N and sample format) through one host pipeline."""
        planes = [np.ascontiguousarray(p) for p in planes]
        n = planes[0].shape[0]
        if any(p.shape[0] != n for p in planes):
            raise Error("all planes need the same number of frames")
        outs = [np.empty_like(p) for p in planes]
        arr = (_lib.HostPlane * len(planes))()
        for a, p, o in zip(arr, planes, outs):
            a.src, a.src_stride, a.src_frame_bytes = p.ctypes.data, p.strides[1], p.strides[0]
            a.dst, a.dst_stride, a.dst_frame_bytes = o.ctypes.data, o.strides[1], o.strides[0]
            a.width, a.height = p.shape[2], p.shape[1]
        _lib.check(self._lib.dfttest2_b200_process_clip_planes_host(self.handle, arr, len(planes), n, sample_type,
                                                                    bits))
        return outs

    def process_planes_device(self, planes: Sequence[dict], sample_type: int, bits: int, stream: int = 0) -> None:
        """Device pointers; each dict has src (list of 2r+1 pointers), src_stride,
        dst, dst_stride, width, height (strides in bytes).  Asynchronous."""
        arr = (_lib.Plane * max(1, len(planes)))()
        for i, d in enumerate(planes):
            for t, ptr in enumerate(d["src"]):
                arr[i].src[t] = ptr
            arr[i].src_stride = d["src_stride"]
            arr[i].dst = d["dst"]
            arr[i].dst_stride = d["dst_stride"]
            arr[i].width = d["width"]
            arr[i].height = d["height"]
        _lib.check(self._lib.dfttest2_b200_process_planes(self.handle, arr, len(planes), sample_type, bits,
                                                          ctypes.c_void_p(stream)))

    def process_clip_device(self, frames, sample_type: int, bits: int, out=None, stream: int | None = None):
        """All frames of one plane held in a CUDA tensor (N, H, W)."""
        import torch

        frames = frames.contiguous()
        n, h, w = frames.shape
        if out is None:
            out = torch.empty_like(frames)
        es = frames.element_size()
        r = self.radius
        planes = []
        for i in range(n):
            src = [frames[min(max(i - r + t, 0), n - 1)].data_ptr() for t in range(2 * r + 1)]
            planes.append(dict(src=src, src_stride=w * es, dst=out[i].data_ptr(), dst_stride=w * es, width=w,
                               height=h))
        if stream is None:
            stream = torch.cuda.current_stream(frames.device).cuda_stream
        self.process_planes_device(planes, sample_type, bits, stream)
        return out


class _Plugin:
    """Namespace object standing in for ``core.dfttest2_b200``."""

    Error = Error

    def DFTTest(self, clip: Clip, window, sigma, sigma2, pmin, pmax, filter_type, radius=None, block_size=None,
                block_step=None, zero_mean=None, window_freq=None, planes=None, device_id=None, num_streams=None,
                synthesis_slice=None) -> Clip:
        fmt = clip.format
        if fmt.sample_type == 0 and fmt.bits_per_sample > 16:
            raise Error("only 8-16 bit integer format input is supported")
        if fmt.sample_type == 1 and fmt.bits_per_sample != 32:
            raise Error("only 32-bit float format input is supported")
        process = [planes is None or len(planes) == 0] * 3
        if planes is not None:
            if isinstance(planes, int):
                planes = [planes]
            for p in planes:
                if p < 0 or p >= fmt.num_planes:
                    raise Error("plane index out of range")
                if process[p]:
                    raise Error("plane specified twice")
                process[p] = True
        flt = Filter(window, sigma, sigma2, pmin, pmax, filter_type, radius, block_size, block_step, zero_mean,
                     window_freq, device_id, num_streams, synthesis_slice)
        try:
            out = list(clip.planes)
            todo = [p for p in range(fmt.num_planes) if process[p]]
            if clip.on_gpu:
                for p in todo:
                    out[p] = flt.process_clip_device(clip.planes[p], fmt.sample_type, fmt.bits_per_sample)
            elif todo:
                # every processed plane through one host pipeline
                for p, o in zip(todo, flt.process_clip_planes_host([clip.planes[p] for p in todo], fmt.sample_type,
                                                                   fmt.bits_per_sample)):
                    out[p] = o
            if clip.on_gpu:
                flt.check()  # waits for the launches; raises if a kernel reported a failure
        finally:
            flt.close()
        return Clip(out, fmt)

    def RDFT(self, data, shape) -> list[float]:
        lib = _lib.load()
        shape = [int(s) for s in shape]
        ndim = len(shape)
        if ndim not in (1, 2, 3):
            raise Error('"shape" must be an array of ints with 1, 2 or 3 values')
        d = _lib.as_double_array(list(data))
        outer = 1
        for s in shape[:-1]:
            outer *= s
        n_out = outer * (shape[-1] // 2 + 1) * 2 if shape[-1] > 0 else 0
        out = (ctypes.c_double * max(1, n_out))()
        sh = (ctypes.c_int * ndim)(*shape)
        _lib.check(lib.dfttest2_b200_rdft(d, len(d), sh, ndim, out, n_out))
        return list(out[:n_out])

    def Version(self) -> dict:
        return {"version": _lib.load().dfttest2_b200_version().decode()}


dfttest2_b200 = _Plugin()
