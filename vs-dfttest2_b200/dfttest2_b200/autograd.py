"""Differentiable DFTTest for float clips on the GPU.

``DFTTestFunction.apply(clips, sigma, flt)`` filters a batch of clips
(C, N, H, W) float32 CUDA tensor with a per-bin sigma array
(2r+1, B, B/2+1) that can require grad; the backward pass runs the
adjoint kernel (dfttest2_b200_backward_planes), which recomputes block
spectra instead of storing them, and returns gradients w.r.t. the clips
and sigma.  ``flt`` is a :class:`dfttest2_b200.plugin.Filter` holding the
window, window spectrum and filter type.

Sigma units are those of the plugin argument (after the front end's
``wscale`` scaling, i.e. the 0-255 sample domain), laid out as the
reference's sigma array (python/dfttest2.py:293-315).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .plugin import Filter

__all__ = ["DFTTestFunction", "DFTTestModule", "frame_planes"]


def _dtype_of(struct) -> np.dtype:
    """numpy view of a ctypes plane structure (pointer arrays as uint64)."""
    names, formats, offsets = [], [], []
    for name, ctype in struct._fields_:
        names.append(name)
        offsets.append(getattr(struct, name).offset)
        if isinstance(ctype, type) and issubclass(ctype, ctypes.Array):
            formats.append(("u8", ctype._length_))  # pointer arrays
        elif ctype in (ctypes.c_int, ctypes.c_int32):
            formats.append("i4")
        elif ctype in (ctypes.c_ssize_t, ctypes.c_int64, ctypes.c_longlong):
            formats.append("i8")
        else:
            formats.append("u8")
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": ctypes.sizeof(struct)})


_PLANE_DT = _dtype_of(_lib.Plane)
_GRAD_PLANE_DT = _dtype_of(_lib.GradPlane)


def _frame_index(C: int, N: int, r: int) -> np.ndarray:
    """(C*N, 2r+1) flat frame index of every temporal tap of every output frame."""
    n = np.arange(N)[:, None]
    t = np.arange(2 * r + 1)[None, :]
    k = np.clip(n - r + t, 0, N - 1)  # clip-end clamp, cpu_source/getframe_impl.cpp:296-298
    return (np.arange(C)[:, None, None] * N + k[None]).reshape(C * N, 2 * r + 1)


def frame_planes(clips: torch.Tensor, out: torch.Tensor, r: int):
    """C-ABI plane list: every output frame of every (contiguous) clip."""
    C, N, H, W = clips.shape
    fb = H * W * clips.element_size()
    buf = np.zeros(C * N, _PLANE_DT)
    buf["src"][:, :2 * r + 1] = clips.data_ptr() + _frame_index(C, N, r).astype(np.uint64) * fb
    buf["src_stride"] = W * clips.element_size()
    buf["dst"] = out.data_ptr() + np.arange(C * N, dtype=np.uint64) * fb
    buf["dst_stride"] = W * out.element_size()
    buf["width"], buf["height"] = W, H
    return (_lib.Plane * (C * N)).from_buffer(buf)


def grad_planes(clips: torch.Tensor, grad_clips: torch.Tensor, grad_out: torch.Tensor, r: int):
    """C-ABI gradient plane list matching :func:`frame_planes` (float32, contiguous)."""
    C, N, H, W = clips.shape
    fb = H * W * 4
    idx = _frame_index(C, N, r).astype(np.uint64) * fb
    buf = np.zeros(C * N, _GRAD_PLANE_DT)
    buf["src"][:, :2 * r + 1] = clips.data_ptr() + idx
    buf["grad_src"][:, :2 * r + 1] = grad_clips.data_ptr() + idx
    buf["grad_dst"] = grad_out.data_ptr() + np.arange(C * N, dtype=np.uint64) * fb
    buf["src_stride"] = buf["grad_src_stride"] = buf["grad_dst_stride"] = W * 4
    buf["width"], buf["height"] = W, H
    return (_lib.GradPlane * (C * N)).from_buffer(buf)


class DFTTestFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, clips: torch.Tensor, sigma: torch.Tensor, flt: Filter):
        if clips.dtype != torch.float32 or not clips.is_cuda or clips.dim() != 4:
            raise ValueError("clips must be a (C, N, H, W) float32 CUDA tensor")
        clips = clips.contiguous()
        sigma = sigma.detach().to(torch.float32).contiguous()
        out = torch.empty_like(clips)
        planes = frame_planes(clips, out, flt.radius)
        stream = torch.cuda.current_stream(clips.device).cuda_stream
        lib = _lib.load()
        _lib.check(lib.dfttest2_b200_process_planes_sigma(flt.handle, planes, len(planes), _lib.FLOAT, 32,
                                                          ctypes.c_void_p(sigma.data_ptr()), ctypes.c_void_p(stream)))
        ctx.save_for_backward(clips, sigma)
        ctx.flt = flt
        return out

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        clips, sigma = ctx.saved_tensors
        flt = ctx.flt
        r = flt.radius
        grad_out = grad_out.contiguous().to(torch.float32)
        gin = torch.zeros_like(clips)
        gsig = torch.zeros_like(sigma)
        arr = grad_planes(clips, gin, grad_out, r)
        stream = torch.cuda.current_stream(clips.device).cuda_stream
        lib = _lib.load()
        _lib.check(lib.dfttest2_b200_backward_planes(flt.handle, arr, len(arr), ctypes.c_void_p(sigma.data_ptr()),
                                                     ctypes.c_void_p(gsig.data_ptr()), ctypes.c_void_p(stream)))
        return gin, gsig.reshape(ctx.saved_tensors[1].shape), None


class DFTTestModule(torch.nn.Module):
    """DFTTest with a learnable per-bin sigma array.

    ``args`` are the plugin arguments (e.g. from
    :func:`dfttest2_b200.frontend.plugin_arguments`); ``sigma_init`` is a
    scalar or a (2r+1, B, B/2+1) array."""

    def __init__(self, args: dict, sigma_init, device="cuda"):
        super().__init__()
        T = 2 * args["radius"] + 1
        B = args["block_size"]
        X = B // 2 + 1
        s = torch.as_tensor(sigma_init, dtype=torch.float32)
        if s.numel() == 1:
            s = s.reshape(1).expand(T * B * X).clone()
        self.sigma = torch.nn.Parameter(s.reshape(T, B, X).to(device))
        full = dict(args)
        full["sigma"] = [float(v) for v in self.sigma.detach().cpu().reshape(-1)]
        dev = torch.device(device)
        self.flt = Filter(device_id=dev.index or 0, **full)

    def forward(self, clips: torch.Tensor) -> torch.Tensor:
        return DFTTestFunction.apply(clips, self.sigma, self.flt)
