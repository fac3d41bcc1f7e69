"""TEST INFRASTRUCTURE ONLY: DFTTest's per-plane pipeline in float64 torch.

A differentiable restatement used as the reference for the adjoint (the
gradient w.r.t. input pixels and the sigma array) and as a second FP64
forward.  Steps (reference semantics, vs-dfttest2):

* mirror padding without edge repeat       cpu_source/getframe_impl.cpp:22-65
  (torch's 'reflect' mode)
* gather + analysis window * scale         getframe_impl.cpp:105-156
* 3D real DFT, zero-mean, gain             cpu_source/kernel.hpp:1819-1952
* inverse DFT of the centre frame          kernel.hpp:1954-1983 (irfftn
  ignores the imaginary parts of the x-bins 0 and B/2, like the c2r codelet)
* synthesis window + overlap-add, / scale  getframe_impl.cpp:158-221
  (synthesis slice r, as the GPU backends)

Not part of the product; the product never imports this file.
"""
from __future__ import annotations

import math

import torch
import torch.nn.functional as F


def pad_size(n, B, S):
    return n + ((B - n % B) if n % B else 0) + 2 * max(B - S, S)


def _sqrt0(v):
    """sqrt with derivative 0 (not inf) where v == 0: the limit of the gain
    term m'(psd) d as d -> 0, which autograd of a plain sqrt turns into NaN."""
    pos = v > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, v, torch.ones_like(v))), torch.zeros_like(v))


def _pow0(v, p):
    pos = v > 0
    return torch.where(pos, torch.where(pos, v, torch.ones_like(v)) ** p, torch.zeros_like(v))


def gain(psd, sigma, ftype, sigma2, pmin, pmax):
    eps = 1e-15
    if ftype == 0:
        return torch.clamp((psd - sigma) / (psd + eps), min=0.0)
    if ftype == 1:
        return (psd >= sigma).to(psd.dtype) + 0.0 * sigma
    if ftype == 2:
        return sigma + 0.0 * psd
    if ftype == 3:
        inside = (psd >= pmin) & (psd <= pmax)
        return torch.where(inside, sigma + 0.0 * psd, torch.full_like(psd, sigma2))
    if ftype == 4:
        return sigma * _sqrt0(psd * (pmax / ((psd + pmin) * (psd + pmax) + eps)))
    if ftype == 5:
        return _pow0(torch.clamp((psd - sigma) / (psd + eps), min=0.0), pmin)
    return _sqrt0(torch.clamp((psd - sigma) / (psd + eps), min=0.0))


def dfttest_plane(frames, args, sigma=None, scale=255.0, synthesis_slice=None):
    """frames: (2r+1, H, W) float64 tensor (time clamp applied).
    sigma: optional (2r+1, B, B/2+1) float64 tensor overriding args['sigma'].
    Returns the (H, W) output before quantisation (acc / scale)."""
    r = args["radius"]
    T = 2 * r + 1
    B = args["block_size"]
    S = args["block_step"]
    X = B // 2 + 1
    _, H, W = frames.shape
    dev, dt = frames.device, torch.float64
    pw, ph = pad_size(W, B, S), pad_size(H, B, S)
    ox, oy = (pw - W) // 2, (ph - H) // 2
    x = F.pad(frames[None], (ox, pw - W - ox, oy, ph - H - oy), mode="reflect")[0]  # (T, ph, pw)
    blocks = x.unfold(1, B, S).unfold(2, B, S)  # (T, ny, nx, B, B)
    blocks = blocks.permute(1, 2, 0, 3, 4)  # (ny, nx, T, B, B)
    win = torch.tensor(args["window"], dtype=dt, device=dev).float().double().reshape(T, B, B)
    z = (torch.tensor(scale, dtype=torch.float32).double() * win) * blocks
    Z = torch.fft.rfftn(z, dim=(-3, -2, -1))
    if sigma is None:
        s = torch.tensor(args["sigma"], dtype=dt, device=dev).float().double()
        sigma = s.expand(T * B * X).reshape(T, B, X) if s.numel() == 1 else s.reshape(T, B, X)
    if args["zero_mean"]:
        wf = torch.tensor(args["window_freq"], dtype=dt, device=dev).float().double().reshape(T, B, X, 2)
        WF = torch.complex(wf[..., 0], wf[..., 1])
        g = Z[..., 0, 0, 0].real / WF[0, 0, 0].real
        gW = g[..., None, None, None] * WF
    else:
        gW = torch.zeros((), dtype=Z.dtype, device=dev)
    d = Z - gW
    psd = d.real ** 2 + d.imag ** 2
    m = gain(psd, sigma, args["filter_type"], float(args["sigma2"]), float(args["pmin"]), float(args["pmax"]))
    Y = m * d + gW
    y = torch.fft.irfftn(Y, s=(T, B, B), dim=(-3, -2, -1), norm="forward")
    syn = r if synthesis_slice is None else synthesis_slice
    out_blocks = y[:, :, r] * win[syn]  # (ny, nx, B, B)
    ny, nx = out_blocks.shape[:2]
    cols = out_blocks.reshape(ny * nx, B * B).T[None]  # (1, B*B, L)
    acc = F.fold(cols, output_size=(ph, pw), kernel_size=B, stride=S)[0, 0]
    return acc[oy:oy + H, ox:ox + W] / scale


def dfttest_clip(clip, args, sigma=None):
    """clip: (N, H, W) float64; returns (N, H, W) with the clip-end clamp."""
    r = args["radius"]
    N = clip.shape[0]
    outs = []
    for n in range(N):
        idx = [min(max(n - r + t, 0), N - 1) for t in range(2 * r + 1)]
        outs.append(dfttest_plane(clip[idx], args, sigma=sigma))
    return torch.stack(outs)
