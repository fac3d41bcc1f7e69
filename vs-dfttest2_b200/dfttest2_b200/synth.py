"""Seeded synthetic clips for tests and the benchmark.

Clean content: 0.5 plus 16 drifting 2D sinusoids per plane,
    0.5 + sum_k a_k sin(2 pi (fx_k (x - dx_k t) + fy_k (y - dy_k t)) + phi_k)
with fx, fy ~ U[0, 0.25] cycles/px, a ~ U[0, 0.1], drift dx, dy ~ U[-1, 1]
px/frame, phi ~ U[0, 2 pi).  Noise: additive i.i.d. Gaussian, optional
salt-and-pepper.  Integer formats quantise round(clip(v, 0, 1) * peak).
No public dataset is involved.

The sum over sinusoids of each frame is one small matrix product
(sin(a+b) = sin a cos b + cos a sin b), so full-HD clips build quickly.
"""
from __future__ import annotations

import numpy as np

from .clip import FLOAT, Clip, VideoFormat, plane_dims


def sinusoid_plane(rng: np.random.Generator, n: int, h: int, w: int, k: int = 16) -> np.ndarray:
    fx = rng.uniform(0, 0.25, k)
    fy = rng.uniform(0, 0.25, k)
    a = rng.uniform(0, 0.1, k)
    dx = rng.uniform(-1, 1, k)
    dy = rng.uniform(-1, 1, k)
    phi = rng.uniform(0, 2 * np.pi, k)
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    out = np.empty((n, h, w), np.float32)
    for t in range(n):
        ax = 2 * np.pi * np.outer(xs, fx)                              # (w, k)
        ay = 2 * np.pi * np.outer(ys, fy) + (phi - 2 * np.pi * t * (fx * dx + fy * dy))  # (h, k)
        left = np.concatenate([np.sin(ay) * a, np.cos(ay) * a], axis=1)   # (h, 2k)
        right = np.concatenate([np.cos(ax), np.sin(ax)], axis=1).T        # (2k, w)
        out[t] = (0.5 + left @ right).astype(np.float32)
    return out


def make_clip(fmt: VideoFormat, width: int, height: int, frames: int, seed: int, noise_sigma: float,
              salt_pepper: float = 0.0) -> tuple[Clip, Clip]:
    """Returns (noisy, clean) clips; noise_sigma is in [0, 1] units."""
    rng = np.random.default_rng(seed)
    noisy, clean = [], []
    for p in range(fmt.num_planes):
        pw, ph = plane_dims(fmt, width, height, p)
        c = sinusoid_plane(rng, frames, ph, pw)
        v = c + rng.standard_normal(c.shape, dtype=np.float32) * np.float32(noise_sigma)
        if salt_pepper > 0:
            u = rng.random(c.shape, dtype=np.float32)
            v = np.where(u < salt_pepper / 2, 0.0, np.where(u < salt_pepper, 1.0, v)).astype(np.float32)
        if fmt.sample_type == FLOAT:
            noisy.append(v.astype(np.float32))
            clean.append(c)
        else:
            peak = (1 << fmt.bits_per_sample) - 1
            noisy.append(np.round(np.clip(v, 0, 1) * peak).astype(fmt.dtype))
            clean.append(np.round(np.clip(c, 0, 1) * peak).astype(fmt.dtype))
    return Clip(noisy, fmt), Clip(clean, fmt)


def make_clip_device(fmt: VideoFormat, width: int, height: int, frames: int, seed: int, noise_sigma: float,
                     device="cuda") -> list:
    """The same generator evaluated by torch on the device (float32 phases),
    for workloads too large to build on the host.  Returns the noisy planes
    as (N, H, W) CUDA tensors of the format's sample type."""
    import torch

    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    planes = []
    for p in range(fmt.num_planes):
        pw, ph = plane_dims(fmt, width, height, p)
        k = 16
        fx, fy, a, dx, dy = (torch.tensor(rng.uniform(lo, hi, k), dtype=torch.float32, device=device)
                             for lo, hi in ((0, 0.25), (0, 0.25), (0, 0.1), (-1, 1), (-1, 1)))
        phi = torch.tensor(rng.uniform(0, 2 * np.pi, k), dtype=torch.float32, device=device)
        xs = torch.arange(pw, dtype=torch.float32, device=device)
        ys = torch.arange(ph, dtype=torch.float32, device=device)
        ts = torch.arange(frames, dtype=torch.float32, device=device)
        ax = 2 * np.pi * torch.outer(xs, fx)                                      # (w, k)
        right = torch.cat([torch.cos(ax), torch.sin(ax)], dim=1).T                # (2k, w)
        ay = (2 * np.pi * torch.outer(ys, fy))[None] + (phi - 2 * np.pi * torch.outer(ts, fx * dx + fy * dy))[:, None]
        left = torch.cat([torch.sin(ay) * a, torch.cos(ay) * a], dim=2)           # (n, h, 2k)
        v = 0.5 + left @ right
        v += torch.randn(v.shape, generator=gen, device=device) * noise_sigma
        if fmt.sample_type == FLOAT:
            planes.append(v.contiguous())
        else:
            peak = (1 << fmt.bits_per_sample) - 1
            q = torch.round(torch.clamp(v, 0, 1) * peak)
            if fmt.bits_per_sample <= 8:
                planes.append(q.to(torch.uint8).contiguous())
            else:  # 16-bit samples travel as int16 tensors holding the unsigned bit pattern
                qi = q.to(torch.int32)
                planes.append(torch.where(qi >= 32768, qi - 65536, qi).to(torch.int16).contiguous())
    return planes


def batch_specs(seed: int = 0, nclips: int = 32, small: bool = False) -> list[dict]:
    """Clips of the multi-clip batching workload: resolution from {640x360,
    1280x720, 1920x1080, 3840x2160} (only 640x360 with `small`, a case
    where single clips leave the GPU partly idle), 4..32 frames, GRAYS /
    YUV420P8 / YUV420P16, sbsize in {8, 16, 32} with sosize = 3/4 sbsize,
    tbsize in {1, 3, 5}, ftype in {0, 1}, flat sigma ~ U[2, 16]."""
    from .clip import GRAYS, YUV420P8, YUV420P16

    rng = np.random.default_rng(seed)
    res = [(640, 360)] * 4 if small else [(640, 360), (1280, 720), (1920, 1080), (3840, 2160)]
    fmts = [GRAYS, YUV420P8, YUV420P16]
    out = []
    for i in range(nclips):
        w, h = res[int(rng.integers(4))]
        sb = int(rng.choice([8, 16, 32]))
        out.append(dict(width=w, height=h, frames=int(rng.integers(4, 33)), fmt=fmts[int(rng.integers(3))], sbsize=sb,
                        sosize=sb * 3 // 4, tbsize=int(rng.choice([1, 3, 5])), ftype=int(rng.integers(2)),
                        sigma=float(rng.uniform(2, 16)), seed=seed * 1000 + i))
    return out
