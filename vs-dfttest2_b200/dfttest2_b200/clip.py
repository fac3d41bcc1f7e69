"""Minimal clip container standing in for a VapourSynth VideoNode.

A clip is a list of planes; plane p is an array of shape
(num_frames, height_p, width_p) in host memory (numpy) or on the GPU (a
torch CUDA tensor).  Formats carry what the plugin needs from
vapoursynth.VideoFormat: sample type, bits per sample, chroma subsampling
and the number of planes.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

INTEGER = 0
FLOAT = 1


@dataclass(frozen=True)
class VideoFormat:
    name: str
    sample_type: int
    bits_per_sample: int
    subsampling_w: int = 0
    subsampling_h: int = 0
    num_planes: int = 1

    @property
    def bytes_per_sample(self) -> int:
        return 4 if self.sample_type == FLOAT else (1 if self.bits_per_sample <= 8 else 2)

    @property
    def dtype(self):
        return np.float32 if self.sample_type == FLOAT else (np.uint8 if self.bits_per_sample <= 8 else np.uint16)


GRAY8 = VideoFormat("GRAY8", INTEGER, 8)
GRAY16 = VideoFormat("GRAY16", INTEGER, 16)
GRAYS = VideoFormat("GRAYS", FLOAT, 32)
YUV420P8 = VideoFormat("YUV420P8", INTEGER, 8, 1, 1, 3)
YUV420P10 = VideoFormat("YUV420P10", INTEGER, 10, 1, 1, 3)
YUV420P16 = VideoFormat("YUV420P16", INTEGER, 16, 1, 1, 3)
YUV444PS = VideoFormat("YUV444PS", FLOAT, 32, 0, 0, 3)


def plane_dims(fmt: VideoFormat, width: int, height: int, plane: int) -> tuple[int, int]:
    if plane == 0:
        return width, height
    return width >> fmt.subsampling_w, height >> fmt.subsampling_h


class Clip:
    def __init__(self, planes, fmt: VideoFormat):
        if len(planes) != fmt.num_planes:
            raise ValueError(f"{fmt.name} needs {fmt.num_planes} planes, got {len(planes)}")
        n, h, w = planes[0].shape
        for p, arr in enumerate(planes):
            pw, ph = plane_dims(fmt, w, h, p)
            if tuple(arr.shape) != (n, ph, pw):
                raise ValueError(f"plane {p} has shape {tuple(arr.shape)}, expected {(n, ph, pw)}")
        self.planes = list(planes)
        self.format = fmt
        self.num_frames = n
        self.width = w
        self.height = h

    @property
    def on_gpu(self) -> bool:
        return not isinstance(self.planes[0], np.ndarray)

    def __repr__(self) -> str:
        where = "cuda" if self.on_gpu else "host"
        return f"Clip({self.format.name}, {self.width}x{self.height}, {self.num_frames} frames, {where})"
