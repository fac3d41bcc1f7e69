"""Host-side construction of the analysis window and of sigma-vs-frequency.

Restatement of the reference's ``python/helpers.py`` (vs-dfttest2), which in
turn follows DFTTest.cpp of VapourSynth-DFTTest.  The window coefficient
table and every formula are kept identical because they define the filter:

* ``COSINE_WINDOWS``  helpers.py:8-25  (cosine-sum coefficients)
* ``_i0``             helpers.py:28-40 (truncated Bessel I0 series)
* ``normalize``       helpers.py:45-47
* ``get_window_value``helpers.py:52-71
* ``get_window``      helpers.py:74-96
* ``get_location``    helpers.py:99-104
* ``get_sigma``       helpers.py:108-109

All arithmetic is FP64 on the host; the GPU never sees FP64.
"""
from __future__ import annotations

import itertools
import math
from collections.abc import Callable, Sequence

__all__ = ["get_location", "get_sigma", "get_window", "get_window_value", "normalize", "COSINE_WINDOWS"]

# window mode -> coefficients c_k of sum_k c_k cos(2 k pi x / N)
COSINE_WINDOWS: dict[int, tuple[float, ...]] = {
    0: (0.5, -0.5),  # Hanning
    1: (0.53836, -0.46164),  # Hamming
    2: (0.42, -0.5, 0.08),  # Blackman
    3: (0.35875, -0.48829, 0.14128, -0.01168),  # 4-term Blackman-Harris
    5: (
        0.27105140069342415,
        -0.433297939234486060,
        0.218122999543110620,
        -0.065925446388030898,
        0.010811742098372268,
        -7.7658482522509342e-4,
        1.3887217350903198e-5,
    ),  # 7-term Blackman-Harris
    6: (0.2810639, -0.5208972, 0.1980399),  # flat top
    10: (0.355768, -0.487396, 0.144232, -0.012604),  # Nuttall
    11: (0.3635819, -0.4891775, 0.1365995, -0.0106411),  # Blackman-Nuttall
}


def _i0(p: float) -> float:
    """Series for the modified Bessel function I0(p), stopped after 14 terms
    or once a term drops to 1e-8 (the reference's truncation)."""
    half = p / 2
    num = den = total = 1.0
    k = 1
    while True:
        num *= half
        den *= k
        term = num / den
        total += term * term
        k += 1
        if k >= 15 or term <= 1e-8:
            return total


def normalize(window: Sequence[float], size: int, step: int) -> list[float]:
    """Divide every tap by the root-sum-square of the taps that overlap it
    when blocks advance by ``step``."""
    norms = [math.sqrt(sum(window[h] ** 2 for h in range(rem, size, step))) for rem in range(step)]
    return [w / norms[q % step] for q, w in enumerate(window)]


def get_window_value(location: float, size: int, mode: int, beta: float) -> float:
    arg = math.pi * location / size
    coeffs = COSINE_WINDOWS.get(mode)
    if coeffs is not None:
        return sum(c * math.cos(2 * k * arg) for k, c in enumerate(coeffs))
    if mode == 4:  # Kaiser-Bessel
        v = 2 * location / size - 1
        return _i0(math.pi * beta * math.sqrt(1 - v * v)) / _i0(math.pi * beta)
    if mode == 7:  # rectangular
        return 1.0
    if mode == 8:  # Bartlett
        return 1.0 - 2.0 * abs(location - size / 2) / size
    if mode == 9:  # Bartlett-Hann
        return 0.62 - 0.48 * (location / size - 0.5) - 0.38 * math.cos(2 * arg)
    raise ValueError(f"unknown window: {mode}")


def get_window(
    radius: int,
    block_size: int,
    block_step: int,
    spatial_window_mode: int,
    spatial_beta: float,
    temporal_window_mode: int,
    temporal_beta: float,
) -> list[float]:
    """Separable (t, y, x) analysis window, flattened row-major, scaled by
    1/(sqrt(2r+1) * block_size) so that forward and inverse DFT need no
    normalisation."""
    t_len = 2 * radius + 1
    temporal = [get_window_value(i + 0.5, t_len, temporal_window_mode, temporal_beta) for i in range(t_len)]
    spatial = normalize(
        [get_window_value(i + 0.5, block_size, spatial_window_mode, spatial_beta) for i in range(block_size)],
        block_size,
        block_step,
    )
    scale = 1.0 / (math.sqrt(t_len) * block_size)
    spatial_2d = [a * b * scale for a, b in itertools.product(spatial, spatial)]
    return [t * s for t, s in itertools.product(temporal, spatial_2d)]


def get_location(position: float, length: int) -> float:
    """Normalised frequency in [0, 1] of bin ``position`` on an axis of
    ``length`` bins (the rfft axis is treated as a full period too)."""
    if length == 1:
        return 0.0
    half = length // 2
    return (length - position if position > half else position) / half


def get_sigma(position: float, length: int, func: Callable[[float], float]) -> float:
    return 1.0 if length == 1 else func(get_location(position, length))
