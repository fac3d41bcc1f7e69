"""User-level front end: ``DFTTest`` and ``DFTTest2``.

Restates the reference's ``python/dfttest2.py`` (vs-dfttest2) on top of the
``dfttest2_b200`` plugin namespace:

* ``DFTTest``  dfttest2.py:24-237  parameter checks, sigma functions from
  slocation / ssx / ssy / sst with the cube-root (or square-root)
  normalisation, backend selection;
* ``DFTTest2`` dfttest2.py:240-421 translation to plugin arguments: filter
  type from ftype / f0beta, radius and block step, the sigma array
  (ssystem 0 / 1), the window, ``wscale`` scaling of sigma / sigma2 /
  pmin / pmax, ``window_freq = RDFT(255 * window)`` and the plugin call;
* ``flatten`` / ``to_func``  dfttest2.py:424-452.

The check order and messages follow the reference.  ``plugin_arguments``
returns the translated arguments without filtering (used by tests and the
benchmark).
"""
from __future__ import annotations

import itertools
import math
from collections.abc import Callable, Sequence

from .backends import Backend, as_b200, select_backend
from .clip import FLOAT, INTEGER, Clip
from .helpers import get_location, get_sigma, get_window
from .plugin import dfttest2_b200

__all__ = ["DFTTest", "DFTTest2", "plugin_arguments", "flatten", "to_func"]


def DFTTest(
    clip: Clip,
    ftype: int = 0,
    sigma: float = 8.0,
    sigma2: float = 8.0,
    pmin: float = 0.0,
    pmax: float = 500.0,
    sbsize: int = 16,
    smode: int = 1,
    sosize: int = 12,
    tbsize: int = 3,
    swin: int = 0,
    twin: int = 7,
    sbeta: float = 2.5,
    tbeta: float = 2.5,
    zmean: bool = True,
    f0beta: float = 1.0,
    nlocation=None,
    alpha: float | None = None,
    slocation=None,
    ssx=None,
    ssy=None,
    sst=None,
    ssystem: int = 0,
    planes=None,
    backend=None,
) -> Clip:
    """2D/3D frequency-domain denoiser (interface of core.dfttest.DFTTest).

    See the reference's docstring (python/dfttest2.py:52-162) for every
    parameter; ``backend`` defaults to ``Backend.B200``.
    """
    fmt = clip.format
    if (
        clip.width == 0
        or clip.height == 0
        or (fmt.sample_type == INTEGER and fmt.bits_per_sample > 16)
        or (fmt.sample_type == FLOAT and fmt.bits_per_sample != 32)
    ):
        raise ValueError("only constant format 8-16 bit integer and 32 bit float input supported")
    if ftype < 0 or ftype > 4:
        raise ValueError("ftype must be 0, 1, 2, 3, or 4")
    if sbsize < 1:
        raise ValueError("sbsize must be greater than or equal to 1")
    if smode != 1:
        raise ValueError('"smode" must be 1')
    if sosize > sbsize // 2 and (sbsize % (sbsize - sosize) != 0):
        raise ValueError("spatial overlap greater than 50% requires that sbsize-sosize is a divisor of sbsize")
    if tbsize < 1:
        raise ValueError('"tbsize" must be at least 1')
    if not 0 <= swin <= 11:
        raise ValueError("swin must be between 0 and 11 (inclusive)")
    if not 0 <= twin <= 11:
        raise ValueError("twin must be between 0 and 11 (inclusive)")
    if nlocation is not None:
        raise ValueError('"nlocation" must be None')
    for name, loc in (("slocation", slocation), ("ssx", ssx), ("ssy", ssy), ("sst", sst)):
        if loc and len(loc) % 2 != 0:
            raise ValueError(f"number of elements in {name} must be a multiple of 2")
    if ssystem not in (0, 1):
        raise ValueError("ssystem must be 0 or 1")

    def norm(x: float) -> float:
        if slocation is not None and ssystem == 1:
            return x
        if tbsize == 1:
            return math.sqrt(x)
        return math.cbrt(x)

    if slocation is not None:
        sigma_norm = [to_func(flatten(slocation), norm, sigma)] * 3
    elif any(ss is not None for ss in (ssx, ssy, sst)):
        sigma_norm = [to_func(flatten(ss), norm, sigma) for ss in (ssx, ssy, sst)]
    else:
        sigma_norm = sigma

    return DFTTest2(
        clip=clip, ftype=ftype, sigma=sigma_norm, sigma2=sigma2, pmin=pmin, pmax=pmax, sbsize=sbsize,
        sosize=sosize, tbsize=tbsize, swin=swin, twin=twin, sbeta=sbeta, tbeta=tbeta, zmean=zmean, f0beta=f0beta,
        ssystem=ssystem, planes=planes, backend=select_backend(backend, sbsize, tbsize),
    )


def plugin_arguments(
    ftype: int = 0,
    sigma=8.0,
    sigma2: float = 8.0,
    pmin: float = 0.0,
    pmax: float = 500.0,
    sbsize: int = 16,
    sosize: int = 12,
    tbsize: int = 3,
    swin: int = 0,
    twin: int = 7,
    sbeta: float = 2.5,
    tbeta: float = 2.5,
    zmean: bool = True,
    f0beta: float = 1.0,
    ssystem: int = 0,
    full_sigma: bool = False,
    rdft=None,
) -> dict:
    """The plugin arguments DFTTest2 derives (python/dfttest2.py:262-341).

    ``full_sigma`` expands a flat sigma to the full array (what the CPU
    backends receive, dfttest2.py:364); ``rdft`` overrides the RDFT used
    for window_freq (defaults to the plugin's)."""
    if ftype == 0:
        if abs(f0beta - 1) < 0.00005:
            filter_type = 0
        elif abs(f0beta - 0.5) < 0.0005:
            filter_type = 6
        else:
            filter_type = 5
    else:
        filter_type = ftype

    radius = (tbsize - 1) // 2
    block_size = sbsize
    block_step = sbsize - sosize
    t_len = 2 * radius + 1
    y_len = block_size
    x_len = block_size // 2 + 1

    if not isinstance(sigma, Sequence) and not callable(sigma):
        sigma_norm = float(sigma)
    else:
        funcs = [sigma] if callable(sigma) else list(sigma)[:3]
        funcs += [funcs[-1]] * (3 - len(funcs))
        fx, fy, ft = funcs
        if ssystem == 0:
            st = [get_sigma(t, t_len, ft) for t in range(t_len)]
            sy = [get_sigma(y, y_len, fy) for y in range(y_len)]
            sx = [get_sigma(x, x_len, fx) for x in range(x_len)]
            sigma_norm = [a * b * c for a, b, c in itertools.product(st, sy, sx)]
        else:
            lt = [get_location(t, t_len) ** 2 for t in range(t_len)]
            ly = [get_location(y, y_len) ** 2 for y in range(y_len)]
            lx = [get_location(x, x_len) ** 2 for x in range(x_len)]
            inv_ndim = 1.0 / (3 if radius > 0 else 2)
            sigma_norm = [ft(math.sqrt((a + b + c) * inv_ndim)) for a, b, c in itertools.product(lt, ly, lx)]

    window = get_window(
        radius=radius, block_size=block_size, block_step=block_step, spatial_window_mode=swin,
        temporal_window_mode=twin, spatial_beta=sbeta, temporal_beta=tbeta,
    )
    wscale = math.fsum(w * w for w in window)
    if ftype < 2:
        if not isinstance(sigma_norm, list):
            sigma_norm *= wscale
        else:
            sigma_norm = [s * wscale for s in sigma_norm]
        sigma2 *= wscale
    if filter_type == 5:
        pmin = f0beta  # unscaled, as the reference
    else:
        pmin *= wscale
    pmax *= wscale

    shape = (block_size, block_size) if radius == 0 else (t_len, block_size, block_size)
    rdft = rdft or dfttest2_b200.RDFT
    window_freq = rdft([w * 255 for w in window], shape)
    if isinstance(sigma_norm, list):
        sigma_val = sigma_norm
    elif full_sigma:
        sigma_val = [sigma_norm] * (t_len * y_len * x_len)
    else:
        sigma_val = [sigma_norm]
    return dict(
        window=window, sigma=sigma_val, sigma2=sigma2, pmin=pmin, pmax=pmax, filter_type=filter_type,
        radius=radius, block_size=block_size, block_step=block_step, zero_mean=int(zmean),
        window_freq=window_freq if zmean else None,
    )


def DFTTest2(
    clip: Clip,
    ftype: int = 0,
    sigma=8.0,
    sigma2: float = 8.0,
    pmin: float = 0.0,
    pmax: float = 500.0,
    sbsize: int = 16,
    sosize: int = 12,
    tbsize: int = 3,
    swin: int = 0,
    twin: int = 7,
    sbeta: float = 2.5,
    tbeta: float = 2.5,
    zmean: bool = True,
    f0beta: float = 1.0,
    ssystem: int = 0,
    planes=None,
    backend=Backend.B200,
) -> Clip:
    """this interface is not stable (as in the reference)"""
    inst = as_b200(backend)
    radius = (tbsize - 1) // 2
    if radius not in range(4):
        raise ValueError("invalid radius (tbsize)")
    if sbsize not in (8, 16, 32):
        raise ValueError("invalid block_size (sbsize)")
    args = plugin_arguments(
        ftype=ftype, sigma=sigma, sigma2=sigma2, pmin=pmin, pmax=pmax, sbsize=sbsize, sosize=sosize, tbsize=tbsize,
        swin=swin, twin=twin, sbeta=sbeta, tbeta=tbeta, zmean=zmean, f0beta=f0beta, ssystem=ssystem,
    )
    return dfttest2_b200.DFTTest(clip, planes=planes, device_id=inst.device_id, num_streams=inst.num_streams, **args)


def flatten(data):
    if not data:
        return None
    if isinstance(data[0], (int, float)):
        return list(data)
    return list(itertools.chain.from_iterable(data))


def to_func(data, norm: Callable[[float], float], sigma: float) -> Callable[[float], float]:
    """Piecewise-linear sigma(location) through (location, sigma) knots,
    interpolating the normalised sigma values."""
    if data is None:
        return lambda _: norm(sigma)
    locations = data[::2]
    sigmas = data[1::2]
    packs = sorted(zip(locations, sigmas), key=lambda group: group[0])

    def func(x: float) -> float:
        for (x0, y0), (x1, y1) in itertools.pairwise(packs):
            if x <= x1:
                weight = (x - x0) / (x1 - x0)
                return (1 - weight) * norm(y0) + weight * norm(y1)
        raise ValueError(f"Value {x} out of range")

    return func
