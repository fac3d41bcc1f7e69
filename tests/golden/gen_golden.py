#!/usr/bin/env python3
"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs only where the reference tree is present (read-only); its path comes from
the DFTTEST2_REF environment variable.

* Plugin arguments: the reference's own Python front end
  (python/dfttest2.py DFTTest -> DFTTest2, python/helpers.py) is imported
  with a stub ``vapoursynth`` module whose plugin object records the
  arguments of ``DFTTest`` instead of filtering.  ``RDFT`` in the stub is
  numpy's rfftn (the reference computes the same FP64 direct DFT in C++).
* Outputs: the reference's CPU math (gcc_source/kernel.hpp, built unchanged
  into oracle/_ref by oracle/Makefile) on seeded synthetic planes.

Writes:
  args_<case>.json      recorded plugin arguments per parameter set
  plane_<case>.npz      input planes (2r+1), recorded arguments, reference output
  helpers.json          windows / locations from python/helpers.py

Usage: python tests/golden/gen_golden.py
"""
from __future__ import annotations

import enum
import importlib
import json
import os
import sys
import types

import numpy as np

# the reference tree (vs-dfttest2 sources), given by the caller; no default
REF = os.environ.get("DFTTEST2_REF", "")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "vs-dfttest2_b200")]


class _Recorder:
    def __init__(self, name):
        self.name = name
        self.calls = []

    def RDFT(self, data, shape):
        a = np.asarray(data, dtype=np.float64).reshape(shape)
        out = np.fft.rfftn(a)
        return list(np.stack([out.real, out.imag], axis=-1).ravel())

    def DFTTest(self, clip, **kwargs):
        self.calls.append(kwargs)
        return clip


def import_reference(plugins):
    """Import the reference package with a stub vapoursynth module."""
    vs = types.ModuleType("vapoursynth")

    class SampleType(enum.IntEnum):
        INTEGER = 0
        FLOAT = 1

    class VideoNode:  # only used as a type annotation by the reference
        pass

    core = types.SimpleNamespace(**plugins)
    vs.SampleType = SampleType
    vs.VideoNode = VideoNode
    vs.core = core
    sys.modules["vapoursynth"] = vs
    sys.path.insert(0, REF)
    for m in [k for k in sys.modules if k == "python" or k.startswith("python.")]:
        del sys.modules[m]
    pkg = importlib.import_module("python")
    helpers = importlib.import_module("python.helpers")
    # python/dfttest2.py aliases TypeIs to typing.Any before Python 3.13, and
    # subscripting Any fails when flatten() runs; give it the real TypeIs.
    import typing_extensions

    importlib.import_module("python.dfttest2").TypeIs = typing_extensions.TypeIs
    return pkg, helpers, SampleType


class _Clip:
    def __init__(self, SampleType, sample_type, bits):
        self.width = 64
        self.height = 48
        self.format = types.SimpleNamespace(sample_type=SampleType(sample_type), bits_per_sample=bits)


# parameter sets: name -> (DFTTest kwargs, backend, sample_type, bits)
CASES = {
    "grays_default": (dict(), "CPU", 1, 32),
    "grays_t1": (dict(tbsize=1), "CPU", 1, 32),
    "gray16_sloc": (dict(slocation=[0.0, 12.0, 1 / 3, 28 / 3, 2 / 3, 20 / 3, 1.0, 4.0]), "CPU", 0, 16),
    "gray8_hard": (dict(ftype=1, sigma=20.0, tbsize=5, swin=2), "CPU", 0, 8),
    "gray16_mult": (dict(ftype=2, sigma=0.7, zmean=False, tbsize=3), "CPU", 0, 16),
    "grays_switch": (dict(ftype=3, sigma=1.1, sigma2=0.4, pmin=2.0, pmax=80.0, tbsize=3, swin=1), "CPU", 1, 32),
    "gray16_ft4": (dict(ftype=4, sigma=1.2, pmin=3.0, pmax=400.0, tbsize=7, swin=3, twin=7), "CPU", 0, 16),
    "grays_f0beta": (dict(f0beta=0.7, sigma=6.0, tbsize=3, swin=4, sbeta=3.0), "CPU", 1, 32),
    "gray8_sqrt": (dict(f0beta=0.5, sigma=10.0, tbsize=3, swin=5, sosize=8), "CPU", 0, 8),
    "grays_ssxyt": (dict(ssx=[0.0, 4.0, 1.0, 12.0], ssy=[0.0, 6.0, 1.0, 2.0], sst=[0.0, 8.0, 1.0, 8.0], tbsize=5,
                         swin=10, twin=0), "CPU", 1, 32),
    "gray16_ssystem1": (dict(slocation=[0.0, 4.0, 0.5, 10.0, 1.0, 2.0], ssystem=1, tbsize=3, swin=11), "CPU", 0, 16),
    "nvrtc_flat": (dict(sigma=5.0, tbsize=3), "NVRTC", 0, 16),
    "cufft_b8": (dict(sbsize=8, sosize=6, sigma=6.0, tbsize=3), "cuFFT", 1, 32),
    "cufft_b32": (dict(sbsize=32, sosize=24, sigma=6.0, tbsize=1, swin=8), "cuFFT", 1, 32),
}


def synthetic(seed, n, h, w, dtype, bits):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    frames = []
    for t in range(n):
        v = 0.5 + 0.1 * np.sin(2 * np.pi * (0.07 * (xx - 0.5 * t) + 0.11 * yy)) + 0.08 * np.sin(
            2 * np.pi * (0.19 * xx + 0.03 * (yy + t)) + 1.0)
        v += rng.standard_normal((h, w)) * 0.04
        if dtype == np.float32:
            frames.append(v.astype(np.float32))
        else:
            peak = (1 << bits) - 1
            frames.append(np.round(np.clip(v, 0, 1) * peak).astype(dtype))
    return frames


def main():
    from oracle import oracle as O

    if not REF or not os.path.isdir(os.path.join(REF, "python")):
        raise SystemExit("set DFTTEST2_REF to the vs-dfttest2 source tree")

    O.build()
    plugins = {name: _Recorder(name) for name in
               ("dfttest2_cpu", "dfttest2_gcc", "dfttest2_nvrtc", "dfttest2_cuda", "dfttest2_hip", "dfttest2_hiprtc")}
    pkg, helpers, SampleType = import_reference(plugins)
    Backend = pkg.Backend

    # helpers
    hj = {"windows": {}, "locations": {}}
    for mode in range(12):
        for size in (1, 3, 5, 7, 8, 16, 32):
            hj["windows"][f"{mode}_{size}"] = [helpers.get_window_value(i + 0.5, size, mode, 2.5) for i in range(size)]
    for length in (1, 3, 5, 9, 16, 17, 32):
        hj["locations"][str(length)] = [helpers.get_location(i, length) for i in range(length)]
    hj["get_window"] = {
        "r1_16_4_0_7": helpers.get_window(1, 16, 4, 0, 2.5, 7, 2.5),
        "r2_8_2_4_0": helpers.get_window(2, 8, 2, 4, 3.0, 0, 2.5),
        "r0_32_8_9_7": helpers.get_window(0, 32, 8, 9, 2.5, 7, 2.5),
    }
    with open(os.path.join(HERE, "helpers.json"), "w") as f:
        json.dump(hj, f)

    for idx, (case, (kw, backend, st, bits)) in enumerate(CASES.items()):
        for p in plugins.values():
            p.calls.clear()
        clip = _Clip(SampleType, st, bits)
        pkg.DFTTest(clip, backend=getattr(Backend, backend)(), **kw)
        calls = [c for p in plugins.values() for c in p.calls]
        assert len(calls) == 1, case
        args = {k: v for k, v in calls[0].items()}
        args.pop("planes", None)
        for k in ("window", "sigma", "window_freq"):
            if args.get(k) is not None:
                args[k] = [float(x) for x in args[k]]
        with open(os.path.join(HERE, f"args_{case}.json"), "w") as f:
            json.dump({"dfttest_kwargs": kw, "backend": backend, "sample_type": st, "bits": bits, "args": args}, f)
        if args.get("block_size", 16) != 16:
            continue  # the reference CPU math exists for block_size 16 only
        radius = args.get("radius", 0)
        dtype = np.float32 if st == 1 else (np.uint8 if bits <= 8 else np.uint16)
        frames = synthetic(100 + idx, 2 * radius + 1, 48, 64, dtype, bits)
        full = dict(args)
        full.setdefault("zero_mean", 1)
        full.setdefault("window_freq", None)
        full.setdefault("block_step", 16)
        out = O.ref_plane(frames, full, bits)
        np.savez_compressed(os.path.join(HERE, f"plane_{case}.npz"), frames=np.stack(frames), out=out)
        print(case, out.dtype, out.shape)


if __name__ == "__main__":
    main()
