"""TEST INFRASTRUCTURE ONLY: Python access to the two CPU oracles.

* ``ref_plane``   -- the reference's own CPU math (vs-dfttest2
  gcc_source/kernel.hpp, compiled unchanged by oracle/Makefile into
  oracle/_ref/libdfttest_ref.so, driven by oracle/ref_harness.cpp).  B=16
  only, FP32, with dfttest2_cpu's rounding and output conversion.
* ``ref_cufft_plane`` -- the reference's general-block-size GPU path
  (cuda_source/kernels.cu of vs-dfttest2 compiled unchanged, with cuFFT;
  oracle/ref_cufft.cu), the checker for block sizes 8 and 32.
* ``fp64_plane``  -- oracle/dfttest_oracle.c, an FP64 restatement of the
  same pipeline for any block size / radius; returns un-rounded values.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, as the checker.  Nothing in the product imports it.

Parity of the FP64 restatement is pinned against the reference build
(tests/test_oracle.py) and against committed fixtures generated with the
reference build (tests/golden/).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_longlong, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FP64_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB_V3 = os.path.join(HERE, "_ref", "libdfttest_ref.so")      # x86-64-v3 (AVX2)
REF_LIB_V4 = os.path.join(HERE, "_ref", "libdfttest_ref_v4.so")   # x86-64-v4 (AVX-512)


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_isa() -> str:
    """ISA of the reference build this host runs: the AVX-512 build where the
    CPU has the x86-64-v4 extensions (as dfttest2_cpu's dispatch picks its
    widest build, cpu_source/source.cpp:221-265), else the AVX2 build."""
    v4 = {"avx512f", "avx512bw", "avx512dq", "avx512vl"}
    return "x86-64-v4" if v4 <= _cpu_flags() and os.path.exists(REF_LIB_V4) else "x86-64-v3"



_fp64 = None
_ref = None


def build() -> None:
    """Build the oracle libraries (the reference part only when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_fp64():
    global _fp64
    if _fp64 is None:
        if not os.path.exists(FP64_LIB):
            build()
        lib = ctypes.CDLL(FP64_LIB)
        lib.oracle_dfttest_plane.restype = c_int
        lib.oracle_dfttest_plane.argtypes = [
            POINTER(c_void_p), c_int, c_int, c_longlong, c_int, c_double, POINTER(c_double), POINTER(c_double),
            POINTER(c_double), c_double, c_double, c_double, c_int, c_int, POINTER(c_double), c_int, c_int, c_int,
            c_int,
        ]
        _fp64 = lib
    return _fp64


def ref_available() -> bool:
    return os.path.exists(REF_LIB_V3)


def _load_ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError(f"{REF_LIB_V3} not built (needs the reference tree; see oracle/Makefile)")
        lib = ctypes.CDLL(REF_LIB_V4 if ref_isa() == "x86-64-v4" else REF_LIB_V3)
        lib.ref_dfttest_plane.restype = c_int
        lib.ref_dfttest_plane.argtypes = [
            POINTER(c_void_p), c_int, c_int, c_int, c_int, c_int, c_void_p, c_int, POINTER(c_double),
            POINTER(c_double), c_double, c_double, c_double, c_int, c_int, POINTER(c_double), c_int, c_int,
        ]
        _ref = lib
    return _ref


REF_CUFFT_LIB = os.path.join(HERE, "_ref", "libdfttest_ref_cufft.so")
_ref_cufft = None


def ref_cufft_available() -> bool:
    return os.path.exists(REF_CUFFT_LIB)


def ref_cufft_plane(frames, args: dict, bits: int) -> np.ndarray:
    """Output of the reference's cuFFT GPU path (cuda_source/kernels.cu +
    cuFFT, oracle/ref_cufft.cu) for one plane, any block size; runs on the
    current CUDA device.  Synthesis window slice r, as that backend."""
    global _ref_cufft
    if _ref_cufft is None:
        lib = ctypes.CDLL(REF_CUFFT_LIB)
        lib.ref_cufft_plane.restype = c_int
        lib.ref_cufft_plane.argtypes = [
            POINTER(c_void_p), c_int, c_int, c_int, c_int, c_int, c_void_p, c_int, POINTER(c_double),
            POINTER(c_double), c_int, c_double, c_double, c_double, c_int, c_int, POINTER(c_double), c_int, c_int,
            c_int,
        ]
        _ref_cufft = lib
    src = [np.ascontiguousarray(f) for f in frames]
    h, w = src[0].shape
    out = np.empty_like(src[0])
    ptrs = (c_void_p * len(src))(*[a.ctypes.data for a in src])
    win, win_p = _dbl(args["window"])
    sig, sig_p = _dbl(args["sigma"])
    wf_vals = args["window_freq"] if args["window_freq"] is not None else np.zeros(1)
    wf, wf_p = _dbl(wf_vals)
    st = 1 if src[0].dtype == np.float32 else 0
    rc = _ref_cufft.ref_cufft_plane(ptrs, w, h, w, st, 32 if st else bits, out.ctypes.data, w, win_p, sig_p,
                                    len(sig), args["sigma2"], args["pmin"], args["pmax"], args["filter_type"],
                                    args["zero_mean"], wf_p, args["radius"], args["block_size"], args["block_step"])
    if rc != 0:
        raise RuntimeError(f"reference cuFFT path failed ({rc})")
    return out


def _dbl(values) -> ctypes.Array:
    a = np.ascontiguousarray(np.asarray(values, dtype=np.float64))
    return a, a.ctypes.data_as(POINTER(c_double))


def _kind(arr: np.ndarray) -> int:
    return {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2}[arr.dtype]


def full_sigma(args: dict) -> np.ndarray:
    T = 2 * args["radius"] + 1
    B = args["block_size"]
    n = T * B * (B // 2 + 1)
    s = np.asarray(args["sigma"], dtype=np.float64)
    return np.full(n, s[0]) if s.size == 1 else s


def scale_of(arr: np.ndarray, bits: int) -> float:
    return 255.0 if arr.dtype == np.float32 else 1.0 / (1 << (bits - 8))


def ref_plane(frames, args: dict, bits: int) -> np.ndarray:
    """Reference CPU output for one plane; ``frames`` are the 2r+1 source
    planes (time clamp applied), ``args`` the plugin arguments."""
    lib = _load_ref()
    assert args["block_size"] == 16
    src = [np.ascontiguousarray(f) for f in frames]
    h, w = src[0].shape
    out = np.empty_like(src[0])
    ptrs = (c_void_p * len(src))(*[a.ctypes.data for a in src])
    win, win_p = _dbl(args["window"])
    sig, sig_p = _dbl(full_sigma(args))
    wf_vals = args["window_freq"] if args["window_freq"] is not None else np.zeros(1)
    wf, wf_p = _dbl(wf_vals)
    st = 1 if src[0].dtype == np.float32 else 0
    rc = lib.ref_dfttest_plane(ptrs, w, h, w, st, 32 if st else bits, out.ctypes.data, w, win_p, sig_p,
                               args["sigma2"], args["pmin"], args["pmax"], args["filter_type"], args["zero_mean"],
                               wf_p, args["radius"], args["block_step"])
    if rc != 0:
        raise RuntimeError("reference harness failed")
    return out


def fp64_plane(frames, args: dict, bits: int, synthesis_slice: int | None = None) -> np.ndarray:
    """FP64 oracle: un-rounded output (acc / scale) for one plane."""
    lib = _load_fp64()
    src = [np.ascontiguousarray(f) for f in frames]
    h, w = src[0].shape
    out = np.empty((h, w), np.float64)
    ptrs = (c_void_p * len(src))(*[a.ctypes.data for a in src])
    win, win_p = _dbl(args["window"])
    sig, sig_p = _dbl(full_sigma(args))
    wf_vals = args["window_freq"] if args["window_freq"] is not None else np.zeros(1)
    wf, wf_p = _dbl(wf_vals)
    syn = args["radius"] if synthesis_slice is None else synthesis_slice
    rc = lib.oracle_dfttest_plane(ptrs, w, h, w, _kind(src[0]), scale_of(src[0], bits),
                                  out.ctypes.data_as(POINTER(c_double)), win_p, sig_p, args["sigma2"], args["pmin"],
                                  args["pmax"], args["filter_type"], args["zero_mean"], wf_p, args["radius"],
                                  args["block_size"], args["block_step"], syn)
    if rc != 0:
        raise RuntimeError("fp64 oracle failed")
    return out


def quantize(values: np.ndarray, dtype, bits: int) -> np.ndarray:
    """Output conversion of cpu_source/getframe_impl.cpp:177-221 applied to
    FP64 values (integer: trunc(v + 0.5) clamped to [0, peak])."""
    if dtype == np.float32:
        return values.astype(np.float32)
    peak = (1 << bits) - 1
    return np.clip(np.trunc(values + 0.5), 0, peak).astype(dtype)


def clip_frames(planes: np.ndarray, n: int, radius: int):
    """The 2r+1 source planes of output frame n with the clip-end clamp
    (cpu_source/getframe_impl.cpp:296-298)."""
    N = planes.shape[0]
    return [planes[min(max(n - radius + t, 0), N - 1)] for t in range(2 * radius + 1)]
